// tma_interior.cuh -- the interior box of one half step with its planes staged
// through the Tensor Memory Accelerator.
//
// A CTA owns a TX x TY tile of the interior box and marches through a chunk
// of z planes.  Thread 0 streams every plane the chunk touches into a ring
// of S shared-memory stages with cp.async.bulk.tensor (one tensor map per
// field and tile shape, completion counted on one mbarrier per stage); the
// other threads never issue a global load.  A stage holds one plane's
//   A  the field differentiated along x and y, with a 4-cell x and a
//      (2,1) / (1,2) y halo              E phase: Hz   H phase: Ez
//   B  the field differentiated along x  E: Hy         H: Ey
//   C  the field differentiated along y  E: Hx         H: Ex
//   own-cell tiles                        E: m Ex Ey Ez H: Hx Hy Hz [dt/mu]
//      (OWN_SMEM; otherwise each thread loads its own cells directly,
//      before waiting for the plane, and the ring stage is half the size)
// B and C are also differentiated along z: their centre values of planes
// k-L .. k+U ride in a rolling register window, so a plane's stage is needed
// only while it is the window's newest plane and while it is plane k.  After
// each plane a __syncthreads() frees the stage of plane k and thread 0 refills
// it S planes ahead.  Each thread computes VX = 2 x cells from shared memory
// (8- or 16-byte reads at compile-time offsets) with exactly the fma forms of
// the interior body in stencil.cuh, so results are bit-identical to it, and
// stores its cells (and, in the E phase, the DFT ring) straight to HBM.
//
// Every mbarrier wait is bounded (TmaTiling::spin_limit polls; the handle's
// default is kMbarSpinLimit).  A wait that gives up sets bit 1 of the
// error word (the host reports MITTET_ERR_DEVICE_TIMEOUT) and the CTA's abort
// flag; after the next __syncthreads() every thread leaves the plane loop
// together, thread 0 issues no further copy and waits (again bounded) for
// the copies it has in flight, and the CTA returns.  CTAs that start, or are
// waiting, after the error word is set abort the same way at once.
//
// TMA rules kept: every x coordinate is a multiple of 4 elements (the
// interior box and the tiles start on multiples of 4, the halo is 4 wide),
// so each copy starts on a 16-byte boundary; the boxes' inner extents
// (TX or TX+8 elements) are multiples of 16 bytes; no multicast.
#pragma once
#include <cuda.h>

namespace mittet {

// Tensor maps of one phase: [0] A, [1] B, [2] C, [3 ..] own-cell tiles in the
// order E: m Ex Ey Ez, H: Hx Hy Hz dt/mu.  The model volumes (m, dt/mu) have
// no shot axis.
struct TmaMaps {
    CUtensorMap map[8];
};

// Tiles of the interior box handed to the TMA kernel.
struct TmaTiling {
    int x0, y0, z0, x1, y1, z1;  // interior box [x0, x1) x [y0, y1) x [z0, z1)
    int ntx, nty, zc;            // tiles in x and y, z planes per chunk
    int spin_limit;              // polls before an mbarrier wait gives up
};

// Stage geometry shared by the host (shared-memory size) and the kernel;
// OWN = own-cell tiles staged per plane (4) or loaded by the threads (0).
template <typename T, int TX, int TY, int OWN>
struct TmaStage {
    static constexpr int PA = TX + 8;  // pitch of the A and B tiles
    static constexpr int NA = PA * (TY + 3), NB = PA * TY, NC = TX * (TY + 3), NO = TX * TY;
    static constexpr int r32(int n) { return (n + 31) / 32 * 32; }
    static constexpr int OA = 0, OB = r32(NA), OC = OB + r32(NB), OO = OC + r32(NC);
    static constexpr int ELEMS = OO + OWN * NO;  // stage size in elements (multiple of 32)
    static constexpr size_t bytes(int S) { return (size_t)S * ELEMS * sizeof(T) + (size_t)S * 8; }
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Non-blocking test of the same phase: one poll costs a few cycles, so a
// wait limited to a few polls gives up before any copy can land.
__device__ __forceinline__ bool mbar_test_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, int x, int y, int z, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

constexpr int kMbarSpinLimit = 1 << 20;   // default try_wait polls before a wait gives up
constexpr int kMbarQuickLimit = 4096;     // limits below this poll with test_wait
constexpr int kMbarDrainLimit = 1 << 16;  // polls per in-flight copy when draining

template <typename T, int TX, int TY, int S, bool EPH, bool OWN_SMEM>
__global__ void __launch_bounds__((TX / 2) * TY) interior_tma_kernel(const PhaseArgs<T> a, const TmaTiling tl,
                                                                     const __grid_constant__ TmaMaps maps, int nown,
                                                                     int *__restrict__ err) {
    constexpr int VX = 2;
    using G = TmaStage<T, TX, TY, OWN_SMEM ? 4 : 0>;
    constexpr int PA = G::PA, L = EPH ? 2 : 1, U = EPH ? 1 : 2, YH = EPH ? 2 : 1;
    static_assert(S >= U + 2, "ring too shallow for the window");
    extern __shared__ __align__(128) unsigned char smraw[];
    T *sm = reinterpret_cast<T *>(smraw);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smraw + (size_t)S * G::ELEMS * sizeof(T));

    int b = blockIdx.x;
    const int tx = b % tl.ntx;
    b /= tl.ntx;
    const int ty = b % tl.nty, tz = b / tl.nty;
    const int X0 = tl.x0 + tx * TX, Y0 = tl.y0 + ty * TY;
    const int kb = tl.z0 + tz * tl.zc, ke = min(kb + tl.zc, tl.z1);
    const int shot = blockIdx.y;
    const int NP = (ke - kb) + L + U;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int lx = threadIdx.x * VX, ly = threadIdx.y;
    const int i0 = X0 + lx, j = Y0 + ly;
    const bool inside = i0 < tl.x1 && j < tl.y1;
    const int zs = shot * a.nz;
    const uint32_t bytes = (uint32_t)((G::NA + G::NB + G::NC + (OWN_SMEM ? nown * G::NO : 0)) * sizeof(T));

    // s_abort lets a wait that gave up release the CTA's other waits at once;
    // every decision to leave is taken through __syncthreads_or, so it is the
    // same in every thread.
    __shared__ int s_abort;
    int gave_up = 0;
    if (tid == 0) {
        for (int s = 0; s < S; s++) mbar_init(smem_addr(&bars[s]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    if (__syncthreads_or(tid == 0 && (*(volatile int *)err & 2))) return;  // an earlier CTA gave up: nothing issued

    int issued = 0;  // meaningful in thread 0 only
    auto issue = [&](int r) {
        const int s = r % S, p = kb - L + r;
        const uint32_t bar = smem_addr(&bars[s]);
        T *st = sm + (size_t)s * G::ELEMS;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(bar, bytes);
        tma_load_3d(smem_addr(st + G::OA), &maps.map[0], X0 - 4, Y0 - YH, zs + p, bar);
        tma_load_3d(smem_addr(st + G::OB), &maps.map[1], X0 - 4, Y0, zs + p, bar);
        tma_load_3d(smem_addr(st + G::OC), &maps.map[2], X0, Y0 - YH, zs + p, bar);
        for (int q = 0; q < (OWN_SMEM ? nown : 0); q++) {
            const bool model = EPH ? q == 0 : q == 3;
            tma_load_3d(smem_addr(st + G::OO + q * G::NO), &maps.map[3 + q], X0, Y0, model ? p : zs + p, bar);
        }
    };
    // tl.spin_limit below kMbarQuickLimit (a caller's short limit) polls with
    // the non-blocking test_wait, so the limit counts a few cycles each.
    const int spin = tl.spin_limit;
    const bool quick = spin < kMbarQuickLimit;
    auto wait = [&](int r) {
        const uint32_t bar = smem_addr(&bars[r % S]);
        const uint32_t par = (uint32_t)(r / S) & 1u;
        for (int it = 0; !(quick ? mbar_test_wait(bar, par) : mbar_try_wait(bar, par)); it++) {
            if (*(volatile int *)&s_abort || ((it & 1023) == 1023 && (*(volatile int *)err & 2))) {
                gave_up = 1;
                s_abort = 1;
                return;
            }
            if (it >= spin) {
                atomicOr(err, 2);
                gave_up = 1;
                s_abort = 1;
                return;
            }
        }
    };
    if (tid == 0)
        while (issued < NP && issued < S) issue(issued++);
    bool aborted = false;

    // window: centres of B and C for planes k-L .. k+U
    T wx[4][VX], wy[4][VX];
#pragma unroll
    for (int q = 0; q < L + U; q++) {
        wait(q);
        const T *st = sm + (size_t)(q % S) * G::ELEMS;
        ldv_rw<T, VX>(wx[q], st + G::OC + (ly + YH) * TX + lx);
        ldv_rw<T, VX>(wy[q], st + G::OB + ly * PA + lx + 4);
    }

    const long long sb = (long long)shot * a.fshot;
    const int py = a.px, pz = (int)a.plane;
    const T c1 = a.c1, c2 = a.c2, sg = a.sgn;
    const T ikx = a.ik[0], iky = a.ik[1], ikz = a.ik[2];
    const int slot = (EPH && a.ring_k > 0) ? (*a.d_step) % a.ring_k : 0;

    for (int i = 0; i < ke - kb; i++) {
        const int k = kb + i;
        const int rn = i + L + U, ro = i + L;
        const int c = k * pz + j * py + i0;
        // own cells of plane k: staged tiles, or plain loads issued before the wait
        T o0[VX], o1[VX], o2[VX], o3[VX];
        if constexpr (!OWN_SMEM) {
            if (inside) {
                if constexpr (EPH) {
                    ldv<T, VX>(o0, a.m + c);
                    ldv_rw<T, VX>(o1, a.f[0] + sb + c);
                    ldv_rw<T, VX>(o2, a.f[1] + sb + c);
                    ldv_rw<T, VX>(o3, a.f[2] + sb + c);
                } else {
                    ldv_rw<T, VX>(o0, a.f[3] + sb + c);
                    ldv_rw<T, VX>(o1, a.f[4] + sb + c);
                    ldv_rw<T, VX>(o2, a.f[5] + sb + c);
                    if (a.dtmu) {
                        ldv<T, VX>(o3, a.dtmu + c);
                    } else {
#pragma unroll
                        for (int v = 0; v < VX; v++) o3[v] = a.dtmu0;
                    }
                }
            } else {
                zerov<T, VX>(o0); zerov<T, VX>(o1); zerov<T, VX>(o2); zerov<T, VX>(o3);
            }
        }
        wait(rn);
        const T *sn = sm + (size_t)(rn % S) * G::ELEMS;
        const T *so = sm + (size_t)(ro % S) * G::ELEMS;
        ldv_rw<T, VX>(wx[3], sn + G::OC + (ly + YH) * TX + lx);
        ldv_rw<T, VX>(wy[3], sn + G::OB + ly * PA + lx + 4);
        const T *A = so + G::OA, *B = so + G::OB, *C = so + G::OC, *O = so + G::OO;
        // A row of this cell, columns x-2 .. x+3; B row, columns x-2 .. x+3
        T a6[6], b6[6];
        {
            const T *ar = A + (ly + YH) * PA + lx + 2;
            const T *br = B + ly * PA + lx + 2;
            T t[VX];
#pragma unroll
            for (int h = 0; h < 3; h++) {
                ldv_rw<T, VX>(t, ar + 2 * h);
                a6[2 * h] = t[0];
                a6[2 * h + 1] = t[1];
                ldv_rw<T, VX>(t, br + 2 * h);
                b6[2 * h] = t[0];
                b6[2 * h + 1] = t[1];
            }
        }
        if constexpr (EPH) {
            // rows y-2, y-1, y+1 of A (Hz) and C (Hx)
            T hzm2[VX], hzm1[VX], hzp1[VX], hxm2[VX], hxm1[VX], hxp1[VX];
            ldv_rw<T, VX>(hzm2, A + (ly + 0) * PA + lx + 4);
            ldv_rw<T, VX>(hzm1, A + (ly + 1) * PA + lx + 4);
            ldv_rw<T, VX>(hzp1, A + (ly + 3) * PA + lx + 4);
            ldv_rw<T, VX>(hxm2, C + (ly + 0) * TX + lx);
            ldv_rw<T, VX>(hxm1, C + (ly + 1) * TX + lx);
            ldv_rw<T, VX>(hxp1, C + (ly + 3) * TX + lx);
            T m[VX], ex[VX], ey[VX], ez[VX];
            if constexpr (OWN_SMEM) {
                ldv_rw<T, VX>(m, O + 0 * G::NO + ly * TX + lx);
                ldv_rw<T, VX>(ex, O + 1 * G::NO + ly * TX + lx);
                ldv_rw<T, VX>(ey, O + 2 * G::NO + ly * TX + lx);
                ldv_rw<T, VX>(ez, O + 3 * G::NO + ly * TX + lx);
            } else {
#pragma unroll
                for (int v = 0; v < VX; v++) { m[v] = o0[v]; ex[v] = o1[v]; ey[v] = o2[v]; ez[v] = o3[v]; }
            }
#pragma unroll
            for (int v = 0; v < VX; v++) {
                const T dyHz = d4(c1, c2, a6[2 + v], hzm1[v], hzp1[v], hzm2[v]);
                const T dyHx = d4(c1, c2, wx[2][v], hxm1[v], hxp1[v], hxm2[v]);
                const T dxHz = d4(c1, c2, a6[2 + v], a6[1 + v], a6[3 + v], a6[v]);
                const T dxHy = d4(c1, c2, b6[2 + v], b6[1 + v], b6[3 + v], b6[v]);
                const T dzHy = d4(c1, c2, wy[2][v], wy[1][v], wy[3][v], wy[0][v]);
                const T dzHx = d4(c1, c2, wx[2][v], wx[1][v], wx[3][v], wx[0][v]);
                const T mv = m[v];
                ex[v] = leap(T(1), sg * mv, curl2(dyHz, iky, dzHy, ikz), ex[v]);
                ey[v] = leap(T(1), sg * mv, curl2(dzHx, ikz, dxHz, ikx), ey[v]);
                ez[v] = leap(T(1), sg * mv, curl2(dxHy, ikx, dyHx, iky), ez[v]);
            }
            if (inside) {
                stv<T, VX>(a.fo[0] + sb + c, ex);
                stv<T, VX>(a.fo[1] + sb + c, ey);
                stv<T, VX>(a.fo[2] + sb + c, ez);
                if (a.ring_k > 0) {
                    const long long e = sb + c;
                    if (a.vmask & 1) stv_stream<T, VX>(a.ring + ring_index(a.ring_comp, a.ring_k, 0, e, slot), ex);
                    if (a.vmask & 2) stv_stream<T, VX>(a.ring + ring_index(a.ring_comp, a.ring_k, 1, e, slot), ey);
                    if (a.vmask & 4) stv_stream<T, VX>(a.ring + ring_index(a.ring_comp, a.ring_k, 2, e, slot), ez);
                }
            }
        } else {
            // rows y-1, y+1, y+2 of A (Ez) and C (Ex)
            T ezm1[VX], ezp1[VX], ezp2[VX], exm1[VX], exp1[VX], exp2[VX];
            ldv_rw<T, VX>(ezm1, A + (ly + 0) * PA + lx + 4);
            ldv_rw<T, VX>(ezp1, A + (ly + 2) * PA + lx + 4);
            ldv_rw<T, VX>(ezp2, A + (ly + 3) * PA + lx + 4);
            ldv_rw<T, VX>(exm1, C + (ly + 0) * TX + lx);
            ldv_rw<T, VX>(exp1, C + (ly + 2) * TX + lx);
            ldv_rw<T, VX>(exp2, C + (ly + 3) * TX + lx);
            T hx[VX], hy[VX], hz[VX], dm[VX];
            if constexpr (OWN_SMEM) {
                ldv_rw<T, VX>(hx, O + 0 * G::NO + ly * TX + lx);
                ldv_rw<T, VX>(hy, O + 1 * G::NO + ly * TX + lx);
                ldv_rw<T, VX>(hz, O + 2 * G::NO + ly * TX + lx);
                if (nown > 3) {
                    ldv_rw<T, VX>(dm, O + 3 * G::NO + ly * TX + lx);
                } else {
#pragma unroll
                    for (int v = 0; v < VX; v++) dm[v] = a.dtmu0;
                }
            } else {
#pragma unroll
                for (int v = 0; v < VX; v++) { hx[v] = o0[v]; hy[v] = o1[v]; hz[v] = o2[v]; dm[v] = o3[v]; }
            }
#pragma unroll
            for (int v = 0; v < VX; v++) {
                const T ez = a6[2 + v];
                const T dyEz = d4(c1, c2, ezp1[v], ez, ezp2[v], ezm1[v]);
                const T dyEx = d4(c1, c2, exp1[v], wx[1][v], exp2[v], exm1[v]);
                const T dxEz = d4(c1, c2, a6[3 + v], ez, a6[4 + v], a6[1 + v]);
                const T dxEy = d4(c1, c2, b6[3 + v], b6[2 + v], b6[4 + v], b6[1 + v]);
                const T dzEy = d4(c1, c2, wy[2][v], wy[1][v], wy[3][v], wy[0][v]);
                const T dzEx = d4(c1, c2, wx[2][v], wx[1][v], wx[3][v], wx[0][v]);
                const T dmv = dm[v];
                hx[v] = leap(T(1), -sg * dmv, curl2(dyEz, iky, dzEy, ikz), hx[v]);
                hy[v] = leap(T(1), -sg * dmv, curl2(dzEx, ikz, dxEz, ikx), hy[v]);
                hz[v] = leap(T(1), -sg * dmv, curl2(dxEy, ikx, dyEx, iky), hz[v]);
            }
            if (inside) {
                stv<T, VX>(a.fo[3] + sb + c, hx);
                stv<T, VX>(a.fo[4] + sb + c, hy);
                stv<T, VX>(a.fo[5] + sb + c, hz);
            }
        }
#pragma unroll
        for (int v = 0; v < VX; v++) {
            wx[0][v] = wx[1][v]; wx[1][v] = wx[2][v]; wx[2][v] = wx[3][v];
            wy[0][v] = wy[1][v]; wy[1][v] = wy[2][v]; wy[2][v] = wy[3][v];
        }
        if (__syncthreads_or(gave_up)) {  // every thread is done with plane k's stage
            aborted = true;
            break;
        }
        if (tid == 0)
            while (issued < NP && issued < i + L + 1 + S) issue(issued++);
    }
    if (tid == 0 && aborted) {  // left the loop early: drain the last S copies, bounded
        for (int r = max(0, issued - S); r < issued; r++) {
            const uint32_t bar = smem_addr(&bars[r % S]);
            for (int it = 0; it < kMbarDrainLimit && !mbar_try_wait(bar, (uint32_t)(r / S) & 1u); it++) {
            }
        }
    }
}

}  // namespace mittet
