// stencil.cuh -- the two half-step kernels of the (2,4) Yee + CPML update.
//
// Work decomposition.  The grid of one phase is split on the host into an
// interior box (no CPML profile, no psi slab, every component inside its
// update range, every derivative defined) cut into whole tiles, six faces
// around it that need the reference's CPML/range handling along one axis
// only, and twelve edge/corner boxes that need it along several.  The body
// is one template specialised by a mask GM of the axes handled generally, so
// the interior (GM = 0) is straight-line code, a face carries one axis's
// CPML terms, and only edges and corners (GM = 7) pay for all of them.
// Five launches per phase (interior, x faces, y faces, z faces, edges), each
// with its own thread-tile shape; blockIdx.x enumerates tiles through a TileMap in global
// memory, blockIdx.y is the shot.  The interior box's x edges lie on 32-cell
// (128-byte) line boundaries inside the exact interior (multiples of 4 cells
// on grids too narrow for that), so its last tile in x and y may be
// partial.  Every body uses the same explicit fma forms, so a cell gets
// bit-identical results whichever body computes it.
//
// Thread mapping: a BX x BY block covers one tile in (x, y); each thread owns
// VX consecutive x cells (one aligned float2/float4/double2 per field and
// plane) and marches through the tile's ZC z planes, keeping the four planes
// of the two fields it differentiates along z in a rolling register window,
// so each plane costs one new load of each.  x neighbours come from the
// aligned vectors at i0-VX, i0, i0+VX; y neighbours are whole vectors.  All
// loads of a plane are issued before its first store (every pointer is
// __restrict__, fields read in a phase are never written in it), and the
// psi slabs are loaded with the fields, so a warp keeps ~17 independent
// 8-16 byte loads in flight per plane.
//
// E half step (ncver0027/cpu_eh_field_cpml42.f90:114-158, cpu_cpml4.f90:271-361):
//   Ex = ca_x Ex + s cb_x (Dy(Hz)/kedy - Dz(Hy)/kedz),  cyclic for Ey, Ez,
//   D(F)[v] = c1 (F[v]-F[v-1]) + c2 (F[v+1]-F[v-2]),
//   ca = (1-h)/(1+h), cb = m/(1+h), h = esig_axis * m / 2,  m = 2 w0 dt / sigma;
//   in the slabs psi = be psi + ce/d D(F) and E += / -= cb psi (x, then y, then z).
// H half step (cpu_eh_field_cpml42.f90:210-253, cpu_cpml4.f90:384-474):
//   Hx = da_x Hx - s db_x (D+y(Ez)/khdy - D+z(Ey)/khdz),  cyclic,
//   D+(F)[v] = c1 (F[v+1]-F[v]) + c2 (F[v+2]-F[v-1]),
//   da = (1-h)/(1+h), db = (dt/mu)/(1+h), h = msig_axis * m / 2.
#pragma once

namespace mittet {

// Boxes of one phase, in the order their tiles are enumerated: the interior
// box, the two x faces, the two y faces, the two z faces (CPML / range
// handling along one axis only), then the edge and corner boxes (general
// handling).  kind = mask of the axes that need general handling (0
// interior, 1/2/4 faces, 7 general).  Part p (0 interior, 1 x faces, 2 y
// faces, 3 z faces, 4 edges) is boxes [pbox[p], pbox[p+1]), tiles
// [start[pbox[p]], start[pbox[p+1]]).
constexpr int kParts = 5;
struct TileMap {
    int nbox;
    int zc;            // z planes per tile (each thread marches through them)
    int pbox[kParts + 1];
    int start[25];     // first tile of each box
    int kind[24];
    int lo[24][3], hi[24][3];
    int ntx[24], nty[24];
};

template <typename T, int VX>
struct VecT;
template <> struct VecT<float, 2> { using type = float2; };
template <> struct VecT<float, 4> { using type = float4; };
template <> struct VecT<double, 2> { using type = double2; };

template <typename T, int VX>
__device__ __forceinline__ void ldv(T (&dst)[VX], const T *__restrict__ p) {
    using V = typename VecT<T, VX>::type;
    const V v = __ldg(reinterpret_cast<const V *>(p));
    const T *s = reinterpret_cast<const T *>(&v);
#pragma unroll
    for (int q = 0; q < VX; q++) dst[q] = s[q];
}
// Loads of values this launch may also write (fields, psi).  CG = false:
// the read-only path (every launch of the stepped graph only reads the other
// phase's fields).  CG = true: L2-coherent loads (ld.global.cg), for a
// persistent kernel in which the same array is written by another CTA in an
// earlier phase of the same launch.
template <typename T, int VX, bool CG>
__device__ __forceinline__ void ldf(T (&dst)[VX], const T *__restrict__ p) {
    using V = typename VecT<T, VX>::type;
    const V v = CG ? __ldcg(reinterpret_cast<const V *>(p)) : __ldg(reinterpret_cast<const V *>(p));
    const T *s = reinterpret_cast<const T *>(&v);
#pragma unroll
    for (int q = 0; q < VX; q++) dst[q] = s[q];
}
template <typename T, bool CG>
__device__ __forceinline__ T ldx(const T *__restrict__ p) {
    return CG ? __ldcg(p) : __ldg(p);
}
template <typename T, int VX>
__device__ __forceinline__ void ldv_rw(T (&dst)[VX], const T *__restrict__ p) {
    using V = typename VecT<T, VX>::type;
    const V v = *reinterpret_cast<const V *>(p);
    const T *s = reinterpret_cast<const T *>(&v);
#pragma unroll
    for (int q = 0; q < VX; q++) dst[q] = s[q];
}
template <typename T, int VX>
__device__ __forceinline__ void stv(T *__restrict__ p, const T (&src)[VX]) {
    using V = typename VecT<T, VX>::type;
    V v;
    T *d = reinterpret_cast<T *>(&v);
#pragma unroll
    for (int q = 0; q < VX; q++) d[q] = src[q];
    *reinterpret_cast<V *>(p) = v;
}
// Streaming store (evict-first in L2) for the DFT ring: nothing reads it
// before the flush, ring_k steps later, so its lines should not push the
// fields' halo rows out of L2.
template <typename T, int VX>
__device__ __forceinline__ void stv_stream(T *__restrict__ p, const T (&src)[VX]) {
    using V = typename VecT<T, VX>::type;
    V v;
    T *d = reinterpret_cast<T *>(&v);
#pragma unroll
    for (int q = 0; q < VX; q++) d[q] = src[q];
    __stcs(reinterpret_cast<V *>(p), v);
}
template <typename T, int VX>
__device__ __forceinline__ void zerov(T (&d)[VX]) {
#pragma unroll
    for (int q = 0; q < VX; q++) d[q] = T(0);
}

// psi values o .. o+VX-1 of the lanes in mask: one vector access when every
// lane is active, else one scalar access per active lane.  A cell's psi is
// read once, before its owner thread writes it, and by no other thread, so
// the read-only path is valid.
template <typename T, int VX, bool CG>
__device__ __forceinline__ void ld_psi(T (&d)[VX], const T *__restrict__ p, int o, unsigned mask) {
    if (mask == (1u << VX) - 1u) {
        ldf<T, VX, CG>(d, p + o);
    } else {
#pragma unroll
        for (int v = 0; v < VX; v++) d[v] = (mask >> v & 1) ? ldx<T, CG>(p + o + v) : T(0);
    }
}
template <typename T, int VX>
__device__ __forceinline__ void st_psi(T *__restrict__ p, int o, const T (&s)[VX], unsigned mask) {
    if (mask == (1u << VX) - 1u) {
        stv<T, VX>(p + o, s);
    } else {
#pragma unroll
        for (int v = 0; v < VX; v++)
            if (mask >> v & 1) p[o + v] = s[v];
    }
}

template <int VX>
__device__ __forceinline__ unsigned xmask(int i0, int lo, int hi) {
    unsigned m = 0;
#pragma unroll
    for (int v = 0; v < VX; v++) m |= (unsigned)(i0 + v >= lo && i0 + v < hi) << v;
    return m;
}

// Explicit fma forms shared by both bodies.
template <typename T>
__device__ __forceinline__ T d4(T c1, T c2, T a, T b, T c, T d) {  // c1 (a-b) + c2 (c-d)
    return fma(c1, a - b, c2 * (c - d));
}
template <typename T>
__device__ __forceinline__ T curl2(T a, T ia, T b, T ib) {  // a ia - b ib
    return fma(a, ia, -(b * ib));
}
template <typename T>
__device__ __forceinline__ T leap(T ca, T sgcb, T x, T e) {  // ca e + (s cb) x
    return fma(sgcb, x, ca * e);
}

// Minimum resident blocks per SM (__launch_bounds__) of a body, NT threads:
// marching interior bodies get up to 80 (VX = 2 FP32) or 128 registers; the
// marching face and edge bodies carry psi and profile state and get up to
// 128 or 168 (3 x 128 threads per SM) instead of spilling; the single-plane
// bodies hold no window, so the interior fits 64 or 80 registers and the
// general ones 80 or 128.
template <typename T, int VX, int NT, int GM, int BZ>
constexpr int part_min_blocks() {
    const bool narrow = sizeof(T) == 4 && VX == 2;
    if (BZ > 0) return GM == 0 ? (narrow ? 1024 : 768) / NT : (narrow ? 768 : 512) / NT;
    if (BZ == -1 && GM == 0) return 512 / NT;  // the prefetching interior holds two planes
    if (BZ == -2 && GM == 0) return 768 / NT;  // the interior held to 85 registers: 6 x 128 threads per SM
    return GM == 0 ? (narrow ? 768 : 512) / NT : (narrow ? 512 : 384) / NT;
}

// ------------------------------------------------------------------ E phase
template <typename T, int VX, int GM, bool ONE, bool CG = false>
__device__ __forceinline__ void e_cells(const PhaseArgs<T> &a, int shot, int i0, int j, int kb, int ke,
                                        int step = -1) {
    const long long sb = (long long)shot * a.fshot;
    const T *__restrict__ Ex = a.f[0] + sb;
    const T *__restrict__ Ey = a.f[1] + sb;
    const T *__restrict__ Ez = a.f[2] + sb;
    T *__restrict__ Exo = a.fo[0] + sb;
    T *__restrict__ Eyo = a.fo[1] + sb;
    T *__restrict__ Ezo = a.fo[2] + sb;
    const T *__restrict__ Hx = a.f[3] + sb;
    const T *__restrict__ Hy = a.f[4] + sb;
    const T *__restrict__ Hz = a.f[5] + sb;
    const T *__restrict__ M = a.m;
    const T *__restrict__ P = a.prof;
    const int py = a.px, pz = (int)a.plane, nx = a.nx, ny = a.ny, nz = a.nz, ps = a.nmax;
    const T c1 = a.c1, c2 = a.c2, sg = a.sgn;

    // GM bit 0/1/2: general handling along x/y/z; a clear bit means every
    // cell of the box is interior along that axis (no CPML profile, no psi
    // slab, inside every update range, derivative defined).
    constexpr bool GX = (GM & 1) != 0, GY = (GM & 2) != 0, GZ = (GM & 4) != 0;
    T esh_x[VX], ik_x[VX];
    T esh_y, ik_y;
    if constexpr (GX) {
        ldv<T, VX>(esh_x, P + 0 * ps + i0);
        ldv<T, VX>(ik_x, P + 6 * ps + i0);
    } else {
#pragma unroll
        for (int v = 0; v < VX; v++) { esh_x[v] = T(0); ik_x[v] = a.ik[0]; }
    }
    if constexpr (GY) {
        esh_y = __ldg(P + 8 * ps + j);
        ik_y = __ldg(P + 14 * ps + j);
    } else {
        esh_y = T(0);
        ik_y = a.ik[1];
    }
    const bool vy = GY ? ((j >= 2) && (j + 1 < ny)) : true;
    const bool has_l = GX ? (i0 >= VX) : true;
    const bool has_r = GX ? (i0 + VX < nx) : true;
    unsigned vxm = (1u << VX) - 1u;
    if constexpr (GX) {
        vxm = 0;
#pragma unroll
        for (int v = 0; v < VX; v++) vxm |= (unsigned)(i0 + v >= 2 && i0 + v + 1 < nx) << v;
    }
    const DBox U0 = a.upd[0], U1 = a.upd[1], U2 = a.upd[2];
    const unsigned all = (1u << VX) - 1u;
    const unsigned ux = (!GY || (j >= U0.lo[1] && j < U0.hi[1])) ? (GX ? xmask<VX>(i0, U0.lo[0], U0.hi[0]) : all) : 0u;
    const unsigned uy = (!GY || (j >= U1.lo[1] && j < U1.hi[1])) ? (GX ? xmask<VX>(i0, U1.lo[0], U1.hi[0]) : all) : 0u;
    const unsigned uz = (!GY || (j >= U2.lo[1] && j < U2.hi[1])) ? (GX ? xmask<VX>(i0, U2.lo[0], U2.hi[0]) : all) : 0u;
    const DSlab S0 = a.slab[0], S1 = a.slab[1], S2 = a.slab[2];
    unsigned sxm = 0;
    if constexpr (GX) {
#pragma unroll
        for (int v = 0; v < VX; v++) sxm |= (unsigned)(slab_local(S0, i0 + v) >= 0) << v;
        if (GY && !(j >= S0.other.lo[1] && j < S0.other.hi[1])) sxm = 0u;
    }
    const int ly = GY ? slab_local(S1, j) : -1;
    const unsigned sym = ly >= 0 ? (GX ? xmask<VX>(i0, S1.other.lo[0], S1.other.hi[0]) : all) : 0u;
    const unsigned szm = GZ ? ((!GY || (j >= S2.other.lo[1] && j < S2.other.hi[1])) ? (GX ? xmask<VX>(i0, S2.other.lo[0], S2.other.hi[0]) : all) : 0u) : 0u;
    const int col = j * py + i0;

    // psi recurrence coefficients of the x and y slabs (fixed along z) and
    // this shot's psi slabs.
    T be_x[VX], ced_x[VX];
    int lx[VX];
    T be_y = T(0), ced_y = T(0);
    if constexpr (GX) {
        ldv<T, VX>(be_x, P + 2 * ps + i0);
        ldv<T, VX>(ced_x, P + 3 * ps + i0);
#pragma unroll
        for (int v = 0; v < VX; v++) lx[v] = slab_local(S0, i0 + v);
    }
    if constexpr (GY) {
        be_y = __ldg(P + 10 * ps + j);
        ced_y = __ldg(P + 11 * ps + j);
    }
    T *__restrict__ sx0 = a.psi[0][0] + shot * a.pshot[0];
    T *__restrict__ sx1 = a.psi[0][1] + shot * a.pshot[0];
    T *__restrict__ sy0 = a.psi[1][0] + shot * a.pshot[1];
    T *__restrict__ sy1 = a.psi[1][1] + shot * a.pshot[1];
    T *__restrict__ sz0 = a.psi[2][0] + shot * a.pshot[2];
    T *__restrict__ sz1 = a.psi[2][1] + shot * a.pshot[2];

    // rolling z window: wx/wy[0..3] = planes k-2 .. k+1 of Hx and Hy
    T wx[4][VX], wy[4][VX];
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const int kk = kb - 2 + q;
        if (!GZ || (kk >= 0 && kk < nz)) {
            ldf<T, VX, CG>(wx[q], Hx + kk * pz + col);
            ldf<T, VX, CG>(wy[q], Hy + kk * pz + col);
        } else {
            zerov<T, VX>(wx[q]);
            zerov<T, VX>(wy[q]);
        }
    }
    const int slot = a.ring_k > 0 ? (step >= 0 ? step : *a.d_step) % a.ring_k : 0;

    // ONE: this thread owns the single plane kb (a compile-time trip count
    // of one, so the window is three loads and a fourth, not a rotation)
    const int kend = ONE ? kb + 1 : ke;
#pragma unroll 2
    for (int k = kb; k < kend; k++) {
        {
            const int kk = k + 1;
            if (!GZ || kk < nz) {
                ldf<T, VX, CG>(wx[3], Hx + kk * pz + col);
                ldf<T, VX, CG>(wy[3], Hy + kk * pz + col);
            } else {
                zerov<T, VX>(wx[3]);
                zerov<T, VX>(wy[3]);
            }
        }
        const int c = k * pz + col;
        T hzx[3 * VX], hyx[3 * VX];
        {
            T t[VX];
            ldf<T, VX, CG>(t, Hz + c);
#pragma unroll
            for (int v = 0; v < VX; v++) { hzx[VX + v] = t[v]; hyx[VX + v] = wy[2][v]; }
            if (has_l) {
                ldf<T, VX, CG>(t, Hz + c - VX);
#pragma unroll
                for (int v = 0; v < VX; v++) hzx[v] = t[v];
                ldf<T, VX, CG>(t, Hy + c - VX);
#pragma unroll
                for (int v = 0; v < VX; v++) hyx[v] = t[v];
            } else {
#pragma unroll
                for (int v = 0; v < VX; v++) { hzx[v] = T(0); hyx[v] = T(0); }
            }
            if (has_r) {
                ldf<T, VX, CG>(t, Hz + c + VX);
#pragma unroll
                for (int v = 0; v < VX; v++) hzx[2 * VX + v] = t[v];
                ldf<T, VX, CG>(t, Hy + c + VX);
#pragma unroll
                for (int v = 0; v < VX; v++) hyx[2 * VX + v] = t[v];
            } else {
#pragma unroll
                for (int v = 0; v < VX; v++) { hzx[2 * VX + v] = T(0); hyx[2 * VX + v] = T(0); }
            }
        }
        T hzm2[VX], hzm1[VX], hzp1[VX], hxm2[VX], hxm1[VX], hxp1[VX];
        if (vy) {
            ldf<T, VX, CG>(hzm2, Hz + c - 2 * py);
            ldf<T, VX, CG>(hzm1, Hz + c - py);
            ldf<T, VX, CG>(hzp1, Hz + c + py);
            ldf<T, VX, CG>(hxm2, Hx + c - 2 * py);
            ldf<T, VX, CG>(hxm1, Hx + c - py);
            ldf<T, VX, CG>(hxp1, Hx + c + py);
        } else {
            zerov<T, VX>(hzm2); zerov<T, VX>(hzm1); zerov<T, VX>(hzp1);
            zerov<T, VX>(hxm2); zerov<T, VX>(hxm1); zerov<T, VX>(hxp1);
        }
        T m[VX], ex[VX], ey[VX], ez[VX];
        ldv<T, VX>(m, M + c);
        // own cells: read once, before this thread writes them, and read by no
        // other thread in this phase, so the read-only path is valid and lets
        // the next plane's loads move above this plane's stores
        ldf<T, VX, CG>(ex, Ex + c);
        ldf<T, VX, CG>(ey, Ey + c);
        ldf<T, VX, CG>(ez, Ez + c);
        T esh_z, ik_z;
        bool vz, kx, ky, kz;
        int lz;
        if constexpr (!GZ) {
            esh_z = T(0);
            ik_z = a.ik[2];
            vz = kx = ky = kz = true;
            lz = -1;
        } else {
            esh_z = __ldg(P + 16 * ps + k);
            ik_z = __ldg(P + 22 * ps + k);
            vz = (k >= 2) && (k + 1 < nz);
            kx = k >= U0.lo[2] && k < U0.hi[2];
            ky = k >= U1.lo[2] && k < U1.hi[2];
            kz = k >= U2.lo[2] && k < U2.hi[2];
            lz = slab_local(S2, k);
        }
        const bool s0k = !GZ || (k >= S0.other.lo[2] && k < S0.other.hi[2]);
        const bool s1k = !GZ || (k >= S1.other.lo[2] && k < S1.other.hi[2]);

        // psi of the slabs this row crosses, loaded together with the fields
        const unsigned mx = (GX && s0k) ? sxm : 0u;
        const unsigned my = (GY && s1k) ? sym : 0u;
        const unsigned mz = (GZ && lz >= 0) ? szm : 0u;
        const int ox = (k * ny + j) * S0.width;
        const int oy = (k * S1.width + ly) * py + i0;
        const int oz = (lz * ny + j) * py + i0;
        T qx0[VX], qx1[VX], qy0[VX], qy1[VX], qz0[VX], qz1[VX];
        T be_z = T(0), ced_z = T(0);
        if constexpr (GX) {
#pragma unroll
            for (int v = 0; v < VX; v++) {
                qx0[v] = (mx >> v & 1) ? ldx<T, CG>(sx0 + ox + lx[v]) : T(0);
                qx1[v] = (mx >> v & 1) ? ldx<T, CG>(sx1 + ox + lx[v]) : T(0);
            }
        }
        if constexpr (GY) {
            ld_psi<T, VX, CG>(qy0, sy0, oy, my);
            ld_psi<T, VX, CG>(qy1, sy1, oy, my);
        }
        if constexpr (GZ) {
            ld_psi<T, VX, CG>(qz0, sz0, oz, mz);
            ld_psi<T, VX, CG>(qz1, sz1, oz, mz);
            be_z = __ldg(P + 18 * ps + k);
            ced_z = __ldg(P + 19 * ps + k);
        }

#pragma unroll
        for (int v = 0; v < VX; v++) {
            const bool vx = vxm >> v & 1;
            const T dyHz = vy ? d4(c1, c2, hzx[VX + v], hzm1[v], hzp1[v], hzm2[v]) : T(0);
            const T dyHx = vy ? d4(c1, c2, wx[2][v], hxm1[v], hxp1[v], hxm2[v]) : T(0);
            const T dxHz = vx ? d4(c1, c2, hzx[VX + v], hzx[VX + v - 1], hzx[VX + v + 1], hzx[VX + v - 2]) : T(0);
            const T dxHy = vx ? d4(c1, c2, hyx[VX + v], hyx[VX + v - 1], hyx[VX + v + 1], hyx[VX + v - 2]) : T(0);
            const T dzHy = vz ? d4(c1, c2, wy[2][v], wy[1][v], wy[3][v], wy[0][v]) : T(0);
            const T dzHx = vz ? d4(c1, c2, wx[2][v], wx[1][v], wx[3][v], wx[0][v]) : T(0);
            const T mv = m[v];
            T ca_x = T(1), cb_x = mv, ca_y = T(1), cb_y = mv, ca_z = T(1), cb_z = mv;
            if (GX && esh_x[v] != T(0)) { const T h = esh_x[v] * mv; const T r = rcp(T(1) + h); ca_x = (T(1) - h) * r; cb_x = mv * r; }
            if (GY && esh_y != T(0)) { const T h = esh_y * mv; const T r = rcp(T(1) + h); ca_y = (T(1) - h) * r; cb_y = mv * r; }
            if (GZ && esh_z != T(0)) { const T h = esh_z * mv; const T r = rcp(T(1) + h); ca_z = (T(1) - h) * r; cb_z = mv * r; }
            if (kx && (ux >> v & 1)) ex[v] = leap(ca_x, sg * cb_x, curl2(dyHz, ik_y, dzHy, ik_z), ex[v]);
            if (ky && (uy >> v & 1)) ey[v] = leap(ca_y, sg * cb_y, curl2(dzHx, ik_z, dxHz, ik_x[v]), ey[v]);
            if (kz && (uz >> v & 1)) ez[v] = leap(ca_z, sg * cb_z, curl2(dxHy, ik_x[v], dyHx, ik_y), ez[v]);

            if (GX && (mx >> v & 1)) {
                const T p0 = fma(be_x[v], qx0[v], ced_x[v] * dxHy);  // psi_Ezx
                const T p1 = fma(be_x[v], qx1[v], ced_x[v] * dxHz);  // psi_Eyx
                sx0[ox + lx[v]] = p0;
                sx1[ox + lx[v]] = p1;
                ez[v] = fma(cb_z, p0, ez[v]);
                ey[v] = fma(-cb_y, p1, ey[v]);
            }
            if (GY && (my >> v & 1)) {
                qy0[v] = fma(be_y, qy0[v], ced_y * dyHz);  // psi_Exy
                qy1[v] = fma(be_y, qy1[v], ced_y * dyHx);  // psi_Ezy
                ex[v] = fma(cb_x, qy0[v], ex[v]);
                ez[v] = fma(-cb_z, qy1[v], ez[v]);
            }
            if (GZ && (mz >> v & 1)) {
                qz0[v] = fma(be_z, qz0[v], ced_z * dzHx);  // psi_Eyz
                qz1[v] = fma(be_z, qz1[v], ced_z * dzHy);  // psi_Exz
                ey[v] = fma(cb_y, qz0[v], ey[v]);
                ex[v] = fma(-cb_x, qz1[v], ex[v]);
            }
        }
        if constexpr (GY) {
            st_psi<T, VX>(sy0, oy, qy0, my);
            st_psi<T, VX>(sy1, oy, qy1, my);
        }
        if constexpr (GZ) {
            st_psi<T, VX>(sz0, oz, qz0, mz);
            st_psi<T, VX>(sz1, oz, qz1, mz);
        }
        stv<T, VX>(Exo + c, ex);
        stv<T, VX>(Eyo + c, ey);
        stv<T, VX>(Ezo + c, ez);
        if (a.ring_k > 0) {
            const long long e = sb + c;
            if (a.vmask & 1) stv_stream<T, VX>(a.ring + ring_index(a.ring_comp, a.ring_k, 0, e, slot), ex);
            if (a.vmask & 2) stv_stream<T, VX>(a.ring + ring_index(a.ring_comp, a.ring_k, 1, e, slot), ey);
            if (a.vmask & 4) stv_stream<T, VX>(a.ring + ring_index(a.ring_comp, a.ring_k, 2, e, slot), ez);
        }
#pragma unroll
        for (int v = 0; v < VX; v++) {
            wx[0][v] = wx[1][v]; wx[1][v] = wx[2][v]; wx[2][v] = wx[3][v];
            wy[0][v] = wy[1][v]; wy[1][v] = wy[2][v]; wy[2][v] = wy[3][v];
        }
    }
}

// ------------------------------------------------------------------ H phase
template <typename T, int VX, int GM, bool ONE, bool CG = false>
__device__ __forceinline__ void h_cells(const PhaseArgs<T> &a, int shot, int i0, int j, int kb, int ke) {
    const long long sb = (long long)shot * a.fshot;
    const T *__restrict__ Ex = a.f[0] + sb;
    const T *__restrict__ Ey = a.f[1] + sb;
    const T *__restrict__ Ez = a.f[2] + sb;
    const T *__restrict__ Hx = a.f[3] + sb;
    const T *__restrict__ Hy = a.f[4] + sb;
    const T *__restrict__ Hz = a.f[5] + sb;
    T *__restrict__ Hxo = a.fo[3] + sb;
    T *__restrict__ Hyo = a.fo[4] + sb;
    T *__restrict__ Hzo = a.fo[5] + sb;
    const T *__restrict__ M = a.m;
    const T *__restrict__ DM = a.dtmu;
    const T *__restrict__ P = a.prof;
    const int py = a.px, pz = (int)a.plane, nx = a.nx, ny = a.ny, nz = a.nz, ps = a.nmax;
    const T c1 = a.c1, c2 = a.c2, c2t = a.c2t, sg = a.sgn;

    // GM bit 0/1/2: general handling along x/y/z; a clear bit means every
    // cell of the box is interior along that axis (no CPML profile, no psi
    // slab, inside every update range, derivative defined).
    constexpr bool GX = (GM & 1) != 0, GY = (GM & 2) != 0, GZ = (GM & 4) != 0;
    T msh_x[VX], ik_x[VX];
    T msh_y, ik_y;
    if constexpr (GX) {
        ldv<T, VX>(msh_x, P + 1 * ps + i0);
        ldv<T, VX>(ik_x, P + 7 * ps + i0);
    } else {
#pragma unroll
        for (int v = 0; v < VX; v++) { msh_x[v] = T(0); ik_x[v] = a.ik[0]; }
    }
    if constexpr (GY) {
        msh_y = __ldg(P + 9 * ps + j);
        ik_y = __ldg(P + 15 * ps + j);
    } else {
        msh_y = T(0);
        ik_y = a.ik[1];
    }
    const bool vy = GY ? ((j >= 1) && (j + 2 < ny)) : true;
    const bool has_l = GX ? (i0 >= VX) : true;
    const bool has_r = GX ? (i0 + VX < nx) : true;
    unsigned vxm = (1u << VX) - 1u;
    if constexpr (GX) {
        vxm = 0;
#pragma unroll
        for (int v = 0; v < VX; v++) vxm |= (unsigned)(i0 + v >= 1 && i0 + v + 2 < nx) << v;
    }
    const DBox U0 = a.upd[0], U1 = a.upd[1], U2 = a.upd[2];
    const unsigned all = (1u << VX) - 1u;
    const unsigned ux = (!GY || (j >= U0.lo[1] && j < U0.hi[1])) ? (GX ? xmask<VX>(i0, U0.lo[0], U0.hi[0]) : all) : 0u;
    const unsigned uy = (!GY || (j >= U1.lo[1] && j < U1.hi[1])) ? (GX ? xmask<VX>(i0, U1.lo[0], U1.hi[0]) : all) : 0u;
    const unsigned uz = (!GY || (j >= U2.lo[1] && j < U2.hi[1])) ? (GX ? xmask<VX>(i0, U2.lo[0], U2.hi[0]) : all) : 0u;
    const DSlab S0 = a.slab[0], S1 = a.slab[1], S2 = a.slab[2];
    unsigned sxm = 0;
    if constexpr (GX) {
#pragma unroll
        for (int v = 0; v < VX; v++) sxm |= (unsigned)(slab_local(S0, i0 + v) >= 0) << v;
        if (GY && !(j >= S0.other.lo[1] && j < S0.other.hi[1])) sxm = 0u;
    }
    const int ly = GY ? slab_local(S1, j) : -1;
    const unsigned sym = ly >= 0 ? (GX ? xmask<VX>(i0, S1.other.lo[0], S1.other.hi[0]) : all) : 0u;
    const unsigned szm = GZ ? ((!GY || (j >= S2.other.lo[1] && j < S2.other.hi[1])) ? (GX ? xmask<VX>(i0, S2.other.lo[0], S2.other.hi[0]) : all) : 0u) : 0u;
    const int col = j * py + i0;

    // psi recurrence coefficients of the x and y slabs (fixed along z) and
    // this shot's psi slabs.
    T bh_x[VX], chd_x[VX];
    int lx[VX];
    T bh_y = T(0), chd_y = T(0);
    if constexpr (GX) {
        ldv<T, VX>(bh_x, P + 4 * ps + i0);
        ldv<T, VX>(chd_x, P + 5 * ps + i0);
#pragma unroll
        for (int v = 0; v < VX; v++) lx[v] = slab_local(S0, i0 + v);
    }
    if constexpr (GY) {
        bh_y = __ldg(P + 12 * ps + j);
        chd_y = __ldg(P + 13 * ps + j);
    }
    T *__restrict__ sx0 = a.psi[0][0] + shot * a.pshot[0];
    T *__restrict__ sx1 = a.psi[0][1] + shot * a.pshot[0];
    T *__restrict__ sy0 = a.psi[1][0] + shot * a.pshot[1];
    T *__restrict__ sy1 = a.psi[1][1] + shot * a.pshot[1];
    T *__restrict__ sz0 = a.psi[2][0] + shot * a.pshot[2];
    T *__restrict__ sz1 = a.psi[2][1] + shot * a.pshot[2];

    // rolling z window: wx/wy[0..3] = planes k-1 .. k+2 of Ex and Ey
    T wx[4][VX], wy[4][VX];
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const int kk = kb - 1 + q;
        if (!GZ || (kk >= 0 && kk < nz)) {
            ldf<T, VX, CG>(wx[q], Ex + kk * pz + col);
            ldf<T, VX, CG>(wy[q], Ey + kk * pz + col);
        } else {
            zerov<T, VX>(wx[q]);
            zerov<T, VX>(wy[q]);
        }
    }

    // ONE: this thread owns the single plane kb (a compile-time trip count
    // of one, so the window is three loads and a fourth, not a rotation)
    const int kend = ONE ? kb + 1 : ke;
#pragma unroll 2
    for (int k = kb; k < kend; k++) {
        {
            const int kk = k + 2;
            if (!GZ || kk < nz) {
                ldf<T, VX, CG>(wx[3], Ex + kk * pz + col);
                ldf<T, VX, CG>(wy[3], Ey + kk * pz + col);
            } else {
                zerov<T, VX>(wx[3]);
                zerov<T, VX>(wy[3]);
            }
        }
        const int c = k * pz + col;
        T ezx[3 * VX], eyx[3 * VX];
        {
            T t[VX];
            ldf<T, VX, CG>(t, Ez + c);
#pragma unroll
            for (int v = 0; v < VX; v++) { ezx[VX + v] = t[v]; eyx[VX + v] = wy[1][v]; }
            if (has_l) {
                ldf<T, VX, CG>(t, Ez + c - VX);
#pragma unroll
                for (int v = 0; v < VX; v++) ezx[v] = t[v];
                ldf<T, VX, CG>(t, Ey + c - VX);
#pragma unroll
                for (int v = 0; v < VX; v++) eyx[v] = t[v];
            } else {
#pragma unroll
                for (int v = 0; v < VX; v++) { ezx[v] = T(0); eyx[v] = T(0); }
            }
            if (has_r) {
                ldf<T, VX, CG>(t, Ez + c + VX);
#pragma unroll
                for (int v = 0; v < VX; v++) ezx[2 * VX + v] = t[v];
                ldf<T, VX, CG>(t, Ey + c + VX);
#pragma unroll
                for (int v = 0; v < VX; v++) eyx[2 * VX + v] = t[v];
            } else {
#pragma unroll
                for (int v = 0; v < VX; v++) { ezx[2 * VX + v] = T(0); eyx[2 * VX + v] = T(0); }
            }
        }
        T ezm1[VX], ezp1[VX], ezp2[VX], exm1[VX], exp1[VX], exp2[VX];
        if (vy) {
            ldf<T, VX, CG>(ezm1, Ez + c - py);
            ldf<T, VX, CG>(ezp1, Ez + c + py);
            ldf<T, VX, CG>(ezp2, Ez + c + 2 * py);
            ldf<T, VX, CG>(exm1, Ex + c - py);
            ldf<T, VX, CG>(exp1, Ex + c + py);
            ldf<T, VX, CG>(exp2, Ex + c + 2 * py);
        } else {
            zerov<T, VX>(ezm1); zerov<T, VX>(ezp1); zerov<T, VX>(ezp2);
            zerov<T, VX>(exm1); zerov<T, VX>(exp1); zerov<T, VX>(exp2);
        }
        T m[VX], dm[VX], hx[VX], hy[VX], hz[VX];
        ldv<T, VX>(m, M + c);
        if (DM) {
            ldv<T, VX>(dm, DM + c);
        } else {
#pragma unroll
            for (int v = 0; v < VX; v++) dm[v] = a.dtmu0;
        }
        // own cells: read once before being written, by this thread only
        ldf<T, VX, CG>(hx, Hx + c);
        ldf<T, VX, CG>(hy, Hy + c);
        ldf<T, VX, CG>(hz, Hz + c);
        T msh_z, ik_z;
        bool vz, kx, ky, kz;
        int lz;
        if constexpr (!GZ) {
            msh_z = T(0);
            ik_z = a.ik[2];
            vz = kx = ky = kz = true;
            lz = -1;
        } else {
            msh_z = __ldg(P + 17 * ps + k);
            ik_z = __ldg(P + 23 * ps + k);
            vz = (k >= 1) && (k + 2 < nz);
            kx = k >= U0.lo[2] && k < U0.hi[2];
            ky = k >= U1.lo[2] && k < U1.hi[2];
            kz = k >= U2.lo[2] && k < U2.hi[2];
            lz = slab_local(S2, k);
        }
        const bool s0k = !GZ || (k >= S0.other.lo[2] && k < S0.other.hi[2]);
        const bool s1k = !GZ || (k >= S1.other.lo[2] && k < S1.other.hi[2]);

        // psi of the slabs this row crosses, loaded together with the fields
        const unsigned mx = (GX && s0k) ? sxm : 0u;
        const unsigned my = (GY && s1k) ? sym : 0u;
        const unsigned mz = (GZ && lz >= 0) ? szm : 0u;
        const int ox = (k * ny + j) * S0.width;
        const int oy = (k * S1.width + ly) * py + i0;
        const int oz = (lz * ny + j) * py + i0;
        T qx0[VX], qx1[VX], qy0[VX], qy1[VX], qz0[VX], qz1[VX];
        T bh_z = T(0), chd_z = T(0);
        if constexpr (GX) {
#pragma unroll
            for (int v = 0; v < VX; v++) {
                qx0[v] = (mx >> v & 1) ? ldx<T, CG>(sx0 + ox + lx[v]) : T(0);
                qx1[v] = (mx >> v & 1) ? ldx<T, CG>(sx1 + ox + lx[v]) : T(0);
            }
        }
        if constexpr (GY) {
            ld_psi<T, VX, CG>(qy0, sy0, oy, my);
            ld_psi<T, VX, CG>(qy1, sy1, oy, my);
        }
        if constexpr (GZ) {
            ld_psi<T, VX, CG>(qz0, sz0, oz, mz);
            ld_psi<T, VX, CG>(qz1, sz1, oz, mz);
            bh_z = __ldg(P + 20 * ps + k);
            chd_z = __ldg(P + 21 * ps + k);
        }

#pragma unroll
        for (int v = 0; v < VX; v++) {
            const bool vx = vxm >> v & 1;
            const T ez = ezx[VX + v];
            const T dyEz = vy ? d4(c1, c2, ezp1[v], ez, ezp2[v], ezm1[v]) : T(0);
            const T dyEx = vy ? d4(c1, c2, exp1[v], wx[1][v], exp2[v], exm1[v]) : T(0);
            const T dxEz = vx ? d4(c1, c2, ezx[VX + v + 1], ez, ezx[VX + v + 2], ezx[VX + v - 1]) : T(0);
            const T dxEy = vx ? d4(c1, c2, eyx[VX + v + 1], eyx[VX + v], eyx[VX + v + 2], eyx[VX + v - 1]) : T(0);
            const T dzEy = vz ? d4(c1, c2, wy[2][v], wy[1][v], wy[3][v], wy[0][v]) : T(0);
            const T dzEx = vz ? d4(c1, c2, wx[2][v], wx[1][v], wx[3][v], wx[0][v]) : T(0);
            const T mv = m[v], dmv = dm[v];
            T da_x = T(1), db_x = dmv, da_y = T(1), db_y = dmv, da_z = T(1), db_z = dmv;
            if (GX && msh_x[v] != T(0)) { const T h = msh_x[v] * mv; const T r = rcp(T(1) + h); da_x = (T(1) - h) * r; db_x = dmv * r; }
            if (GY && msh_y != T(0)) { const T h = msh_y * mv; const T r = rcp(T(1) + h); da_y = (T(1) - h) * r; db_y = dmv * r; }
            if (GZ && msh_z != T(0)) { const T h = msh_z * mv; const T r = rcp(T(1) + h); da_z = (T(1) - h) * r; db_z = dmv * r; }
            if (kx && (ux >> v & 1)) hx[v] = leap(da_x, -sg * db_x, curl2(dyEz, ik_y, dzEy, ik_z), hx[v]);
            if (ky && (uy >> v & 1)) hy[v] = leap(da_y, -sg * db_y, curl2(dzEx, ik_z, dxEz, ik_x[v]), hy[v]);
            if (kz && (uz >> v & 1)) hz[v] = leap(da_z, -sg * db_z, curl2(dxEy, ik_x[v], dyEx, ik_y), hz[v]);

            if (GX && (mx >> v & 1)) {
                // psi_Hyx stencil (cpu_cpml4.f90:400): c1 Ez(i+1) - c2t Ez(i) + c2 Ez(i+2) - c2 Ez(i-1)
                const T dxEzt = vx ? fma(c1, ezx[VX + v + 1], -(c2t * ez)) + c2 * (ezx[VX + v + 2] - ezx[VX + v - 1]) : T(0);
                const T p0 = fma(bh_x[v], qx0[v], chd_x[v] * dxEy);   // psi_Hzx
                const T p1 = fma(bh_x[v], qx1[v], chd_x[v] * dxEzt);  // psi_Hyx
                sx0[ox + lx[v]] = p0;
                sx1[ox + lx[v]] = p1;
                hz[v] = fma(-db_z, p0, hz[v]);
                hy[v] = fma(db_y, p1, hy[v]);
            }
            if (GY && (my >> v & 1)) {
                qy0[v] = fma(bh_y, qy0[v], chd_y * dyEz);  // psi_Hxy
                qy1[v] = fma(bh_y, qy1[v], chd_y * dyEx);  // psi_Hzy
                hx[v] = fma(-db_x, qy0[v], hx[v]);
                hz[v] = fma(db_z, qy1[v], hz[v]);
            }
            if (GZ && (mz >> v & 1)) {
                qz0[v] = fma(bh_z, qz0[v], chd_z * dzEx);  // psi_Hyz
                qz1[v] = fma(bh_z, qz1[v], chd_z * dzEy);  // psi_Hxz
                hy[v] = fma(-db_y, qz0[v], hy[v]);
                hx[v] = fma(db_x, qz1[v], hx[v]);
            }
        }
        if constexpr (GY) {
            st_psi<T, VX>(sy0, oy, qy0, my);
            st_psi<T, VX>(sy1, oy, qy1, my);
        }
        if constexpr (GZ) {
            st_psi<T, VX>(sz0, oz, qz0, mz);
            st_psi<T, VX>(sz1, oz, qz1, mz);
        }
        stv<T, VX>(Hxo + c, hx);
        stv<T, VX>(Hyo + c, hy);
        stv<T, VX>(Hzo + c, hz);
#pragma unroll
        for (int v = 0; v < VX; v++) {
            wx[0][v] = wx[1][v]; wx[1][v] = wx[2][v]; wx[2][v] = wx[3][v];
            wy[0][v] = wy[1][v]; wy[1][v] = wy[2][v]; wy[2][v] = wy[3][v];
        }
    }
}

// ------------------------------------------- interior with plane prefetch
// The interior body (GM = 0) with a software pipeline along z: every load
// of plane k + 1 (the x and y neighbours, the own cells, the model word and
// the window's next plane) is issued before plane k is computed, so each
// warp keeps two planes of loads in flight instead of one.  Two planes of
// operands in registers restrict it to two-cell FP32 threads.  Same fma
// forms as e_cells / h_cells: bit-identical.
template <typename T, int VX>
struct EPlane {
    T hz[VX], hzl[VX], hzr[VX], hyl[VX], hyr[VX];
    T hzm2[VX], hzm1[VX], hzp1[VX], hxm2[VX], hxm1[VX], hxp1[VX];
    T m[VX], ex[VX], ey[VX], ez[VX], nx[VX], ny[VX];  // nx, ny: Hx, Hy of plane k + 1
};

template <typename T, int VX>
__device__ __forceinline__ void e_plane_load(EPlane<T, VX> &p, const T *__restrict__ Hx, const T *__restrict__ Hy,
                                             const T *__restrict__ Hz, const T *__restrict__ M,
                                             const T *__restrict__ Ex, const T *__restrict__ Ey,
                                             const T *__restrict__ Ez, int c, int py, int pz) {
    ldv<T, VX>(p.hz, Hz + c);
    ldv<T, VX>(p.hzl, Hz + c - VX);
    ldv<T, VX>(p.hzr, Hz + c + VX);
    ldv<T, VX>(p.hyl, Hy + c - VX);
    ldv<T, VX>(p.hyr, Hy + c + VX);
    ldv<T, VX>(p.hzm2, Hz + c - 2 * py);
    ldv<T, VX>(p.hzm1, Hz + c - py);
    ldv<T, VX>(p.hzp1, Hz + c + py);
    ldv<T, VX>(p.hxm2, Hx + c - 2 * py);
    ldv<T, VX>(p.hxm1, Hx + c - py);
    ldv<T, VX>(p.hxp1, Hx + c + py);
    ldv<T, VX>(p.m, M + c);
    ldv<T, VX>(p.ex, Ex + c);
    ldv<T, VX>(p.ey, Ey + c);
    ldv<T, VX>(p.ez, Ez + c);
    ldv<T, VX>(p.nx, Hx + c + pz);
    ldv<T, VX>(p.ny, Hy + c + pz);
}

template <typename T, int VX>
__device__ __forceinline__ void e_interior_pf(const PhaseArgs<T> &a, int shot, int i0, int j, int kb, int ke) {
    const long long sb = (long long)shot * a.fshot;
    const T *__restrict__ Ex = a.f[0] + sb;
    const T *__restrict__ Ey = a.f[1] + sb;
    const T *__restrict__ Ez = a.f[2] + sb;
    T *__restrict__ Exo = a.fo[0] + sb;
    T *__restrict__ Eyo = a.fo[1] + sb;
    T *__restrict__ Ezo = a.fo[2] + sb;
    const T *__restrict__ Hx = a.f[3] + sb;
    const T *__restrict__ Hy = a.f[4] + sb;
    const T *__restrict__ Hz = a.f[5] + sb;
    const int py = a.px, pz = (int)a.plane;
    const T c1 = a.c1, c2 = a.c2, sg = a.sgn, ikx = a.ik[0], iky = a.ik[1], ikz = a.ik[2];
    const int col = j * py + i0;
    T wx[4][VX], wy[4][VX];
#pragma unroll
    for (int q = 0; q < 3; q++) {
        ldv<T, VX>(wx[q], Hx + (kb - 2 + q) * pz + col);
        ldv<T, VX>(wy[q], Hy + (kb - 2 + q) * pz + col);
    }
    const int slot = a.ring_k > 0 ? (*a.d_step) % a.ring_k : 0;
    EPlane<T, VX> cur, nxt;
    e_plane_load<T, VX>(cur, Hx, Hy, Hz, a.m, Ex, Ey, Ez, kb * pz + col, py, pz);
    for (int k = kb; k < ke; k++) {
        if (k + 1 < ke) e_plane_load<T, VX>(nxt, Hx, Hy, Hz, a.m, Ex, Ey, Ez, (k + 1) * pz + col, py, pz);
        const int c = k * pz + col;
#pragma unroll
        for (int v = 0; v < VX; v++) { wx[3][v] = cur.nx[v]; wy[3][v] = cur.ny[v]; }
        T hzx[3 * VX], hyx[3 * VX];
#pragma unroll
        for (int v = 0; v < VX; v++) {
            hzx[v] = cur.hzl[v]; hzx[VX + v] = cur.hz[v]; hzx[2 * VX + v] = cur.hzr[v];
            hyx[v] = cur.hyl[v]; hyx[VX + v] = wy[2][v]; hyx[2 * VX + v] = cur.hyr[v];
        }
        T ex[VX], ey[VX], ez[VX];
#pragma unroll
        for (int v = 0; v < VX; v++) {
            const T dyHz = d4(c1, c2, hzx[VX + v], cur.hzm1[v], cur.hzp1[v], cur.hzm2[v]);
            const T dyHx = d4(c1, c2, wx[2][v], cur.hxm1[v], cur.hxp1[v], cur.hxm2[v]);
            const T dxHz = d4(c1, c2, hzx[VX + v], hzx[VX + v - 1], hzx[VX + v + 1], hzx[VX + v - 2]);
            const T dxHy = d4(c1, c2, hyx[VX + v], hyx[VX + v - 1], hyx[VX + v + 1], hyx[VX + v - 2]);
            const T dzHy = d4(c1, c2, wy[2][v], wy[1][v], wy[3][v], wy[0][v]);
            const T dzHx = d4(c1, c2, wx[2][v], wx[1][v], wx[3][v], wx[0][v]);
            const T mv = cur.m[v];
            ex[v] = leap(T(1), sg * mv, curl2(dyHz, iky, dzHy, ikz), cur.ex[v]);
            ey[v] = leap(T(1), sg * mv, curl2(dzHx, ikz, dxHz, ikx), cur.ey[v]);
            ez[v] = leap(T(1), sg * mv, curl2(dxHy, ikx, dyHx, iky), cur.ez[v]);
        }
        stv<T, VX>(Exo + c, ex);
        stv<T, VX>(Eyo + c, ey);
        stv<T, VX>(Ezo + c, ez);
        if (a.ring_k > 0) {
            const long long e = sb + c;
            if (a.vmask & 1) stv_stream<T, VX>(a.ring + ring_index(a.ring_comp, a.ring_k, 0, e, slot), ex);
            if (a.vmask & 2) stv_stream<T, VX>(a.ring + ring_index(a.ring_comp, a.ring_k, 1, e, slot), ey);
            if (a.vmask & 4) stv_stream<T, VX>(a.ring + ring_index(a.ring_comp, a.ring_k, 2, e, slot), ez);
        }
#pragma unroll
        for (int v = 0; v < VX; v++) {
            wx[0][v] = wx[1][v]; wx[1][v] = wx[2][v]; wx[2][v] = wx[3][v];
            wy[0][v] = wy[1][v]; wy[1][v] = wy[2][v]; wy[2][v] = wy[3][v];
        }
        cur = nxt;
    }
}

template <typename T, int VX>
struct HPlane {
    T ez[VX], ezl[VX], ezr[VX], eyl[VX], eyr[VX];
    T ezm1[VX], ezp1[VX], ezp2[VX], exm1[VX], exp1[VX], exp2[VX];
    T dm[VX], hx[VX], hy[VX], hz[VX], nx[VX], ny[VX];  // nx, ny: Ex, Ey of plane k + 2
};

template <typename T, int VX>
__device__ __forceinline__ void h_plane_load(HPlane<T, VX> &p, const T *__restrict__ Ex, const T *__restrict__ Ey,
                                             const T *__restrict__ Ez, const T *__restrict__ DM, T dtmu0,
                                             const T *__restrict__ Hx, const T *__restrict__ Hy,
                                             const T *__restrict__ Hz, int c, int py, int pz) {
    ldv<T, VX>(p.ez, Ez + c);
    ldv<T, VX>(p.ezl, Ez + c - VX);
    ldv<T, VX>(p.ezr, Ez + c + VX);
    ldv<T, VX>(p.eyl, Ey + c - VX);
    ldv<T, VX>(p.eyr, Ey + c + VX);
    ldv<T, VX>(p.ezm1, Ez + c - py);
    ldv<T, VX>(p.ezp1, Ez + c + py);
    ldv<T, VX>(p.ezp2, Ez + c + 2 * py);
    ldv<T, VX>(p.exm1, Ex + c - py);
    ldv<T, VX>(p.exp1, Ex + c + py);
    ldv<T, VX>(p.exp2, Ex + c + 2 * py);
    if (DM) {
        ldv<T, VX>(p.dm, DM + c);
    } else {
#pragma unroll
        for (int v = 0; v < VX; v++) p.dm[v] = dtmu0;
    }
    ldv<T, VX>(p.hx, Hx + c);
    ldv<T, VX>(p.hy, Hy + c);
    ldv<T, VX>(p.hz, Hz + c);
    ldv<T, VX>(p.nx, Ex + c + 2 * pz);
    ldv<T, VX>(p.ny, Ey + c + 2 * pz);
}

template <typename T, int VX>
__device__ __forceinline__ void h_interior_pf(const PhaseArgs<T> &a, int shot, int i0, int j, int kb, int ke) {
    const long long sb = (long long)shot * a.fshot;
    const T *__restrict__ Ex = a.f[0] + sb;
    const T *__restrict__ Ey = a.f[1] + sb;
    const T *__restrict__ Ez = a.f[2] + sb;
    const T *__restrict__ Hx = a.f[3] + sb;
    const T *__restrict__ Hy = a.f[4] + sb;
    const T *__restrict__ Hz = a.f[5] + sb;
    T *__restrict__ Hxo = a.fo[3] + sb;
    T *__restrict__ Hyo = a.fo[4] + sb;
    T *__restrict__ Hzo = a.fo[5] + sb;
    const int py = a.px, pz = (int)a.plane;
    const T c1 = a.c1, c2 = a.c2, sg = a.sgn, ikx = a.ik[0], iky = a.ik[1], ikz = a.ik[2];
    const int col = j * py + i0;
    T wx[4][VX], wy[4][VX];  // planes k-1 .. k+2 of Ex and Ey
#pragma unroll
    for (int q = 0; q < 3; q++) {
        ldv<T, VX>(wx[q], Ex + (kb - 1 + q) * pz + col);
        ldv<T, VX>(wy[q], Ey + (kb - 1 + q) * pz + col);
    }
    HPlane<T, VX> cur, nxt;
    h_plane_load<T, VX>(cur, Ex, Ey, Ez, a.dtmu, a.dtmu0, Hx, Hy, Hz, kb * pz + col, py, pz);
    for (int k = kb; k < ke; k++) {
        if (k + 1 < ke) h_plane_load<T, VX>(nxt, Ex, Ey, Ez, a.dtmu, a.dtmu0, Hx, Hy, Hz, (k + 1) * pz + col, py, pz);
        const int c = k * pz + col;
#pragma unroll
        for (int v = 0; v < VX; v++) { wx[3][v] = cur.nx[v]; wy[3][v] = cur.ny[v]; }
        T ezx[3 * VX], eyx[3 * VX];
#pragma unroll
        for (int v = 0; v < VX; v++) {
            ezx[v] = cur.ezl[v]; ezx[VX + v] = cur.ez[v]; ezx[2 * VX + v] = cur.ezr[v];
            eyx[v] = cur.eyl[v]; eyx[VX + v] = wy[1][v]; eyx[2 * VX + v] = cur.eyr[v];
        }
        T hx[VX], hy[VX], hz[VX];
#pragma unroll
        for (int v = 0; v < VX; v++) {
            const T ez = ezx[VX + v];
            const T dyEz = d4(c1, c2, cur.ezp1[v], ez, cur.ezp2[v], cur.ezm1[v]);
            const T dyEx = d4(c1, c2, cur.exp1[v], wx[1][v], cur.exp2[v], cur.exm1[v]);
            const T dxEz = d4(c1, c2, ezx[VX + v + 1], ez, ezx[VX + v + 2], ezx[VX + v - 1]);
            const T dxEy = d4(c1, c2, eyx[VX + v + 1], eyx[VX + v], eyx[VX + v + 2], eyx[VX + v - 1]);
            const T dzEy = d4(c1, c2, wy[2][v], wy[1][v], wy[3][v], wy[0][v]);
            const T dzEx = d4(c1, c2, wx[2][v], wx[1][v], wx[3][v], wx[0][v]);
            const T dmv = cur.dm[v];
            hx[v] = leap(T(1), -sg * dmv, curl2(dyEz, iky, dzEy, ikz), cur.hx[v]);
            hy[v] = leap(T(1), -sg * dmv, curl2(dzEx, ikz, dxEz, ikx), cur.hy[v]);
            hz[v] = leap(T(1), -sg * dmv, curl2(dxEy, ikx, dyEx, iky), cur.hz[v]);
        }
        stv<T, VX>(Hxo + c, hx);
        stv<T, VX>(Hyo + c, hy);
        stv<T, VX>(Hzo + c, hz);
#pragma unroll
        for (int v = 0; v < VX; v++) {
            wx[0][v] = wx[1][v]; wx[1][v] = wx[2][v]; wx[2][v] = wx[3][v];
            wy[0][v] = wy[1][v]; wy[1][v] = wy[2][v]; wy[2][v] = wy[3][v];
        }
        cur = nxt;
    }
}

// Locate this CTA's box and tile (tile index b, boxes [q0, q1)): the
// thread's first x cell i0, its row j and its z planes [kb, ke).
template <int VX, int BX, int BY>
__device__ __forceinline__ void locate(const TileMap *__restrict__ tm, int q0, int q1, int b, int &i0, int &j,
                                       int &kb, int &ke, bool &inside) {
    int q = q0;
    for (int t = q0 + 1; t < q1; t++)
        if (b >= __ldg(&tm->start[t])) q = t;
    const int local = b - __ldg(&tm->start[q]);
    const int ntx = __ldg(&tm->ntx[q]), nty = __ldg(&tm->nty[q]), zc = __ldg(&tm->zc);
    const int tx = local % ntx, r = local / ntx;
    const int ty = r % nty, tz = r / nty;
    i0 = __ldg(&tm->lo[q][0]) + (tx * BX + (int)threadIdx.x) * VX;
    j = __ldg(&tm->lo[q][1]) + ty * BY + (int)threadIdx.y;
    kb = __ldg(&tm->lo[q][2]) + tz * zc;
    ke = min(kb + zc, __ldg(&tm->hi[q][2]));
    inside = i0 < __ldg(&tm->hi[q][0]) && j < __ldg(&tm->hi[q][1]);
}

// One kernel per body: GM = 0 interior, 1/2/4 the x/y/z faces, 7 edges and
// corners.  Tiles [first_tile, first_tile + gridDim.x) of boxes [q0, q1).
// BZ = 0: a BX x BY block, each thread marching the tile's ZC planes.
// BZ > 0: a BX x BY x BZ block over a tile of BZ planes, one plane per
// thread; the body then holds no rolling window and needs far fewer
// registers, so more warps per SM keep loads in flight.
#define MITTET_PHASE_KERNEL(PH)                                                                              \
    template <typename T, int VX, int BX, int BY, int GM, int BZ = 0>                                        \
    __global__ void __launch_bounds__(BX *BY *(BZ > 0 ? BZ : 1),                                             \
                                      (part_min_blocks<T, VX, BX * BY * (BZ > 0 ? BZ : 1), GM, BZ>()))       \
        PH##_part_kernel(const PhaseArgs<T> a, const TileMap *__restrict__ tm, int first_tile, int q0, int q1) { \
        int i0, j, kb, ke;                                                                                   \
        bool inside;                                                                                         \
        locate<VX, BX, BY>(tm, q0, q1, first_tile + blockIdx.x, i0, j, kb, ke, inside);                      \
        if constexpr (BZ > 0) {                                                                              \
            kb += (int)threadIdx.z;                                                                          \
            inside = inside && kb < ke;                                                                      \
        }                                                                                                    \
        if (inside) {                                                                                        \
            if constexpr (BZ == -1 && GM == 0)                                                               \
                PH##_interior_pf<T, VX>(a, blockIdx.y, i0, j, kb, ke);                                       \
            else                                                                                             \
                PH##_cells<T, VX, GM, (BZ > 0)>(a, blockIdx.y, i0, j, kb, ke);                               \
        }                                                                                                    \
    }

// e_part_kernel and h_part_kernel.
MITTET_PHASE_KERNEL(e)
MITTET_PHASE_KERNEL(h)

// The four boundary parts of a phase (x, y, z faces and the edges) in one
// launch: each CTA takes a tile of boxes [pbox[1], nbox) and runs the body of
// its box's kind.  One launch of ~1.6 k CTAs instead of four of a few hundred
// each gives the latency-bound boundary bodies more warps in flight beside
// the interior; it needs the registers of the heaviest body.  Tiles
// [first_tile, first_tile + gridDim.x).
template <typename T, int VX, int BX, int BY, bool EPH>
__global__ void __launch_bounds__(BX *BY, (part_min_blocks<T, VX, BX * BY, 7, 0>()))
    boundary_kernel(const PhaseArgs<T> a, const TileMap *__restrict__ tm, int first_tile, int q0, int q1) {
    const int b = first_tile + blockIdx.x;
    int q = q0;
    for (int t = q0 + 1; t < q1; t++)
        if (b >= __ldg(&tm->start[t])) q = t;
    int i0, j, kb, ke;
    bool inside;
    locate<VX, BX, BY>(tm, q, q + 1, b, i0, j, kb, ke, inside);
    if (!inside) return;
    const int kind = __ldg(&tm->kind[q]);
    if constexpr (EPH) {
        if (kind == 1) e_cells<T, VX, 1, false>(a, blockIdx.y, i0, j, kb, ke);
        else if (kind == 2) e_cells<T, VX, 2, false>(a, blockIdx.y, i0, j, kb, ke);
        else if (kind == 4) e_cells<T, VX, 4, false>(a, blockIdx.y, i0, j, kb, ke);
        else e_cells<T, VX, 7, false>(a, blockIdx.y, i0, j, kb, ke);
    } else {
        if (kind == 1) h_cells<T, VX, 1, false>(a, blockIdx.y, i0, j, kb, ke);
        else if (kind == 2) h_cells<T, VX, 2, false>(a, blockIdx.y, i0, j, kb, ke);
        else if (kind == 4) h_cells<T, VX, 4, false>(a, blockIdx.y, i0, j, kb, ke);
        else h_cells<T, VX, 7, false>(a, blockIdx.y, i0, j, kb, ke);
    }
}

// The interior and the two x faces of a phase in one launch, tiles in band
// order.  A band is BY rows x ZC planes of the interior y-z box; its tiles
// are the left x-face tiles (x-general body, VXF cells per thread), the
// interior tiles (interior body, VXI cells per thread) and the right x-face
// tiles, consecutive in blockIdx.x, so the CTAs in flight at any time read
// and write whole rows (split launches read the 32-cell x-face segments of
// a row apart from the rest of it, and row segments that short move DRAM
// lines well below the copy rate).  The body is chosen per CTA, so no warp
// diverges; the kernel needs the registers of the heavier body.
struct BandMap {
    int x0, x1, nx, y0, y1, z0, z1;  // interior box [x0, x1) x [y0, y1) x [z0, z1), row length nx
    int zc;                          // z planes per band
    int ntl, nti, ntr, nty;          // left-face, interior and right-face tiles per band; bands along y
};

template <typename T, int VXI, int VXF, int BX, int BY, bool EPH>
__global__ void __launch_bounds__(BX *BY, (sizeof(T) == 4 ? 512 : 384) / (BX * BY))
    band_kernel(const PhaseArgs<T> a, const BandMap bm) {
    int b = blockIdx.x;
    const int per = bm.ntl + bm.nti + bm.ntr;
    const int t = b % per;
    b /= per;
    const int ty = b % bm.nty, tz = b / bm.nty;
    const int j = bm.y0 + ty * BY + (int)threadIdx.y;
    const int kb = bm.z0 + tz * bm.zc, ke = min(kb + bm.zc, bm.z1);
    if (j >= bm.y1) return;
    if (t >= bm.ntl && t < bm.ntl + bm.nti) {
        const int i0 = bm.x0 + ((t - bm.ntl) * BX + (int)threadIdx.x) * VXI;
        if (i0 >= bm.x1) return;
        if constexpr (EPH)
            e_cells<T, VXI, 0, false>(a, blockIdx.y, i0, j, kb, ke);
        else
            h_cells<T, VXI, 0, false>(a, blockIdx.y, i0, j, kb, ke);
    } else {
        const bool left = t < bm.ntl;
        const int xe = left ? bm.x0 : bm.nx;
        const int i0 = (left ? 0 : bm.x1) + ((left ? t : t - bm.ntl - bm.nti) * BX + (int)threadIdx.x) * VXF;
        if (i0 >= xe) return;
        if constexpr (EPH)
            e_cells<T, VXF, 1, false>(a, blockIdx.y, i0, j, kb, ke);
        else
            h_cells<T, VXF, 1, false>(a, blockIdx.y, i0, j, kb, ke);
    }
}

// Variants the autotuner chooses from: (VX, BX, BY, ZC, BZ) = x cells per
// thread, thread block in x and y, z planes per tile, threads along z.
// BZ = 0: each thread marches the tile's ZC planes; ZC is a run-time tile
// parameter (the same kernel serves every ZC): short chunks give small boxes
// enough CTAs, long ones amortise the window preload.  BZ > 0 (ZC = BZ): one
// plane per thread (on 256^2 x 192 they lose to the marching bodies on every
// part, by 5-20%; they stay candidates for small boxes).  BZ = -1: marching,
// with the interior part prefetching plane k + 1 (e_interior_pf; the other
// parts march as BZ = 0).  BZ = -2: marching, with the interior body held to
// 6 resident CTAs per SM (85 registers) for more warps in flight.  The
// narrow blocks (x tile of 8 or 16 cells) suit the thin x faces.
#define MITTET_STENCIL_VARIANTS_F32(X) \
    X(2, 32, 4, 2, 0)                     \
    X(2, 32, 4, 4, 0)                     \
    X(2, 32, 4, 8, 0)                     \
    X(2, 32, 4, 16, 0)                    \
    X(2, 16, 8, 2, 0)                     \
    X(2, 16, 8, 4, 0)                     \
    X(2, 16, 8, 8, 0)                     \
    X(4, 16, 8, 2, 0)                     \
    X(4, 16, 8, 4, 0)                     \
    X(4, 16, 8, 8, 0)                     \
    X(4, 8, 16, 4, 0)                     \
    X(4, 16, 4, 4, 0)                     \
    X(2, 8, 16, 4, 0)                     \
    X(2, 8, 16, 8, 0)                     \
    X(2, 4, 32, 4, 0)                     \
    X(4, 16, 8, 2, 2)                     \
    X(2, 16, 4, 4, 4)                     \
    X(2, 8, 8, 4, 4)                      \
    X(2, 32, 4, 8, -1)                    \
    X(2, 16, 8, 8, -1)                    \
    X(2, 32, 4, 16, -1)                   \
    X(4, 16, 8, 8, -2)                    \
    X(4, 16, 4, 8, -2)                    \
    X(4, 16, 8, 4, -2)
#define MITTET_STENCIL_VARIANTS_F64(X) \
    X(2, 32, 4, 2, 0)                     \
    X(2, 32, 4, 4, 0)                     \
    X(2, 32, 4, 8, 0)                     \
    X(2, 16, 8, 2, 0)                     \
    X(2, 16, 8, 4, 0)                     \
    X(2, 16, 8, 8, 0)                     \
    X(2, 16, 4, 4, 0)                     \
    X(2, 8, 16, 4, 0)                     \
    X(2, 16, 4, 4, 4)                     \
    X(2, 8, 8, 4, 4)

}  // namespace mittet
