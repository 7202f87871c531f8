// kernels.cuh -- sm_100a kernels of the Mittet fictitious-wave FDTD step.
//
// One time step of one batch of shots is four launches on one stream:
//   inject_kernel (magnetic points, before E)   ncver0027/cpu_waveform.f90:46-50
//   e_phase_kernel  E update + CPML psi_E        cpu_eh_field_cpml42.f90:114-158, cpu_cpml4.f90:271-361
//   inject_kernel (electric points, after E)    satan_i/fwi3d_cpu_function_v1.4.c:526-527
//   h_phase_kernel  H update + CPML psi_H        cpu_eh_field_cpml42.f90:210-253, cpu_cpml4.f90:384-474
//   sample_kernel   receiver gather + step++     cpu_output.f90:20-30
// The step index lives in device memory (d_step) so a block of steps can be
// captured once in a CUDA graph and replayed.
//
// Layout in HBM: every field component is one array [shot][nz][ny][px]
// (px = nx rounded up to 32 elements so rows start 128-byte aligned).  The
// model is one word per cell, m = dt/eps' = 2 w0 dt / sigma (the interior cb),
// plus dt/mu per cell only when a permeability volume is given.  CPML psi
// variables exist only inside their slabs (compact [shot][...] boxes).
//
// Each thread owns one (i, j) column of a z-chunk and marches k upward,
// keeping the four z-neighbours of the two fields differentiated along z in
// registers; x/y neighbours come through the read-only L1 path (the fields
// read in a phase are never written in that phase).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mittet {

struct DBox {
    int lo[3], hi[3];
};
struct DSlab {
    int nlo, nhi, flo, fhi, width;
    DBox other;
};

template <typename T>
struct PhaseArgs {
    T *f[6];                // Ex Ey Ez Hx Hy Hz, shot 0
    T *psi[3][2];           // psi of this phase's slab groups (axis, which)
    const T *m;             // per-cell 2 w0 dt / sigma
    const T *dtmu;          // per-cell dt/mu or nullptr
    T dtmu0;                // dt/mu0 when dtmu == nullptr
    const T *prof;          // [3][P_COUNT][nmax]
    int nmax;
    int nx, ny, nz, px;
    long long plane;        // px * ny
    long long fshot;        // nz * plane
    long long pshot[3];     // psi elements per shot per slab axis
    DBox upd[3];            // update boxes of the three components of this phase
    DSlab slab[3];          // slab groups of this phase (x, y, z)
    T c1, c2, c2t;          // stencil weights; c2t = c2 (psi_Hyx typo) or c1
    T sgn;                  // +1 / -1 ("bp" updates)
    int zchunk;
    // full-volume DFT ring (E phase only): ring[slot][vcomp][shot][cell]
    T *ring;
    int ring_k;             // ring depth K (0 = no ring)
    int vmask;              // E components written to the ring
    long long ring_comp;    // elements per (slot, vcomp) = nshot * fshot
    const int *d_step;
};

__device__ __forceinline__ bool in_box(const DBox &b, int i, int j, int k) {
    return i >= b.lo[0] && i < b.hi[0] && j >= b.lo[1] && j < b.hi[1] && k >= b.lo[2] && k < b.hi[2];
}

// Local index along the slab axis, or -1 if v is in neither interval.
__device__ __forceinline__ int slab_local(const DSlab &s, int v) {
    if (v >= s.nlo && v < s.nhi) return v - s.nlo;
    if (v >= s.flo && v < s.fhi) return (s.nhi - s.nlo) + (v - s.flo);
    return -1;
}

template <typename T>
__device__ __forceinline__ T ldg(const T *p) {
    return __ldg(p);
}

template <typename T>
__device__ __forceinline__ T rcp(T x);
template <>
__device__ __forceinline__ float rcp<float>(float x) {
    return __frcp_rn(x);
}
template <>
__device__ __forceinline__ double rcp<double>(double x) {
    return 1.0 / x;
}

// Profile value of one axis.
template <typename T>
__device__ __forceinline__ T pv(const PhaseArgs<T> &a, int axis, int which, int i) {
    return ldg(a.prof + ((size_t)axis * 8 + which) * a.nmax + i);
}

// ------------------------------------------------------------------ E phase
//
// Ex = ca_x Ex + s cb_x (Dy(Hz)/kedy - Dz(Hy)/kedz)   with D backward (2,4):
//   D(F)[v] = c1 (F[v] - F[v-1]) + c2 (F[v+1] - F[v-2])
// ca = (1-h)/(1+h), cb = m/(1+h), h = esig * m / 2 on the component's axis.
// CPML: psi = be psi + ce/d * D(F); the E field gets +-cb psi.
template <typename T, int BX, int BY>
__global__ void __launch_bounds__(BX *BY) e_phase_kernel(PhaseArgs<T> a) {
    const int i = blockIdx.x * BX + threadIdx.x;
    const int j = blockIdx.y * BY + threadIdx.y;
    const int nzc = (a.nz + a.zchunk - 1) / a.zchunk;
    const int shot = blockIdx.z / nzc;
    const int k0 = (blockIdx.z % nzc) * a.zchunk;
    const int k1 = min(k0 + a.zchunk, a.nz);
    if (i >= a.nx || j >= a.ny) return;

    const long long sb = (long long)shot * a.fshot;
    T *__restrict__ Ex = a.f[0] + sb;
    T *__restrict__ Ey = a.f[1] + sb;
    T *__restrict__ Ez = a.f[2] + sb;
    const T *__restrict__ Hx = a.f[3] + sb;
    const T *__restrict__ Hy = a.f[4] + sb;
    const T *__restrict__ Hz = a.f[5] + sb;
    const long long py = a.px, pz = a.plane;
    const T c1 = a.c1, c2 = a.c2;

    // per-column profile values
    const T esh_x = pv(a, 0, 0, i), esh_y = pv(a, 1, 0, j);
    const T ik_x = pv(a, 0, 6, i), ik_y = pv(a, 1, 6, j);
    const bool vx = (i >= 2) && (i + 1 < a.nx);
    const bool vy = (j >= 2) && (j + 1 < a.ny);
    const int lx = slab_local(a.slab[0], i);
    const int ly = slab_local(a.slab[1], j);
    const bool sx_col = lx >= 0 && j >= a.slab[0].other.lo[1] && j < a.slab[0].other.hi[1];
    const bool sy_col = ly >= 0 && i >= a.slab[1].other.lo[0] && i < a.slab[1].other.hi[0];
    const bool sz_col = i >= a.slab[2].other.lo[0] && i < a.slab[2].other.hi[0] && j >= a.slab[2].other.lo[1] &&
                        j < a.slab[2].other.hi[1];
    const T be_x = sx_col ? pv(a, 0, 2, i) : T(0), ced_x = sx_col ? pv(a, 0, 3, i) : T(0);
    const T be_y = sy_col ? pv(a, 1, 2, j) : T(0), ced_y = sy_col ? pv(a, 1, 3, j) : T(0);

    const int step = a.ring_k > 0 ? *a.d_step : 0;
    const int slot = a.ring_k > 0 ? step % a.ring_k : 0;

    // z window of Hx and Hy at (i, j): w[0..3] = F(k-2), F(k-1), F(k), F(k+1)
    const long long col = (long long)j * py + i;
    T wx[4], wy[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int kk = k0 - 2 + q;
        const bool ok = kk >= 0 && kk < a.nz;
        wx[q] = ok ? ldg(Hx + kk * pz + col) : T(0);
        wy[q] = ok ? ldg(Hy + kk * pz + col) : T(0);
    }

    for (int k = k0; k < k1; ++k) {
        const long long c = k * pz + col;
        const bool vz = (k >= 2) && (k + 1 < a.nz);
        const T hz = ldg(Hz + c);

        T dyHz = T(0), dxHz = T(0), dxHy = T(0), dyHx = T(0), dzHy = T(0), dzHx = T(0);
        if (vy) {
            dyHz = c1 * (hz - ldg(Hz + c - py)) + c2 * (ldg(Hz + c + py) - ldg(Hz + c - 2 * py));
            dyHx = c1 * (wx[2] - ldg(Hx + c - py)) + c2 * (ldg(Hx + c + py) - ldg(Hx + c - 2 * py));
        }
        if (vx) {
            dxHz = c1 * (hz - ldg(Hz + c - 1)) + c2 * (ldg(Hz + c + 1) - ldg(Hz + c - 2));
            dxHy = c1 * (wy[2] - ldg(Hy + c - 1)) + c2 * (ldg(Hy + c + 1) - ldg(Hy + c - 2));
        }
        if (vz) {
            dzHy = c1 * (wy[2] - wy[1]) + c2 * (wy[3] - wy[0]);
            dzHx = c1 * (wx[2] - wx[1]) + c2 * (wx[3] - wx[0]);
        }

        const T m = ldg(a.m + (long long)k * pz + col);
        const T esh_z = pv(a, 2, 0, k);
        const T ik_z = pv(a, 2, 6, k);
        T ca_x = T(1), cb_x = m, ca_y = T(1), cb_y = m, ca_z = T(1), cb_z = m;
        if (esh_x != T(0)) { const T h = esh_x * m; const T r = rcp(T(1) + h); ca_x = (T(1) - h) * r; cb_x = m * r; }
        if (esh_y != T(0)) { const T h = esh_y * m; const T r = rcp(T(1) + h); ca_y = (T(1) - h) * r; cb_y = m * r; }
        if (esh_z != T(0)) { const T h = esh_z * m; const T r = rcp(T(1) + h); ca_z = (T(1) - h) * r; cb_z = m * r; }

        T ex = Ex[c], ey = Ey[c], ez = Ez[c];
        if (in_box(a.upd[0], i, j, k)) ex = ca_x * ex + a.sgn * cb_x * (dyHz * ik_y - dzHy * ik_z);
        if (in_box(a.upd[1], i, j, k)) ey = ca_y * ey + a.sgn * cb_y * (dzHx * ik_z - dxHz * ik_x);
        if (in_box(a.upd[2], i, j, k)) ez = ca_z * ez + a.sgn * cb_z * (dxHy * ik_x - dyHx * ik_y);

        // CPML_E4: x slabs, y slabs, z slabs
        if (sx_col && k >= a.slab[0].other.lo[2] && k < a.slab[0].other.hi[2]) {
            const long long q = (long long)shot * a.pshot[0] + ((long long)k * a.ny + j) * a.slab[0].width + lx;
            T p0 = a.psi[0][0][q], p1 = a.psi[0][1][q];
            p0 = be_x * p0 + ced_x * dxHy;  // psi_Ezx
            p1 = be_x * p1 + ced_x * dxHz;  // psi_Eyx
            a.psi[0][0][q] = p0;
            a.psi[0][1][q] = p1;
            ez = ez + cb_z * p0;
            ey = ey - cb_y * p1;
        }
        if (sy_col && k >= a.slab[1].other.lo[2] && k < a.slab[1].other.hi[2]) {
            const long long q = (long long)shot * a.pshot[1] + ((long long)k * a.slab[1].width + ly) * a.px + i;
            T p0 = a.psi[1][0][q], p1 = a.psi[1][1][q];
            p0 = be_y * p0 + ced_y * dyHz;  // psi_Exy
            p1 = be_y * p1 + ced_y * dyHx;  // psi_Ezy
            a.psi[1][0][q] = p0;
            a.psi[1][1][q] = p1;
            ex = ex + cb_x * p0;
            ez = ez - cb_z * p1;
        }
        if (sz_col) {
            const int lz = slab_local(a.slab[2], k);
            if (lz >= 0) {
                const long long q = (long long)shot * a.pshot[2] + ((long long)lz * a.ny + j) * a.px + i;
                const T be_z = pv(a, 2, 2, k), ced_z = pv(a, 2, 3, k);
                T p0 = a.psi[2][0][q], p1 = a.psi[2][1][q];
                p0 = be_z * p0 + ced_z * dzHx;  // psi_Eyz
                p1 = be_z * p1 + ced_z * dzHy;  // psi_Exz
                a.psi[2][0][q] = p0;
                a.psi[2][1][q] = p1;
                ey = ey + cb_y * p0;
                ex = ex - cb_x * p1;
            }
        }
        Ex[c] = ex;
        Ey[c] = ey;
        Ez[c] = ez;

        if (a.ring_k > 0) {
            T *r = a.ring + (long long)slot * 3 * a.ring_comp + sb + c;
            if (a.vmask & 1) r[0] = ex;
            if (a.vmask & 2) r[a.ring_comp] = ey;
            if (a.vmask & 4) r[2 * a.ring_comp] = ez;
        }

        // advance the z windows
#pragma unroll
        for (int q = 0; q < 3; q++) { wx[q] = wx[q + 1]; wy[q] = wy[q + 1]; }
        const int kn = k + 2;
        const bool ok = kn < a.nz;
        wx[3] = ok ? ldg(Hx + kn * pz + col) : T(0);
        wy[3] = ok ? ldg(Hy + kn * pz + col) : T(0);
    }
}

// ------------------------------------------------------------------ H phase
//
// Hx = da_x Hx - s db_x (D+y(Ez)/khdy - D+z(Ey)/khdz)  with D+ forward (2,4):
//   D+(F)[v] = c1 (F[v+1] - F[v]) + c2 (F[v+2] - F[v-1])
// da = (1-h)/(1+h), db = (dt/mu)/(1+h), h = msig * m / 2.
template <typename T, int BX, int BY>
__global__ void __launch_bounds__(BX *BY) h_phase_kernel(PhaseArgs<T> a) {
    const int i = blockIdx.x * BX + threadIdx.x;
    const int j = blockIdx.y * BY + threadIdx.y;
    const int nzc = (a.nz + a.zchunk - 1) / a.zchunk;
    const int shot = blockIdx.z / nzc;
    const int k0 = (blockIdx.z % nzc) * a.zchunk;
    const int k1 = min(k0 + a.zchunk, a.nz);
    if (i >= a.nx || j >= a.ny) return;

    const long long sb = (long long)shot * a.fshot;
    const T *__restrict__ Ex = a.f[0] + sb;
    const T *__restrict__ Ey = a.f[1] + sb;
    const T *__restrict__ Ez = a.f[2] + sb;
    T *__restrict__ Hx = a.f[3] + sb;
    T *__restrict__ Hy = a.f[4] + sb;
    T *__restrict__ Hz = a.f[5] + sb;
    const long long py = a.px, pz = a.plane;
    const T c1 = a.c1, c2 = a.c2;

    const T msh_x = pv(a, 0, 1, i), msh_y = pv(a, 1, 1, j);
    const T ik_x = pv(a, 0, 7, i), ik_y = pv(a, 1, 7, j);
    const bool vx = (i >= 1) && (i + 2 < a.nx);
    const bool vy = (j >= 1) && (j + 2 < a.ny);
    const int lx = slab_local(a.slab[0], i);
    const int ly = slab_local(a.slab[1], j);
    const bool sx_col = lx >= 0 && j >= a.slab[0].other.lo[1] && j < a.slab[0].other.hi[1];
    const bool sy_col = ly >= 0 && i >= a.slab[1].other.lo[0] && i < a.slab[1].other.hi[0];
    const bool sz_col = i >= a.slab[2].other.lo[0] && i < a.slab[2].other.hi[0] && j >= a.slab[2].other.lo[1] &&
                        j < a.slab[2].other.hi[1];
    const T bh_x = sx_col ? pv(a, 0, 4, i) : T(0), chd_x = sx_col ? pv(a, 0, 5, i) : T(0);
    const T bh_y = sy_col ? pv(a, 1, 4, j) : T(0), chd_y = sy_col ? pv(a, 1, 5, j) : T(0);

    // z window of Ex and Ey: w[0..3] = F(k-1), F(k), F(k+1), F(k+2)
    const long long col = (long long)j * py + i;
    T wx[4], wy[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int kk = k0 - 1 + q;
        const bool ok = kk >= 0 && kk < a.nz;
        wx[q] = ok ? ldg(Ex + kk * pz + col) : T(0);
        wy[q] = ok ? ldg(Ey + kk * pz + col) : T(0);
    }

    for (int k = k0; k < k1; ++k) {
        const long long c = k * pz + col;
        const bool vz = (k >= 1) && (k + 2 < a.nz);
        const T ez = ldg(Ez + c);

        T dyEz = T(0), dyEx = T(0), dxEz = T(0), dxEy = T(0), dzEy = T(0), dzEx = T(0), dxEzt = T(0);
        if (vy) {
            dyEz = c1 * (ldg(Ez + c + py) - ez) + c2 * (ldg(Ez + c + 2 * py) - ldg(Ez + c - py));
            dyEx = c1 * (ldg(Ex + c + py) - wx[1]) + c2 * (ldg(Ex + c + 2 * py) - ldg(Ex + c - py));
        }
        if (vx) {
            const T ezp1 = ldg(Ez + c + 1), ezp2 = ldg(Ez + c + 2), ezm1 = ldg(Ez + c - 1);
            dxEz = c1 * (ezp1 - ez) + c2 * (ezp2 - ezm1);
            dxEzt = c1 * ezp1 - a.c2t * ez + c2 * ezp2 - c2 * ezm1;  // psi_Hyx stencil (cpu_cpml4.f90:400)
            dxEy = c1 * (ldg(Ey + c + 1) - wy[1]) + c2 * (ldg(Ey + c + 2) - ldg(Ey + c - 1));
        }
        if (vz) {
            dzEy = c1 * (wy[2] - wy[1]) + c2 * (wy[3] - wy[0]);
            dzEx = c1 * (wx[2] - wx[1]) + c2 * (wx[3] - wx[0]);
        }

        const T m = ldg(a.m + (long long)k * pz + col);
        const T dm = a.dtmu ? ldg(a.dtmu + (long long)k * pz + col) : a.dtmu0;
        const T msh_z = pv(a, 2, 1, k);
        const T ik_z = pv(a, 2, 7, k);
        T da_x = T(1), db_x = dm, da_y = T(1), db_y = dm, da_z = T(1), db_z = dm;
        if (msh_x != T(0)) { const T h = msh_x * m; const T r = rcp(T(1) + h); da_x = (T(1) - h) * r; db_x = dm * r; }
        if (msh_y != T(0)) { const T h = msh_y * m; const T r = rcp(T(1) + h); da_y = (T(1) - h) * r; db_y = dm * r; }
        if (msh_z != T(0)) { const T h = msh_z * m; const T r = rcp(T(1) + h); da_z = (T(1) - h) * r; db_z = dm * r; }

        T hx = Hx[c], hy = Hy[c], hz = Hz[c];
        if (in_box(a.upd[0], i, j, k)) hx = da_x * hx - a.sgn * db_x * (dyEz * ik_y - dzEy * ik_z);
        if (in_box(a.upd[1], i, j, k)) hy = da_y * hy - a.sgn * db_y * (dzEx * ik_z - dxEz * ik_x);
        if (in_box(a.upd[2], i, j, k)) hz = da_z * hz - a.sgn * db_z * (dxEy * ik_x - dyEx * ik_y);

        // CPML_H4: x slabs, y slabs, z slabs
        if (sx_col && k >= a.slab[0].other.lo[2] && k < a.slab[0].other.hi[2]) {
            const long long q = (long long)shot * a.pshot[0] + ((long long)k * a.ny + j) * a.slab[0].width + lx;
            T p0 = a.psi[0][0][q], p1 = a.psi[0][1][q];
            p0 = bh_x * p0 + chd_x * dxEy;   // psi_Hzx
            p1 = bh_x * p1 + chd_x * dxEzt;  // psi_Hyx
            a.psi[0][0][q] = p0;
            a.psi[0][1][q] = p1;
            hz = hz - db_z * p0;
            hy = hy + db_y * p1;
        }
        if (sy_col && k >= a.slab[1].other.lo[2] && k < a.slab[1].other.hi[2]) {
            const long long q = (long long)shot * a.pshot[1] + ((long long)k * a.slab[1].width + ly) * a.px + i;
            T p0 = a.psi[1][0][q], p1 = a.psi[1][1][q];
            p0 = bh_y * p0 + chd_y * dyEz;  // psi_Hxy
            p1 = bh_y * p1 + chd_y * dyEx;  // psi_Hzy
            a.psi[1][0][q] = p0;
            a.psi[1][1][q] = p1;
            hx = hx - db_x * p0;
            hz = hz + db_z * p1;
        }
        if (sz_col) {
            const int lz = slab_local(a.slab[2], k);
            if (lz >= 0) {
                const long long q = (long long)shot * a.pshot[2] + ((long long)lz * a.ny + j) * a.px + i;
                const T bh_z = pv(a, 2, 4, k), chd_z = pv(a, 2, 5, k);
                T p0 = a.psi[2][0][q], p1 = a.psi[2][1][q];
                p0 = bh_z * p0 + chd_z * dzEx;  // psi_Hyz
                p1 = bh_z * p1 + chd_z * dzEy;  // psi_Hxz
                a.psi[2][0][q] = p0;
                a.psi[2][1][q] = p1;
                hy = hy - db_y * p0;
                hx = hx + db_x * p1;
            }
        }
        Hx[c] = hx;
        Hy[c] = hy;
        Hz[c] = hz;

#pragma unroll
        for (int q = 0; q < 3; q++) { wx[q] = wx[q + 1]; wy[q] = wy[q + 1]; }
        const int kn = k + 3;
        const bool ok = kn < a.nz;
        wx[3] = ok ? ldg(Ex + kn * pz + col) : T(0);
        wy[3] = ok ? ldg(Ey + kn * pz + col) : T(0);
    }
}

// ---------------------------------------------------------- point sources
struct SrcPoint {
    long long off;  // shot * fshot + cell offset (padded layout)
    int comp;
    int kind;       // 0 magnetic (uses w[n+1]), 1 electric (uses (w[n]+w[n+1])/2)
    double g;       // amp * dt/mu/(dx dy dz)  or  amp * dt * 2 w0/sigma/(dx dy dz)
};

template <typename T>
struct InjectArgs {
    T *f[6];
    const SrcPoint *pts;
    int npts;
    int kind;
    const double *wave;  // w[0..nt]
    const int *d_step;
    T *ring;             // full-volume ring or nullptr
    int ring_k, vmask;
    long long ring_comp;
};

template <typename T>
__global__ void inject_kernel(InjectArgs<T> a) {
    const int n = *a.d_step;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < a.npts; p += gridDim.x * blockDim.x) {
        const SrcPoint s = a.pts[p];
        if (s.kind != a.kind) continue;
        const double w = s.kind == 0 ? a.wave[n + 1] : (a.wave[n] + a.wave[n + 1]) / 2.0;
        T *cell = a.f[s.comp] + s.off;
        const T v = atomicAdd(cell, (T)(-s.g * w)) + (T)(-s.g * w);
        if (a.ring && s.comp < 3 && (a.vmask >> s.comp & 1)) {
            const int slot = n % a.ring_k;
            a.ring[((long long)slot * 3 + s.comp) * a.ring_comp + s.off] = v;
        }
    }
}

// ---------------------------------------------------------------- sampling
template <typename T>
struct SampleArgs {
    const T *f[6];
    const long long *rec_off;  // cell offsets (padded layout, shot 0)
    const int *rec_comp;
    int nrec, nshot;
    long long fshot;
    T *traces;                 // [shot][rec][nt]
    int nt;
    int *d_step;
};

// One block: every thread reads d_step, gathers, then thread 0 advances it.
template <typename T>
__global__ void sample_kernel(SampleArgs<T> a) {
    const int n = *a.d_step;
    const int tot = a.nrec * a.nshot;
    for (int q = threadIdx.x; q < tot; q += blockDim.x) {
        const int s = q / a.nrec, r = q % a.nrec;
        a.traces[(long long)q * a.nt + n] = a.f[a.rec_comp[r]][(long long)s * a.fshot + a.rec_off[r]];
    }
    __syncthreads();
    if (threadIdx.x == 0) *a.d_step = n + 1;
}

// ---------------------------------------------------------- f_to_d (traces)
//
// X(w_f) = sum_n x[n] dt exp((i-1) sqrt(w0 w_f) n dt), times sqrt(-2 w0/(i w_f))
// for H traces when hfac is set (cpu_f_to_d_e.f90:140-148, cpu_f_to_d_h.f90:146-148).
// Block = one frequency; threads stride over traces; the weights of a chunk
// of time samples are computed once per block into shared memory in FP64.
template <typename T>
__global__ void trace_dft_kernel(const T *__restrict__ x, int ntrace, int nt, const double *__restrict__ omega,
                                 int nf, double dt, double omega0, const unsigned char *__restrict__ is_h, int hfac,
                                 double2 *__restrict__ out) {
    constexpr int CH = 256;
    __shared__ double2 w[CH];
    const int f = blockIdx.x;
    if (f >= nf) return;
    const double sw = sqrt(omega0 * omega[f]);
    double2 hf = make_double2(1.0, 0.0);
    if (hfac) {
        // sqrt(-2 w0/(i w)) = sqrt(2 w0/w) * exp(i pi/4)  (principal branch)
        const double r = sqrt(2.0 * omega0 / omega[f]);
        hf = make_double2(r * 0.70710678118654752440, r * 0.70710678118654752440);
    }
    for (int t0 = 0; t0 < ntrace; t0 += blockDim.x) {
        const int t = t0 + threadIdx.x;
        double re = 0.0, im = 0.0;
        for (int n0 = 0; n0 < nt; n0 += CH) {
            __syncthreads();
            for (int q = threadIdx.x; q < CH && n0 + q < nt; q += blockDim.x) {
                const double xa = sw * (double)(n0 + q) * dt;
                double s, c;
                sincos(xa, &s, &c);
                const double e = exp(-xa) * dt;
                w[q] = make_double2(e * c, e * s);
            }
            __syncthreads();
            if (t < ntrace) {
                const T *xt = x + (long long)t * nt + n0;
                const int cnt = min(CH, nt - n0);
                for (int q = 0; q < cnt; q++) {
                    const double v = (double)xt[q];
                    re += v * w[q].x;
                    im += v * w[q].y;
                }
            }
        }
        if (t < ntrace) {
            if (hfac && is_h && is_h[t]) {
                const double r2 = re * hf.x - im * hf.y, i2 = re * hf.y + im * hf.x;
                re = r2;
                im = i2;
            }
            out[(long long)t * nf + f] = make_double2(re, im);
        }
    }
}

// ---------------------------------------------------- full-volume f_to_d
//
// acc[shot][vc][f][cell] += sum_{s<cnt} wt[n0+s][f] * ring[s][vc][shot][cell]
// (weights wt[n][f] = dt exp((i-1) sqrt(w0 w_f) n dt), FP64).
template <typename T>
__global__ void volume_dft_kernel(const T *__restrict__ ring, long long ring_comp, int vmask, int nshot,
                                  long long fshot, int cnt, int n0, const double2 *__restrict__ wt, int nf,
                                  double2 *__restrict__ acc) {
    const long long tot = (long long)nshot * fshot;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        const int shot = (int)(e / fshot);
        const long long cell = e - (long long)shot * fshot;
        for (int vc = 0; vc < 3; vc++) {
            if (!(vmask >> vc & 1)) continue;
            double xs[16];
#pragma unroll
            for (int s = 0; s < 16; s++) xs[s] = s < cnt ? (double)ring[((long long)s * 3 + vc) * ring_comp + e] : 0.0;
            double2 *ap = acc + (((long long)shot * 3 + vc) * nf) * fshot + cell;
            for (int f = 0; f < nf; f++) {
                double2 v = ap[(long long)f * fshot];
#pragma unroll
                for (int s = 0; s < 16; s++) {
                    if (s < cnt) {
                        const double2 w = wt[(long long)(n0 + s) * nf + f];
                        v.x += w.x * xs[s];
                        v.y += w.y * xs[s];
                    }
                }
                ap[(long long)f * fshot] = v;
            }
        }
    }
}

// Non-finite check of the receiver traces: sets *flag if any sample is NaN/Inf.
template <typename T>
__global__ void finite_check_kernel(const T *__restrict__ x, long long n, int *flag) {
    int bad = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        bad |= !isfinite((double)x[e]);
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

}  // namespace mittet
