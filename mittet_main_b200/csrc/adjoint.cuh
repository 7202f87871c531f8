// adjoint.cuh -- discrete adjoint of the forward step, for the FWI gradient.
//
// The forward step is linear in the state (E, H, psi_E, psi_H) for a fixed
// model; its transpose is applied step by step in reverse time.  Each half
// step's transpose is split in two kernels so that no kernel reads a
// neighbour value another thread writes:
//   *_own  (one cell): from the adjoint of the phase output it forms the
//          adjoint weight mu of every derivative the phase used at that cell,
//          the cell's gradient terms, and the adjoint of the phase input of
//          its own field (lambda <- ca lambda, psi-adjoint <- b psi-adjoint);
//   *_gather: adds the transposed (2,4) differences of those mu to the
//          other field's adjoint, reading mu at the neighbours (the gradient
//          launches adjv_*_gather, several x cells per thread; adj_*_gather,
//          one cell per thread, gives the same bits).
// Adjoint step n (reverse of forward step n):
//   inject a_H[n] -> lambda_H ; H_own ; H_gather (-> lambda_E) ;
//   inject a_E[n] -> lambda_E ; source terms ; E_own ; E_gather (-> lambda_H).
// Gradient of the misfit with respect to sigma (m = 2 w0 dt / sigma):
//   E phase, every cell:  lambda_E1 [ (in range) dca E0 + (dcb/cb)(E1 - (in range ? ca E0 : E0)) ],
//     h = esig m / 2, ca = (1-h)/(1+h), dca = 2h/(sigma(1+h)^2), dcb/cb = -1/(sigma(1+h));
//   H phase, CPML cells:  lambda_H1 [ (in range) dda H0 + (ddb/db)(H1 - (in range ? da H0 : H0)) ],
//     h = msig m / 2, dda = 2h/(sigma(1+h)^2), ddb/db = h/(sigma(1+h));
//   electric source gain dt 2 w0/(sigma vol): lambda_E1s g w / sigma.
#pragma once

namespace mittet {

template <typename T>
struct AdjArgs {
    // forward states of this step: E0, H0 = state before the step, E1, H1 = after
    const T *E0[3], *H0[3], *E1[3], *H1[3];
    T *lam[6];        // adjoint fields Ex..Hz, [shot][cell]
    T *lpsi[3][2];    // adjoint psi of this phase's slab groups
    T *mu[7];         // derivative adjoint weights
    double *grad;     // [shot][cell] gradient accumulators
    const T *m;       // model word 2 w0 dt / sigma
    const T *dtmu;
    T dtmu0;
    const T *prof;
    int nmax;
    int nx, ny, nz, px;
    long long plane, fshot;
    long long pshot[3];
    DBox upd[3];
    DSlab slab[3];
    T c1, c2, c2t, sgn;
    double inv2w0dt;  // 1/(2 w0 dt): 1/sigma = m * inv2w0dt
    // Interior box of this phase (no CPML profile, no psi slab, inside every
    // update range, derivative defined; empty if none): there *_own leaves
    // lambda unchanged and only stores mu (and, for E, the gradient term).
    DBox ibox;
    T ik[3];          // 1/d per axis (the interior 1/ked, 1/khd)
};

__device__ __forceinline__ bool adj_cell(int &i, int &j, int &k, int &shot, int nx, int ny, int nz) {
    i = blockIdx.x * blockDim.x + threadIdx.x;
    j = blockIdx.y * blockDim.y + threadIdx.y;
    const int zz = blockIdx.z;
    k = zz % nz;
    shot = zz / nz;
    return i < nx && j < ny;
}

template <typename T>
__device__ __forceinline__ T pget(const AdjArgs<T> &a, int axis, int which, int v) {
    return __ldg(a.prof + ((size_t)axis * 8 + which) * a.nmax + v);
}

// Each kernel loads what its cell needs up front and passes the values to a
// per-cell function.  Measured alternatives that were slower on the
// 128x128x96, 16-shot gradient (about two thirds of its cells in CPML slabs):
// four x cells per thread with vector loads (the lanes serialise the general
// path), and gathers that form the weights of deep-interior neighbours from
// the adjoint fields instead of reading them (more loads: the model at every
// E tap).

// Taps of a (2,4) transposed difference along one axis; o* tell whether a
// tap lies inside the grid.
// (D+^T mu)[u] = c1 mu[u-1] - c1 mu[u] + c2 mu[u-2] - c2 mu[u+1];  typo: c2t replaces c1 on mu[u]
template <typename T>
__device__ __forceinline__ T dplus_v(T mc, T mm1, T mm2, T mp1, bool o1, bool o2, bool op, T c1, T c2, T c1u) {
    T r = -c1u * mc;
    if (o1) r = fma(c1, mm1, r);
    if (o2) r = fma(c2, mm2, r);
    if (op) r = fma(-c2, mp1, r);
    return r;
}
// (D^T mu)[u] = c1 mu[u] - c1 mu[u+1] + c2 mu[u-1] - c2 mu[u+2]
template <typename T>
__device__ __forceinline__ T dminus_v(T mc, T mm1, T mp1, T mp2, bool om, bool op1, bool op2, T c1, T c2) {
    T r = c1 * mc;
    if (op1) r = fma(-c1, mp1, r);
    if (om) r = fma(c2, mm1, r);
    if (op2) r = fma(-c2, mp2, r);
    return r;
}

// ---------------------------------------------------------------- H phase
// mu[0] Dy+Ez, mu[1] Dz+Ey, mu[2] Dz+Ex, mu[3] Dx+Ez, mu[4] typo Dx Ez (psi_Hyx), mu[5] Dx+Ey, mu[6] Dy+Ex

// Resident 256-thread blocks per SM asked of the own kernels: 6 in FP32
// (40 registers, a few bytes of spill; latency-bound, they gain from the
// extra warps: adjoint 6.5 -> 6.2 s), 4 in FP64 (more would spill heavily).
template <typename T>
constexpr int kOwnMinBlocks() {
    return sizeof(T) == 4 ? 6 : 4;
}

// Own half of the transposed H update at one cell: from the adjoint L of H
// after the phase and dt/mu, the seven weights mu and the adjoint of H
// before the phase (lam); the cell's psi adjoints and gradient (CPML cells)
// are updated in memory.  Returns whether lam differs from L.
template <typename T>
__device__ __forceinline__ bool h_own_cell(const AdjArgs<T> &a, int i, int j, int k, int shot, long long c,
                                           long long cm, T L0, T L1, T L2, T dm, T (&mu)[7], T (&lam)[3]) {
    const T s = a.sgn;
    lam[0] = L0; lam[1] = L1; lam[2] = L2;
    if (in_box(a.ibox, i, j, k)) {
        // da = 1, db = dt/mu, every update in range, no psi, no gradient term
        mu[0] = -s * dm * a.ik[1] * L0;
        mu[1] = s * dm * a.ik[2] * L0;
        mu[2] = -s * dm * a.ik[2] * L1;
        mu[3] = s * dm * a.ik[0] * L1;
        mu[4] = T(0);
        mu[5] = -s * dm * a.ik[0] * L2;
        mu[6] = s * dm * a.ik[1] * L2;
        return false;
    }
    const T m = a.m[cm];
    const T msh[3] = {pget(a, 0, 1, i), pget(a, 1, 1, j), pget(a, 2, 1, k)};
    const T ik[3] = {pget(a, 0, 7, i), pget(a, 1, 7, j), pget(a, 2, 7, k)};
    T da[3], db[3];
    for (int q = 0; q < 3; q++) {
        if (msh[q] != T(0)) {
            const T h = msh[q] * m;
            const T r = rcp(T(1) + h);
            da[q] = (T(1) - h) * r;
            db[q] = dm * r;
        } else {
            da[q] = T(1);
            db[q] = dm;
        }
    }
    const bool in0 = in_box(a.upd[0], i, j, k), in1 = in_box(a.upd[1], i, j, k), in2 = in_box(a.upd[2], i, j, k);
    T mu0 = in0 ? -s * db[0] * ik[1] * L0 : T(0);
    T mu1 = in0 ? s * db[0] * ik[2] * L0 : T(0);
    T mu2 = in1 ? -s * db[1] * ik[2] * L1 : T(0);
    T mu3 = in1 ? s * db[1] * ik[0] * L1 : T(0);
    T mu4 = T(0);
    T mu5 = in2 ? -s * db[2] * ik[0] * L2 : T(0);
    T mu6 = in2 ? s * db[2] * ik[1] * L2 : T(0);
    // slab psi adjoints
    const int lx = slab_local(a.slab[0], i), ly = slab_local(a.slab[1], j), lz = slab_local(a.slab[2], k);
    if (lx >= 0 && j >= a.slab[0].other.lo[1] && j < a.slab[0].other.hi[1] && k >= a.slab[0].other.lo[2] &&
        k < a.slab[0].other.hi[2]) {
        const long long o = (long long)shot * a.pshot[0] + ((long long)k * a.ny + j) * a.slab[0].width + lx;
        const T bh = pget(a, 0, 4, i), chd = pget(a, 0, 5, i);
        const T lzx = fma(-db[2], L2, a.lpsi[0][0][o]);  // psi_Hzx
        const T lyx = fma(db[1], L1, a.lpsi[0][1][o]);   // psi_Hyx
        a.lpsi[0][0][o] = bh * lzx;
        a.lpsi[0][1][o] = bh * lyx;
        mu5 = fma(chd, lzx, mu5);
        mu4 = fma(chd, lyx, mu4);
    }
    if (ly >= 0 && i >= a.slab[1].other.lo[0] && i < a.slab[1].other.hi[0] && k >= a.slab[1].other.lo[2] &&
        k < a.slab[1].other.hi[2]) {
        const long long o = (long long)shot * a.pshot[1] + ((long long)k * a.slab[1].width + ly) * a.px + i;
        const T bh = pget(a, 1, 4, j), chd = pget(a, 1, 5, j);
        const T lxy = fma(-db[0], L0, a.lpsi[1][0][o]);  // psi_Hxy
        const T lzy = fma(db[2], L2, a.lpsi[1][1][o]);   // psi_Hzy
        a.lpsi[1][0][o] = bh * lxy;
        a.lpsi[1][1][o] = bh * lzy;
        mu0 = fma(chd, lxy, mu0);
        mu6 = fma(chd, lzy, mu6);
    }
    if (lz >= 0 && i >= a.slab[2].other.lo[0] && i < a.slab[2].other.hi[0] && j >= a.slab[2].other.lo[1] &&
        j < a.slab[2].other.hi[1]) {
        const long long o = (long long)shot * a.pshot[2] + ((long long)lz * a.ny + j) * a.px + i;
        const T bh = pget(a, 2, 4, k), chd = pget(a, 2, 5, k);
        const T lyz = fma(-db[1], L1, a.lpsi[2][0][o]);  // psi_Hyz
        const T lxz = fma(db[0], L0, a.lpsi[2][1][o]);   // psi_Hxz
        a.lpsi[2][0][o] = bh * lyz;
        a.lpsi[2][1][o] = bh * lxz;
        mu2 = fma(chd, lyz, mu2);
        mu1 = fma(chd, lxz, mu1);
    }
    mu[0] = mu0; mu[1] = mu1; mu[2] = mu2; mu[3] = mu3; mu[4] = mu4; mu[5] = mu5; mu[6] = mu6;
    // gradient (CPML cells only: interior da, db do not depend on sigma)
    double gsum = 0.0;
    const double isig = (double)m * a.inv2w0dt;
    const bool in[3] = {in0, in1, in2};
    const T L[3] = {L0, L1, L2};
    for (int q = 0; q < 3; q++) {
        if (msh[q] == T(0)) continue;
        const double h = (double)msh[q] * (double)m;
        const double r = 1.0 / (1.0 + h);
        const double dda = 2.0 * h * isig * r * r;
        const double rdb = h * isig * r;
        const double h0 = (double)a.H0[q][c], h1 = (double)a.H1[q][c];
        const double d = in[q] ? fma(-(double)da[q], h0, h1) : h1 - h0;
        gsum = fma((double)L[q], fma(rdb, d, in[q] ? dda * h0 : 0.0), gsum);
    }
    if (gsum != 0.0) a.grad[c] += gsum;
    lam[0] = in0 ? da[0] * L0 : L0;
    lam[1] = in1 ? da[1] * L1 : L1;
    lam[2] = in2 ? da[2] * L2 : L2;
    return true;
}

template <typename T>
__global__ void __launch_bounds__(256, kOwnMinBlocks<T>()) adj_h_own_kernel(AdjArgs<T> a) {
    int i, j, k, shot;
    if (!adj_cell(i, j, k, shot, a.nx, a.ny, a.nz)) return;
    const long long cm = (long long)k * a.plane + (long long)j * a.px + i;
    const long long c = (long long)shot * a.fshot + cm;
    const T dm = a.dtmu ? a.dtmu[cm] : a.dtmu0;
    T mu[7], lam[3];
    const bool ch = h_own_cell(a, i, j, k, shot, c, cm, a.lam[3][c], a.lam[4][c], a.lam[5][c], dm, mu, lam);
#pragma unroll
    for (int w = 0; w < 7; w++) a.mu[w][c] = mu[w];
    if (ch) { a.lam[3][c] = lam[0]; a.lam[4][c] = lam[1]; a.lam[5][c] = lam[2]; }
}

// h_own_cell for the cells of one box of the phase's tile map (stencil.cuh
// TileMap): along an axis whose bit is clear in GM every cell of the box is
// interior (no profile, no psi slab, inside every update range), so the
// general path drops that axis's profile loads, range and slab tests at
// compile time; GM = 0 is the interior body.  The arithmetic of every term
// is the same as in h_own_cell, so the results are bit-identical.
template <typename T, int GM>
__device__ __forceinline__ bool h_own_cell_gm(const AdjArgs<T> &a, int i, int j, int k, int shot, long long c,
                                              long long cm, T L0, T L1, T L2, T dm, T (&mu)[7], T (&lam)[3]) {
    constexpr bool G[3] = {(GM & 1) != 0, (GM & 2) != 0, (GM & 4) != 0};
    const T s = a.sgn;
    lam[0] = L0; lam[1] = L1; lam[2] = L2;
    if constexpr (GM == 0) {
        mu[0] = -s * dm * a.ik[1] * L0;
        mu[1] = s * dm * a.ik[2] * L0;
        mu[2] = -s * dm * a.ik[2] * L1;
        mu[3] = s * dm * a.ik[0] * L1;
        mu[4] = T(0);
        mu[5] = -s * dm * a.ik[0] * L2;
        mu[6] = s * dm * a.ik[1] * L2;
        return false;
    } else {
        const int v3[3] = {i, j, k};
        const T m = a.m[cm];
        T msh[3], ik[3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            msh[q] = G[q] ? pget(a, q, 1, v3[q]) : T(0);
            ik[q] = G[q] ? pget(a, q, 7, v3[q]) : a.ik[q];
        }
        T da[3], db[3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            if (G[q] && msh[q] != T(0)) {
                const T h = msh[q] * m;
                const T r = rcp(T(1) + h);
                da[q] = (T(1) - h) * r;
                db[q] = dm * r;
            } else {
                da[q] = T(1);
                db[q] = dm;
            }
        }
        auto in_gm = [&](const DBox &b) {
            bool in = true;
#pragma unroll
            for (int q = 0; q < 3; q++)
                if (G[q]) in = in && v3[q] >= b.lo[q] && v3[q] < b.hi[q];
            return in;
        };
        const bool in0 = in_gm(a.upd[0]), in1 = in_gm(a.upd[1]), in2 = in_gm(a.upd[2]);
        T mu0 = in0 ? -s * db[0] * ik[1] * L0 : T(0);
        T mu1 = in0 ? s * db[0] * ik[2] * L0 : T(0);
        T mu2 = in1 ? -s * db[1] * ik[2] * L1 : T(0);
        T mu3 = in1 ? s * db[1] * ik[0] * L1 : T(0);
        T mu4 = T(0);
        T mu5 = in2 ? -s * db[2] * ik[0] * L2 : T(0);
        T mu6 = in2 ? s * db[2] * ik[1] * L2 : T(0);
        if (G[0]) {
            const int lx = slab_local(a.slab[0], i);
            if (lx >= 0 && j >= a.slab[0].other.lo[1] && j < a.slab[0].other.hi[1] && k >= a.slab[0].other.lo[2] &&
                k < a.slab[0].other.hi[2]) {
                const long long o = (long long)shot * a.pshot[0] + ((long long)k * a.ny + j) * a.slab[0].width + lx;
                const T bh = pget(a, 0, 4, i), chd = pget(a, 0, 5, i);
                const T lzx = fma(-db[2], L2, a.lpsi[0][0][o]);
                const T lyx = fma(db[1], L1, a.lpsi[0][1][o]);
                a.lpsi[0][0][o] = bh * lzx;
                a.lpsi[0][1][o] = bh * lyx;
                mu5 = fma(chd, lzx, mu5);
                mu4 = fma(chd, lyx, mu4);
            }
        }
        if (G[1]) {
            const int ly = slab_local(a.slab[1], j);
            if (ly >= 0 && i >= a.slab[1].other.lo[0] && i < a.slab[1].other.hi[0] && k >= a.slab[1].other.lo[2] &&
                k < a.slab[1].other.hi[2]) {
                const long long o = (long long)shot * a.pshot[1] + ((long long)k * a.slab[1].width + ly) * a.px + i;
                const T bh = pget(a, 1, 4, j), chd = pget(a, 1, 5, j);
                const T lxy = fma(-db[0], L0, a.lpsi[1][0][o]);
                const T lzy = fma(db[2], L2, a.lpsi[1][1][o]);
                a.lpsi[1][0][o] = bh * lxy;
                a.lpsi[1][1][o] = bh * lzy;
                mu0 = fma(chd, lxy, mu0);
                mu6 = fma(chd, lzy, mu6);
            }
        }
        if (G[2]) {
            const int lz = slab_local(a.slab[2], k);
            if (lz >= 0 && i >= a.slab[2].other.lo[0] && i < a.slab[2].other.hi[0] && j >= a.slab[2].other.lo[1] &&
                j < a.slab[2].other.hi[1]) {
                const long long o = (long long)shot * a.pshot[2] + ((long long)lz * a.ny + j) * a.px + i;
                const T bh = pget(a, 2, 4, k), chd = pget(a, 2, 5, k);
                const T lyz = fma(-db[1], L1, a.lpsi[2][0][o]);
                const T lxz = fma(db[0], L0, a.lpsi[2][1][o]);
                a.lpsi[2][0][o] = bh * lyz;
                a.lpsi[2][1][o] = bh * lxz;
                mu2 = fma(chd, lyz, mu2);
                mu1 = fma(chd, lxz, mu1);
            }
        }
        mu[0] = mu0; mu[1] = mu1; mu[2] = mu2; mu[3] = mu3; mu[4] = mu4; mu[5] = mu5; mu[6] = mu6;
        double gsum = 0.0;
        const double isig = (double)m * a.inv2w0dt;
        const bool in[3] = {in0, in1, in2};
        const T L[3] = {L0, L1, L2};
#pragma unroll
        for (int q = 0; q < 3; q++) {
            if (!G[q] || msh[q] == T(0)) continue;
            const double h = (double)msh[q] * (double)m;
            const double r = 1.0 / (1.0 + h);
            const double dda = 2.0 * h * isig * r * r;
            const double rdb = h * isig * r;
            const double h0 = (double)a.H0[q][c], h1 = (double)a.H1[q][c];
            const double d = in[q] ? fma(-(double)da[q], h0, h1) : h1 - h0;
            gsum = fma((double)L[q], fma(rdb, d, in[q] ? dda * h0 : 0.0), gsum);
        }
        if (gsum != 0.0) a.grad[c] += gsum;
        lam[0] = in0 ? da[0] * L0 : L0;
        lam[1] = in1 ? da[1] * L1 : L1;
        lam[2] = in2 ? da[2] * L2 : L2;
        return true;
    }
}

// The cells of the boxes [q0, q1) of the H phase's one-cell tile map, one
// thread per cell (tiles [first, first + gridDim.x), blockIdx.y = shot).
template <typename T, int GM>
__global__ void __launch_bounds__(256, kOwnMinBlocks<T>())
    adj_h_own_part_kernel(AdjArgs<T> a, const TileMap *__restrict__ tm, int first, int q0, int q1) {
    int i, j, kb, ke;
    bool inside;
    locate<1, 32, 8>(tm, q0, q1, first + blockIdx.x, i, j, kb, ke, inside);
    if (!inside) return;
    const int shot = blockIdx.y, k = kb;
    const long long cm = (long long)k * a.plane + (long long)j * a.px + i;
    const long long c = (long long)shot * a.fshot + cm;
    const T dm = a.dtmu ? a.dtmu[cm] : a.dtmu0;
    T mu[7], lam[3];
    const bool ch = h_own_cell_gm<T, GM>(a, i, j, k, shot, c, cm, a.lam[3][c], a.lam[4][c], a.lam[5][c], dm, mu, lam);
#pragma unroll
    for (int w = 0; w < 7; w++) a.mu[w][c] = mu[w];
    if (ch) { a.lam[3][c] = lam[0]; a.lam[4][c] = lam[1]; a.lam[5][c] = lam[2]; }
}

// Taps [u, u-1, u-2, u+1] of one weight array along one axis (stride s).
template <typename T>
__device__ __forceinline__ void taps_p(const T *__restrict__ mu, long long c, long long s, int v, int n, T (&t)[4]) {
    t[0] = mu[c];
    t[1] = v >= 1 ? mu[c - s] : T(0);
    t[2] = v >= 2 ? mu[c - 2 * s] : T(0);
    t[3] = v + 1 < n ? mu[c + s] : T(0);
}

// Gather half of the transposed H update at one cell, from the taps
// [u, u-1, u-2, u+1] of the seven weights: adds the transposed differences
// to the cell's lambda_E (lx, ly, lz).
template <typename T>
__device__ __forceinline__ void h_gather_cell(const AdjArgs<T> &a, int i, int j, int k, const T (&t0)[4],
                                              const T (&t1)[4], const T (&t2)[4], const T (&t3)[4], const T (&t4)[4],
                                              const T (&t5)[4], const T (&t6)[4], T &lx, T &ly, T &lz) {
    const T c1 = a.c1, c2 = a.c2;
    const bool y1 = j >= 1, y2 = j >= 2, yp = j + 1 < a.ny;
    const bool z1 = k >= 1, z2 = k >= 2, zp = k + 1 < a.nz;
    const bool x1 = i >= 1, x2 = i >= 2, xp = i + 1 < a.nx;
    const T gz = dplus_v(t0[0], t0[1], t0[2], t0[3], y1, y2, yp, c1, c2, c1) +
                 dplus_v(t3[0], t3[1], t3[2], t3[3], x1, x2, xp, c1, c2, c1) +
                 dplus_v(t4[0], t4[1], t4[2], t4[3], x1, x2, xp, c1, c2, a.c2t);
    const T gy = dplus_v(t1[0], t1[1], t1[2], t1[3], z1, z2, zp, c1, c2, c1) +
                 dplus_v(t5[0], t5[1], t5[2], t5[3], x1, x2, xp, c1, c2, c1);
    const T gx = dplus_v(t2[0], t2[1], t2[2], t2[3], z1, z2, zp, c1, c2, c1) +
                 dplus_v(t6[0], t6[1], t6[2], t6[3], y1, y2, yp, c1, c2, c1);
    lx += gx;
    ly += gy;
    lz += gz;
}

template <typename T>
__global__ void adj_h_gather_kernel(AdjArgs<T> a) {
    int i, j, k, shot;
    if (!adj_cell(i, j, k, shot, a.nx, a.ny, a.nz)) return;
    const long long c = (long long)shot * a.fshot + (long long)k * a.plane + (long long)j * a.px + i;
    const long long sy = a.px, sz = a.plane;
    T t0[4], t1[4], t2[4], t3[4], t4[4], t5[4], t6[4];
    taps_p(a.mu[0], c, sy, j, a.ny, t0);
    taps_p(a.mu[1], c, sz, k, a.nz, t1);
    taps_p(a.mu[2], c, sz, k, a.nz, t2);
    taps_p(a.mu[3], c, 1, i, a.nx, t3);
    taps_p(a.mu[4], c, 1, i, a.nx, t4);
    taps_p(a.mu[5], c, 1, i, a.nx, t5);
    taps_p(a.mu[6], c, sy, j, a.ny, t6);
    T lx = a.lam[0][c], ly = a.lam[1][c], lz = a.lam[2][c];
    h_gather_cell(a, i, j, k, t0, t1, t2, t3, t4, t5, t6, lx, ly, lz);
    a.lam[0][c] = lx;
    a.lam[1][c] = ly;
    a.lam[2][c] = lz;
}

// ---------------------------------------------------------------- E phase
// mu[0] DyHz, mu[1] DzHy, mu[2] DzHx, mu[3] DxHz, mu[4] DxHy, mu[5] DyHx

// Own half of the transposed E update at one cell, from the adjoint L of E
// after the phase, the model word m, the cell's E before (e0) and after (e1)
// the phase and its gradient accumulator g (returned updated): the six
// weights mu and the adjoint of E before the phase (lam); psi adjoints are
// updated in memory.  Returns whether lam differs from L.
template <typename T>
__device__ __forceinline__ bool e_own_cell(const AdjArgs<T> &a, int i, int j, int k, int shot, T m, T L0, T L1,
                                           T L2, const T (&e0)[3], const T (&e1)[3], double &g, T (&mu)[6],
                                           T (&lam)[3]) {
    const T s = a.sgn;
    lam[0] = L0; lam[1] = L1; lam[2] = L2;
    const T L[3] = {L0, L1, L2};
    const double isig = (double)m * a.inv2w0dt;
    if (in_box(a.ibox, i, j, k)) {
        // ca = 1, cb = m, every update in range, no psi; h = 0: dca = 0,
        // dcb/cb = -1/sigma
        mu[0] = s * m * a.ik[1] * L0;
        mu[1] = -s * m * a.ik[2] * L0;
        mu[2] = s * m * a.ik[2] * L1;
        mu[3] = -s * m * a.ik[0] * L1;
        mu[4] = s * m * a.ik[0] * L2;
        mu[5] = -s * m * a.ik[1] * L2;
        const double rcb = -isig;
        double gsum = 0.0;
#pragma unroll
        for (int q = 0; q < 3; q++) gsum = fma((double)L[q], rcb * ((double)e1[q] - (double)e0[q]), gsum);
        g += gsum;
        return false;
    }
    const T esh[3] = {pget(a, 0, 0, i), pget(a, 1, 0, j), pget(a, 2, 0, k)};
    const T ik[3] = {pget(a, 0, 6, i), pget(a, 1, 6, j), pget(a, 2, 6, k)};
    T ca[3], cb[3];
    for (int q = 0; q < 3; q++) {
        if (esh[q] != T(0)) {
            const T h = esh[q] * m;
            const T r = rcp(T(1) + h);
            ca[q] = (T(1) - h) * r;
            cb[q] = m * r;
        } else {
            ca[q] = T(1);
            cb[q] = m;
        }
    }
    const bool in0 = in_box(a.upd[0], i, j, k), in1 = in_box(a.upd[1], i, j, k), in2 = in_box(a.upd[2], i, j, k);
    T mu0 = in0 ? s * cb[0] * ik[1] * L0 : T(0);   // DyHz
    T mu1 = in0 ? -s * cb[0] * ik[2] * L0 : T(0);  // DzHy
    T mu2 = in1 ? s * cb[1] * ik[2] * L1 : T(0);   // DzHx
    T mu3 = in1 ? -s * cb[1] * ik[0] * L1 : T(0);  // DxHz
    T mu4 = in2 ? s * cb[2] * ik[0] * L2 : T(0);   // DxHy
    T mu5 = in2 ? -s * cb[2] * ik[1] * L2 : T(0);  // DyHx
    const int lx = slab_local(a.slab[0], i), ly = slab_local(a.slab[1], j), lz = slab_local(a.slab[2], k);
    if (lx >= 0 && j >= a.slab[0].other.lo[1] && j < a.slab[0].other.hi[1] && k >= a.slab[0].other.lo[2] &&
        k < a.slab[0].other.hi[2]) {
        const long long o = (long long)shot * a.pshot[0] + ((long long)k * a.ny + j) * a.slab[0].width + lx;
        const T be = pget(a, 0, 2, i), ced = pget(a, 0, 3, i);
        const T lzx = fma(cb[2], L2, a.lpsi[0][0][o]);   // psi_Ezx
        const T lyx = fma(-cb[1], L1, a.lpsi[0][1][o]);  // psi_Eyx
        a.lpsi[0][0][o] = be * lzx;
        a.lpsi[0][1][o] = be * lyx;
        mu4 = fma(ced, lzx, mu4);
        mu3 = fma(ced, lyx, mu3);
    }
    if (ly >= 0 && i >= a.slab[1].other.lo[0] && i < a.slab[1].other.hi[0] && k >= a.slab[1].other.lo[2] &&
        k < a.slab[1].other.hi[2]) {
        const long long o = (long long)shot * a.pshot[1] + ((long long)k * a.slab[1].width + ly) * a.px + i;
        const T be = pget(a, 1, 2, j), ced = pget(a, 1, 3, j);
        const T lxy = fma(cb[0], L0, a.lpsi[1][0][o]);   // psi_Exy
        const T lzy = fma(-cb[2], L2, a.lpsi[1][1][o]);  // psi_Ezy
        a.lpsi[1][0][o] = be * lxy;
        a.lpsi[1][1][o] = be * lzy;
        mu0 = fma(ced, lxy, mu0);
        mu5 = fma(ced, lzy, mu5);
    }
    if (lz >= 0 && i >= a.slab[2].other.lo[0] && i < a.slab[2].other.hi[0] && j >= a.slab[2].other.lo[1] &&
        j < a.slab[2].other.hi[1]) {
        const long long o = (long long)shot * a.pshot[2] + ((long long)lz * a.ny + j) * a.px + i;
        const T be = pget(a, 2, 2, k), ced = pget(a, 2, 3, k);
        const T lyz = fma(cb[1], L1, a.lpsi[2][0][o]);   // psi_Eyz
        const T lxz = fma(-cb[0], L0, a.lpsi[2][1][o]);  // psi_Exz
        a.lpsi[2][0][o] = be * lyz;
        a.lpsi[2][1][o] = be * lxz;
        mu2 = fma(ced, lyz, mu2);
        mu1 = fma(ced, lxz, mu1);
    }
    mu[0] = mu0; mu[1] = mu1; mu[2] = mu2; mu[3] = mu3; mu[4] = mu4; mu[5] = mu5;
    // gradient: every cell (cb = m/(1+h) depends on sigma everywhere)
    const bool in[3] = {in0, in1, in2};
    double gsum = 0.0;
    for (int q = 0; q < 3; q++) {
        // an axis without CPML profile (h = 0) gives dca = 0, rcb = -1/sigma
        // exactly: skip its FP64 division
        const bool prof = esh[q] != T(0);
        const double h = (double)esh[q] * (double)m;
        const double r = prof ? 1.0 / (1.0 + h) : 1.0;
        const double dca = prof ? 2.0 * h * isig * r * r : 0.0;
        const double rcb = -isig * r;
        const double x0 = (double)e0[q], x1 = (double)e1[q];
        const double d = in[q] ? fma(-(double)ca[q], x0, x1) : x1 - x0;
        gsum = fma((double)L[q], fma(rcb, d, in[q] ? dca * x0 : 0.0), gsum);
    }
    g += gsum;
    lam[0] = in0 ? ca[0] * L0 : L0;
    lam[1] = in1 ? ca[1] * L1 : L1;
    lam[2] = in2 ? ca[2] * L2 : L2;
    return true;
}

template <typename T>
__global__ void __launch_bounds__(256, kOwnMinBlocks<T>()) adj_e_own_kernel(AdjArgs<T> a) {
    int i, j, k, shot;
    if (!adj_cell(i, j, k, shot, a.nx, a.ny, a.nz)) return;
    const long long cm = (long long)k * a.plane + (long long)j * a.px + i;
    const long long c = (long long)shot * a.fshot + cm;
    const T e0[3] = {a.E0[0][c], a.E0[1][c], a.E0[2][c]}, e1[3] = {a.E1[0][c], a.E1[1][c], a.E1[2][c]};
    double g = a.grad[c];
    T mu[6], lam[3];
    const bool ch = e_own_cell(a, i, j, k, shot, a.m[cm], a.lam[0][c], a.lam[1][c], a.lam[2][c], e0, e1, g, mu, lam);
    a.grad[c] = g;
#pragma unroll
    for (int w = 0; w < 6; w++) a.mu[w][c] = mu[w];
    if (ch) { a.lam[0][c] = lam[0]; a.lam[1][c] = lam[1]; a.lam[2][c] = lam[2]; }
}

// e_own_cell for the cells of one box of the E phase's tile map, with the
// axes not in GM interior at compile time (see h_own_cell_gm); GM = 0 is
// the interior body.  Bit-identical to e_own_cell.
template <typename T, int GM>
__device__ __forceinline__ bool e_own_cell_gm(const AdjArgs<T> &a, int i, int j, int k, int shot, T m, T L0, T L1,
                                              T L2, const T (&e0)[3], const T (&e1)[3], double &g, T (&mu)[6],
                                              T (&lam)[3]) {
    constexpr bool G[3] = {(GM & 1) != 0, (GM & 2) != 0, (GM & 4) != 0};
    const T s = a.sgn;
    lam[0] = L0; lam[1] = L1; lam[2] = L2;
    const T L[3] = {L0, L1, L2};
    const double isig = (double)m * a.inv2w0dt;
    if constexpr (GM == 0) {
        mu[0] = s * m * a.ik[1] * L0;
        mu[1] = -s * m * a.ik[2] * L0;
        mu[2] = s * m * a.ik[2] * L1;
        mu[3] = -s * m * a.ik[0] * L1;
        mu[4] = s * m * a.ik[0] * L2;
        mu[5] = -s * m * a.ik[1] * L2;
        const double rcb = -isig;
        double gsum = 0.0;
#pragma unroll
        for (int q = 0; q < 3; q++) gsum = fma((double)L[q], rcb * ((double)e1[q] - (double)e0[q]), gsum);
        g += gsum;
        return false;
    } else {
        const int v3[3] = {i, j, k};
        T esh[3], ik[3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            esh[q] = G[q] ? pget(a, q, 0, v3[q]) : T(0);
            ik[q] = G[q] ? pget(a, q, 6, v3[q]) : a.ik[q];
        }
        T ca[3], cb[3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            if (G[q] && esh[q] != T(0)) {
                const T h = esh[q] * m;
                const T r = rcp(T(1) + h);
                ca[q] = (T(1) - h) * r;
                cb[q] = m * r;
            } else {
                ca[q] = T(1);
                cb[q] = m;
            }
        }
        auto in_gm = [&](const DBox &b) {
            bool in = true;
#pragma unroll
            for (int q = 0; q < 3; q++)
                if (G[q]) in = in && v3[q] >= b.lo[q] && v3[q] < b.hi[q];
            return in;
        };
        const bool in0 = in_gm(a.upd[0]), in1 = in_gm(a.upd[1]), in2 = in_gm(a.upd[2]);
        T mu0 = in0 ? s * cb[0] * ik[1] * L0 : T(0);
        T mu1 = in0 ? -s * cb[0] * ik[2] * L0 : T(0);
        T mu2 = in1 ? s * cb[1] * ik[2] * L1 : T(0);
        T mu3 = in1 ? -s * cb[1] * ik[0] * L1 : T(0);
        T mu4 = in2 ? s * cb[2] * ik[0] * L2 : T(0);
        T mu5 = in2 ? -s * cb[2] * ik[1] * L2 : T(0);
        if (G[0]) {
            const int lx = slab_local(a.slab[0], i);
            if (lx >= 0 && j >= a.slab[0].other.lo[1] && j < a.slab[0].other.hi[1] && k >= a.slab[0].other.lo[2] &&
                k < a.slab[0].other.hi[2]) {
                const long long o = (long long)shot * a.pshot[0] + ((long long)k * a.ny + j) * a.slab[0].width + lx;
                const T be = pget(a, 0, 2, i), ced = pget(a, 0, 3, i);
                const T lzx = fma(cb[2], L2, a.lpsi[0][0][o]);
                const T lyx = fma(-cb[1], L1, a.lpsi[0][1][o]);
                a.lpsi[0][0][o] = be * lzx;
                a.lpsi[0][1][o] = be * lyx;
                mu4 = fma(ced, lzx, mu4);
                mu3 = fma(ced, lyx, mu3);
            }
        }
        if (G[1]) {
            const int ly = slab_local(a.slab[1], j);
            if (ly >= 0 && i >= a.slab[1].other.lo[0] && i < a.slab[1].other.hi[0] && k >= a.slab[1].other.lo[2] &&
                k < a.slab[1].other.hi[2]) {
                const long long o = (long long)shot * a.pshot[1] + ((long long)k * a.slab[1].width + ly) * a.px + i;
                const T be = pget(a, 1, 2, j), ced = pget(a, 1, 3, j);
                const T lxy = fma(cb[0], L0, a.lpsi[1][0][o]);
                const T lzy = fma(-cb[2], L2, a.lpsi[1][1][o]);
                a.lpsi[1][0][o] = be * lxy;
                a.lpsi[1][1][o] = be * lzy;
                mu0 = fma(ced, lxy, mu0);
                mu5 = fma(ced, lzy, mu5);
            }
        }
        if (G[2]) {
            const int lz = slab_local(a.slab[2], k);
            if (lz >= 0 && i >= a.slab[2].other.lo[0] && i < a.slab[2].other.hi[0] && j >= a.slab[2].other.lo[1] &&
                j < a.slab[2].other.hi[1]) {
                const long long o = (long long)shot * a.pshot[2] + ((long long)lz * a.ny + j) * a.px + i;
                const T be = pget(a, 2, 2, k), ced = pget(a, 2, 3, k);
                const T lyz = fma(cb[1], L1, a.lpsi[2][0][o]);
                const T lxz = fma(-cb[0], L0, a.lpsi[2][1][o]);
                a.lpsi[2][0][o] = be * lyz;
                a.lpsi[2][1][o] = be * lxz;
                mu2 = fma(ced, lyz, mu2);
                mu1 = fma(ced, lxz, mu1);
            }
        }
        mu[0] = mu0; mu[1] = mu1; mu[2] = mu2; mu[3] = mu3; mu[4] = mu4; mu[5] = mu5;
        const bool in[3] = {in0, in1, in2};
        double gsum = 0.0;
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const bool prof = G[q] && esh[q] != T(0);
            const double h = (double)esh[q] * (double)m;
            const double r = prof ? 1.0 / (1.0 + h) : 1.0;
            const double dca = prof ? 2.0 * h * isig * r * r : 0.0;
            const double rcb = -isig * r;
            const double x0 = (double)e0[q], x1 = (double)e1[q];
            const double d = in[q] ? fma(-(double)ca[q], x0, x1) : x1 - x0;
            gsum = fma((double)L[q], fma(rcb, d, in[q] ? dca * x0 : 0.0), gsum);
        }
        g += gsum;
        lam[0] = in0 ? ca[0] * L0 : L0;
        lam[1] = in1 ? ca[1] * L1 : L1;
        lam[2] = in2 ? ca[2] * L2 : L2;
        return true;
    }
}

template <typename T, int GM>
__global__ void __launch_bounds__(256, kOwnMinBlocks<T>())
    adj_e_own_part_kernel(AdjArgs<T> a, const TileMap *__restrict__ tm, int first, int q0, int q1) {
    int i, j, kb, ke;
    bool inside;
    locate<1, 32, 8>(tm, q0, q1, first + blockIdx.x, i, j, kb, ke, inside);
    if (!inside) return;
    const int shot = blockIdx.y, k = kb;
    const long long cm = (long long)k * a.plane + (long long)j * a.px + i;
    const long long c = (long long)shot * a.fshot + cm;
    const T e0[3] = {a.E0[0][c], a.E0[1][c], a.E0[2][c]}, e1[3] = {a.E1[0][c], a.E1[1][c], a.E1[2][c]};
    double g = a.grad[c];
    T mu[6], lam[3];
    const bool ch = e_own_cell_gm<T, GM>(a, i, j, k, shot, a.m[cm], a.lam[0][c], a.lam[1][c], a.lam[2][c], e0, e1, g,
                                         mu, lam);
    a.grad[c] = g;
#pragma unroll
    for (int w = 0; w < 6; w++) a.mu[w][c] = mu[w];
    if (ch) { a.lam[0][c] = lam[0]; a.lam[1][c] = lam[1]; a.lam[2][c] = lam[2]; }
}

// Taps [u, u-1, u+1, u+2] of one weight array along one axis (stride s).
template <typename T>
__device__ __forceinline__ void taps_m(const T *__restrict__ mu, long long c, long long s, int v, int n, T (&t)[4]) {
    t[0] = mu[c];
    t[1] = v >= 1 ? mu[c - s] : T(0);
    t[2] = v + 1 < n ? mu[c + s] : T(0);
    t[3] = v + 2 < n ? mu[c + 2 * s] : T(0);
}

// Gather half of the transposed E update at one cell, from the taps
// [u, u-1, u+1, u+2] of the six weights: adds the transposed differences to
// the cell's lambda_H (lx, ly, lz).
template <typename T>
__device__ __forceinline__ void e_gather_cell(const AdjArgs<T> &a, int i, int j, int k, const T (&t0)[4],
                                              const T (&t1)[4], const T (&t2)[4], const T (&t3)[4], const T (&t4)[4],
                                              const T (&t5)[4], T &lx, T &ly, T &lz) {
    const T c1 = a.c1, c2 = a.c2;
    const bool ym = j >= 1, yp1 = j + 1 < a.ny, yp2 = j + 2 < a.ny;
    const bool zm = k >= 1, zp1 = k + 1 < a.nz, zp2 = k + 2 < a.nz;
    const bool xm = i >= 1, xp1 = i + 1 < a.nx, xp2 = i + 2 < a.nx;
    const T hz = dminus_v(t0[0], t0[1], t0[2], t0[3], ym, yp1, yp2, c1, c2) +
                 dminus_v(t3[0], t3[1], t3[2], t3[3], xm, xp1, xp2, c1, c2);
    const T hy = dminus_v(t1[0], t1[1], t1[2], t1[3], zm, zp1, zp2, c1, c2) +
                 dminus_v(t4[0], t4[1], t4[2], t4[3], xm, xp1, xp2, c1, c2);
    const T hx = dminus_v(t2[0], t2[1], t2[2], t2[3], zm, zp1, zp2, c1, c2) +
                 dminus_v(t5[0], t5[1], t5[2], t5[3], ym, yp1, yp2, c1, c2);
    lx += hx;
    ly += hy;
    lz += hz;
}

template <typename T>
__global__ void adj_e_gather_kernel(AdjArgs<T> a) {
    int i, j, k, shot;
    if (!adj_cell(i, j, k, shot, a.nx, a.ny, a.nz)) return;
    const long long c = (long long)shot * a.fshot + (long long)k * a.plane + (long long)j * a.px + i;
    const long long sy = a.px, sz = a.plane;
    T t0[4], t1[4], t2[4], t3[4], t4[4], t5[4];
    taps_m(a.mu[0], c, sy, j, a.ny, t0);
    taps_m(a.mu[1], c, sz, k, a.nz, t1);
    taps_m(a.mu[2], c, sz, k, a.nz, t2);
    taps_m(a.mu[3], c, 1, i, a.nx, t3);
    taps_m(a.mu[4], c, 1, i, a.nx, t4);
    taps_m(a.mu[5], c, sy, j, a.ny, t5);
    T lx = a.lam[3][c], ly = a.lam[4][c], lz = a.lam[5][c];
    e_gather_cell(a, i, j, k, t0, t1, t2, t3, t4, t5, lx, ly, lz);
    a.lam[3][c] = lx;
    a.lam[4][c] = ly;
    a.lam[5][c] = lz;
}

// ------------------------------------------------ vectorised gathers
// The gathers have no CPML branches, so VX consecutive x cells per thread
// (VX = 4 FP32, 2 FP64; one aligned vector load per weight array and tap)
// pay off there; the own kernels keep one thread per cell, since vector
// lanes would serialise their general path.  Both call the same per-cell
// functions, so the results are bit-identical.

template <int VX>
__device__ __forceinline__ bool adjv_cell(int &i0, int &j, int &k, int &shot, int nx, int ny, int nz) {
    i0 = (blockIdx.x * blockDim.x + threadIdx.x) * VX;
    j = blockIdx.y * blockDim.y + threadIdx.y;
    const int zz = blockIdx.z;
    k = zz % nz;
    shot = zz / nz;
    return i0 < nx && j < ny;
}
// Vector at p, or zeros when !ok.
template <typename T, int VX>
__device__ __forceinline__ void ldv_if(T (&d)[VX], const T *p, bool ok) {
    if (ok) ldv_rw<T, VX>(d, p);
    else zerov<T, VX>(d);
}
// Stores lanes [0, nv) of a vector (the whole vector when nv == VX).
template <typename T, int VX>
__device__ __forceinline__ void stv_n(T *p, const T (&s)[VX], int nv) {
    if (nv == VX) {
        stv<T, VX>(p, s);
    } else {
#pragma unroll
        for (int v = 0; v < VX; v++)
            if (v < nv) p[v] = s[v];
    }
}
// x taps of lane v from the vectors at i0 - VX (l), i0 (m), i0 + VX (r):
// D+ order [u, u-1, u-2, u+1] and D order [u, u-1, u+1, u+2].  Indices are
// clamped so that no branch names an element outside its vector.
template <typename T, int VX>
__device__ __forceinline__ void xtaps_p(const T (&l)[VX], const T (&m)[VX], const T (&r)[VX], int v, T (&t)[4]) {
    t[0] = m[v];
    t[1] = v >= 1 ? m[v >= 1 ? v - 1 : 0] : l[VX - 1];
    t[2] = v >= 2 ? m[v >= 2 ? v - 2 : 0] : l[v < 2 ? VX - 2 + v : 0];
    t[3] = v + 1 < VX ? m[v + 1 < VX ? v + 1 : 0] : r[0];
}
template <typename T, int VX>
__device__ __forceinline__ void xtaps_m(const T (&l)[VX], const T (&m)[VX], const T (&r)[VX], int v, T (&t)[4]) {
    t[0] = m[v];
    t[1] = v >= 1 ? m[v >= 1 ? v - 1 : 0] : l[VX - 1];
    t[2] = v + 1 < VX ? m[v + 1 < VX ? v + 1 : 0] : r[v + 1 >= VX ? v + 1 - VX : 0];
    t[3] = v + 2 < VX ? m[v + 2 < VX ? v + 2 : 0] : r[v + 2 >= VX ? v + 2 - VX : 0];
}

template <typename T, int VX>
__global__ void __launch_bounds__(128) adjv_h_gather_kernel(AdjArgs<T> a) {
    int i0, j, k, shot;
    if (!adjv_cell<VX>(i0, j, k, shot, a.nx, a.ny, a.nz)) return;
    const long long c = (long long)shot * a.fshot + (long long)k * a.plane + (long long)j * a.px + i0;
    const long long sy = a.px, sz = a.plane;
    const int nv = min(VX, a.nx - i0);
    // taps [u, u-1, u-2, u+1] along y and z; x from three whole vectors
    const long long oy[4] = {0, -sy, -2 * sy, sy}, oz[4] = {0, -sz, -2 * sz, sz}, ox[3] = {-VX, 0, VX};
    const bool vy[4] = {true, j >= 1, j >= 2, j + 1 < a.ny}, vz[4] = {true, k >= 1, k >= 2, k + 1 < a.nz};
    const bool vx[3] = {i0 >= VX, true, i0 + VX < a.nx};
    T y0[4][VX], z1[4][VX], z2[4][VX], y6[4][VX], x3[3][VX], x4[3][VX], x5[3][VX];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        ldv_if<T, VX>(y0[q], a.mu[0] + c + oy[q], vy[q]);
        ldv_if<T, VX>(z1[q], a.mu[1] + c + oz[q], vz[q]);
        ldv_if<T, VX>(z2[q], a.mu[2] + c + oz[q], vz[q]);
        ldv_if<T, VX>(y6[q], a.mu[6] + c + oy[q], vy[q]);
    }
#pragma unroll
    for (int q = 0; q < 3; q++) {
        ldv_if<T, VX>(x3[q], a.mu[3] + c + ox[q], vx[q]);
        ldv_if<T, VX>(x4[q], a.mu[4] + c + ox[q], vx[q]);
        ldv_if<T, VX>(x5[q], a.mu[5] + c + ox[q], vx[q]);
    }
    T lx[VX], ly[VX], lz[VX];
    ldv_rw<T, VX>(lx, a.lam[0] + c);
    ldv_rw<T, VX>(ly, a.lam[1] + c);
    ldv_rw<T, VX>(lz, a.lam[2] + c);
#pragma unroll
    for (int v = 0; v < VX; v++) {
        if (v >= nv) continue;
        T t0[4], t1[4], t2[4], t3[4], t4[4], t5[4], t6[4];
#pragma unroll
        for (int q = 0; q < 4; q++) { t0[q] = y0[q][v]; t1[q] = z1[q][v]; t2[q] = z2[q][v]; t6[q] = y6[q][v]; }
        xtaps_p<T, VX>(x3[0], x3[1], x3[2], v, t3);
        xtaps_p<T, VX>(x4[0], x4[1], x4[2], v, t4);
        xtaps_p<T, VX>(x5[0], x5[1], x5[2], v, t5);
        h_gather_cell(a, i0 + v, j, k, t0, t1, t2, t3, t4, t5, t6, lx[v], ly[v], lz[v]);
    }
    stv_n<T, VX>(a.lam[0] + c, lx, nv);
    stv_n<T, VX>(a.lam[1] + c, ly, nv);
    stv_n<T, VX>(a.lam[2] + c, lz, nv);
}

template <typename T, int VX>
__global__ void __launch_bounds__(128) adjv_e_gather_kernel(AdjArgs<T> a) {
    int i0, j, k, shot;
    if (!adjv_cell<VX>(i0, j, k, shot, a.nx, a.ny, a.nz)) return;
    const long long c = (long long)shot * a.fshot + (long long)k * a.plane + (long long)j * a.px + i0;
    const long long sy = a.px, sz = a.plane;
    const int nv = min(VX, a.nx - i0);
    // taps [u, u-1, u+1, u+2]
    const long long oy[4] = {0, -sy, sy, 2 * sy}, oz[4] = {0, -sz, sz, 2 * sz}, ox[3] = {-VX, 0, VX};
    const bool vy[4] = {true, j >= 1, j + 1 < a.ny, j + 2 < a.ny}, vz[4] = {true, k >= 1, k + 1 < a.nz, k + 2 < a.nz};
    const bool vx[3] = {i0 >= VX, true, i0 + VX < a.nx};
    T y0[4][VX], z1[4][VX], z2[4][VX], y5[4][VX], x3[3][VX], x4[3][VX];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        ldv_if<T, VX>(y0[q], a.mu[0] + c + oy[q], vy[q]);
        ldv_if<T, VX>(z1[q], a.mu[1] + c + oz[q], vz[q]);
        ldv_if<T, VX>(z2[q], a.mu[2] + c + oz[q], vz[q]);
        ldv_if<T, VX>(y5[q], a.mu[5] + c + oy[q], vy[q]);
    }
#pragma unroll
    for (int q = 0; q < 3; q++) {
        ldv_if<T, VX>(x3[q], a.mu[3] + c + ox[q], vx[q]);
        ldv_if<T, VX>(x4[q], a.mu[4] + c + ox[q], vx[q]);
    }
    T lx[VX], ly[VX], lz[VX];
    ldv_rw<T, VX>(lx, a.lam[3] + c);
    ldv_rw<T, VX>(ly, a.lam[4] + c);
    ldv_rw<T, VX>(lz, a.lam[5] + c);
#pragma unroll
    for (int v = 0; v < VX; v++) {
        if (v >= nv) continue;
        T t0[4], t1[4], t2[4], t3[4], t4[4], t5[4];
#pragma unroll
        for (int q = 0; q < 4; q++) { t0[q] = y0[q][v]; t1[q] = z1[q][v]; t2[q] = z2[q][v]; t5[q] = y5[q][v]; }
        xtaps_m<T, VX>(x3[0], x3[1], x3[2], v, t3);
        xtaps_m<T, VX>(x4[0], x4[1], x4[2], v, t4);
        e_gather_cell(a, i0 + v, j, k, t0, t1, t2, t3, t4, t5, lx[v], ly[v], lz[v]);
    }
    stv_n<T, VX>(a.lam[3] + c, lx, nv);
    stv_n<T, VX>(a.lam[4] + c, ly, nv);
    stv_n<T, VX>(a.lam[5] + c, lz, nv);
}

// ---------------------------------------------------------------- sources
// Adjoint sources a[shot][rec][n] = sum_f Re(conj(R[shot][rec][f]) W_rf[n]),
// W_rf[n] = hf dt exp((i-1) sqrt(w0 w_f) n dt) with the H factor on H receivers.
__global__ void adj_source_kernel(const double2 *__restrict__ R, int ntr, int nrec, int nf, int nt,
                                  const double *__restrict__ omega, double dt, double omega0,
                                  const unsigned char *__restrict__ is_h, int hfac, double *__restrict__ out) {
    const long long tot = (long long)ntr * nt;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        const int t = (int)(e / nt), n = (int)(e - (long long)t * nt);
        const bool h = hfac && is_h[t % nrec];
        double acc = 0.0;
        for (int f = 0; f < nf; f++) {
            const double xa = sqrt(omega0 * omega[f]) * (double)n * dt;
            double s, cs;
            sincos(xa, &s, &cs);
            const double e0 = exp(-xa) * dt;
            double wr = e0 * cs, wi = e0 * s;
            if (h) {
                const double r = sqrt(2.0 * omega0 / omega[f]) * 0.70710678118654752440;
                const double a2 = wr * r - wi * r, b2 = wr * r + wi * r;
                wr = a2;
                wi = b2;
            }
            const double2 res = R[(long long)t * nf + f];
            acc += res.x * wr + res.y * wi;  // Re(conj(res) * w)
        }
        out[e] = acc;
    }
}

// Adds a[shot][rec][n] to the adjoint field of each receiver of one kind (E or H).
template <typename T>
__global__ void adj_inject_kernel(T *lam0, T *lam1, T *lam2, T *lam3, T *lam4, T *lam5, const long long *rec_off,
                                  const int *rec_comp, int nrec, int nshot, long long fshot, const double *asrc,
                                  int nt, int n, int want_h) {
    T *lam[6] = {lam0, lam1, lam2, lam3, lam4, lam5};
    const int tot = nrec * nshot;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += gridDim.x * blockDim.x) {
        const int s = q / nrec, r = q % nrec;
        const int cpt = rec_comp[r];
        if ((cpt >= 3) != (want_h != 0)) continue;
        atomicAdd(lam[cpt] + (long long)s * fshot + rec_off[r], (T)asrc[(long long)q * nt + n]);
    }
}

struct AdjSrc {
    long long off;   // cell offset within the shot (padded layout)
    long long moff;  // model offset of the cell
    int shot, comp, kind, i, j, k;
    double g;        // gain (as SrcPoint::g)
};

// Source terms of adjoint step n for one kind of point:
//  magnetic (run before the H own kernel, lambda_H is lambda of H after the H phase):
//    the H own kernel used the stored H (before the magnetic injection) as H0; the
//    injection changed H0 by -g w[n+1]: add lambda (d term/d H0) (-g w[n+1]).
//  electric (run before the E own kernel, lambda_E is lambda of E1s):
//    sigma in the gain: + lambda g wbar / sigma, and the E own kernel used E1s as
//    E1 = E1s + g wbar: add lambda (dcb/cb) g wbar.
template <typename T>
__global__ void adj_src_kernel(AdjArgs<T> a, const AdjSrc *__restrict__ pts, int npts, const double *__restrict__ wave,
                               int n, int kind, int shot0, int shot1) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npts) return;
    const AdjSrc p = pts[q];
    if (p.kind != kind || p.shot < shot0 || p.shot >= shot1) return;
    const long long c = (long long)(p.shot - shot0) * a.fshot + p.off;
    const double m = (double)a.m[p.moff];
    const double isig = m * a.inv2w0dt;
    if (kind == 0) {
        if (p.comp < 3) return;
        const int ax = p.comp - 3;
        const int v = ax == 0 ? p.i : (ax == 1 ? p.j : p.k);
        const double msh = (double)pget(a, ax, 1, v);
        if (msh == 0.0) return;
        const double h = msh * m;
        const double da = (1.0 - h) / (1.0 + h);
        const double dda = 2.0 * h * isig / ((1.0 + h) * (1.0 + h));
        const double rdb = h * isig / (1.0 + h);
        const bool in = in_box(a.upd[ax], p.i, p.j, p.k);
        const double dterm = in ? dda - rdb * da : -rdb;
        const double L = (double)a.lam[p.comp][c];
        atomicAdd(a.grad + c, L * dterm * (-p.g * wave[n + 1]));
    } else {
        if (p.comp > 2) return;
        const int ax = p.comp;
        const int v = ax == 0 ? p.i : (ax == 1 ? p.j : p.k);
        const double esh = (double)pget(a, ax, 0, v);
        const double h = esh * m;
        const double rcb = -isig / (1.0 + h);
        const double wbar = (wave[n] + wave[n + 1]) / 2.0;
        const double L = (double)a.lam[p.comp][c];
        atomicAdd(a.grad + c, L * (p.g * wbar * isig + rcb * p.g * wbar));
    }
}

// Copies the six field arrays of a group of shots into one history slot,
// 16 bytes per thread and iteration (len is a multiple of 32 elements, every
// array 16-byte aligned); blockIdx.y is the field.
template <typename T>
__global__ void __launch_bounds__(256) copy_state_kernel(const T *f0, const T *f1, const T *f2, const T *f3,
                                                         const T *f4, const T *f5, T *dst, long long len) {
    constexpr int VX = 16 / sizeof(T);
    using V = typename VecT<T, VX>::type;
    const int c = blockIdx.y;
    const T *src = c == 0 ? f0 : c == 1 ? f1 : c == 2 ? f2 : c == 3 ? f3 : c == 4 ? f4 : f5;
    const V *__restrict__ s = reinterpret_cast<const V *>(src);
    V *__restrict__ d = reinterpret_cast<V *>(dst + c * len);
    const long long nv = len / VX;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nv; e += (long long)gridDim.x * blockDim.x)
        d[e] = __ldcs(s + e);
}

// grad_out[cell] = sum over shots of grad[shot][cell], zero outside the frame
// [ncpml, n-ncpml) on every axis (satan_i calc_gamma, fwi3d_cpu_function_v1.4.c:2359-2361).
__global__ void grad_reduce_kernel(const double *__restrict__ g, int nshot, long long fshot, int nx, int ny, int nz,
                                   int px, long long plane, int ncpml, double *__restrict__ out) {
    const long long n = (long long)nx * ny * nz;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % nx);
        const int j = (int)((e / nx) % ny);
        const int k = (int)(e / ((long long)nx * ny));
        double s = 0.0;
        if (i >= ncpml && i < nx - ncpml && j >= ncpml && j < ny - ncpml && k >= ncpml && k < nz - ncpml) {
            const long long c = (long long)k * plane + (long long)j * px + i;
            for (int q = 0; q < nshot; q++) s += g[(long long)q * fshot + c];
        }
        out[e] = s;
    }
}

// residual R = S - obs and misfit 0.5 sum |R|^2 (one block reduction per launch, atomically added)
__global__ void residual_kernel(const double2 *__restrict__ S, const double2 *__restrict__ obs, long long n,
                                double2 *__restrict__ R, double *misfit) {
    double acc = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const double2 r = make_double2(S[e].x - obs[e].x, S[e].y - obs[e].y);
        R[e] = r;
        acc += 0.5 * (r.x * r.x + r.y * r.y);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(misfit, acc);
}

}  // namespace mittet
