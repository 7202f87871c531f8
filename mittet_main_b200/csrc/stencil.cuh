// stencil.cuh -- the two half-step kernels of the (2,4) Yee + CPML update.
//
// Thread mapping: a BX x BY block covers an (x, y) tile; each thread owns KZ
// consecutive cells of one (i, j) column.  All reads of a thread are issued
// before its first store (every pointer is __restrict__, fields read in a
// phase are never written in it, reads go through the read-only path), so a
// warp keeps ~20-30 independent loads in flight: the kernels are bandwidth
// kernels and live on memory-level parallelism.  The z-neighbours of the two
// fields differentiated along z are loaded once per thread (KZ+3 planes) and
// reused from registers.
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

template <typename T, int BX, int BY, int KZ>
__global__ void __launch_bounds__(BX *BY, ((KZ == 1 && sizeof(T) == 4) ? 1024 / (BX * BY) : 512 / (BX * BY)))
    e_phase_kernel(const PhaseArgs<T> a) {
    const int i = blockIdx.x * BX + threadIdx.x;
    const int j = blockIdx.y * BY + threadIdx.y;
    const int nzc = (a.nz + KZ - 1) / KZ;
    const int shot = blockIdx.z / nzc;
    const int kb = (blockIdx.z - shot * nzc) * KZ;
    if (i >= a.nx || j >= a.ny) return;

    const long long sb = (long long)shot * a.fshot;
    T *__restrict__ Ex = a.f[0] + sb;
    T *__restrict__ Ey = a.f[1] + sb;
    T *__restrict__ Ez = a.f[2] + sb;
    const T *__restrict__ Hx = a.f[3] + sb;
    const T *__restrict__ Hy = a.f[4] + sb;
    const T *__restrict__ Hz = a.f[5] + sb;
    const T *__restrict__ M = a.m;
    const T *__restrict__ P = a.prof;
    const long long py = a.px, pz = a.plane;
    const int nz = a.nz, nmax = a.nmax;
    const T c1 = a.c1, c2 = a.c2;

    const T esh_x = __ldg(P + 0 * nmax + i), ik_x = __ldg(P + 6 * nmax + i);
    const T esh_y = __ldg(P + 8 * nmax + 0 * nmax + j), ik_y = __ldg(P + 8 * nmax + 6 * nmax + j);
    const bool vx = (i >= 2) && (i + 1 < a.nx);
    const bool vy = (j >= 2) && (j + 1 < a.ny);
    const int lx = slab_local(a.slab[0], i);
    const int ly = slab_local(a.slab[1], j);
    const bool sx_col = lx >= 0 && j >= a.slab[0].other.lo[1] && j < a.slab[0].other.hi[1];
    const bool sy_col = ly >= 0 && i >= a.slab[1].other.lo[0] && i < a.slab[1].other.hi[0];
    const bool sz_col = i >= a.slab[2].other.lo[0] && i < a.slab[2].other.hi[0] && j >= a.slab[2].other.lo[1] &&
                        j < a.slab[2].other.hi[1];
    const long long col = (long long)j * py + i;

    // z window: planes kb-2 .. kb+KZ of Hx and Hy
    T wx[KZ + 3], wy[KZ + 3];
#pragma unroll
    for (int q = 0; q < KZ + 3; q++) {
        const int kk = kb - 2 + q;
        const bool ok = kk >= 0 && kk < nz;
        wx[q] = ok ? __ldg(Hx + kk * pz + col) : T(0);
        wy[q] = ok ? __ldg(Hy + kk * pz + col) : T(0);
    }
    const int slot = a.ring_k > 0 ? (*a.d_step) % a.ring_k : 0;

#pragma unroll
    for (int q = 0; q < KZ; q++) {
        const int k = kb + q;
        if (k >= nz) break;
        const long long c = k * pz + col;
        const bool vz = (k >= 2) && (k + 1 < nz);
        const T hz = __ldg(Hz + c);
        T dyHz = T(0), dxHz = T(0), dxHy = T(0), dyHx = T(0), dzHy = T(0), dzHx = T(0);
        if (vy) {
            const T a0 = __ldg(Hz + c - py), a1 = __ldg(Hz + c + py), a2 = __ldg(Hz + c - 2 * py);
            const T b0 = __ldg(Hx + c - py), b1 = __ldg(Hx + c + py), b2 = __ldg(Hx + c - 2 * py);
            dyHz = c1 * (hz - a0) + c2 * (a1 - a2);
            dyHx = c1 * (wx[q + 2] - b0) + c2 * (b1 - b2);
        }
        if (vx) {
            const T a0 = __ldg(Hz + c - 1), a1 = __ldg(Hz + c + 1), a2 = __ldg(Hz + c - 2);
            const T b0 = __ldg(Hy + c - 1), b1 = __ldg(Hy + c + 1), b2 = __ldg(Hy + c - 2);
            dxHz = c1 * (hz - a0) + c2 * (a1 - a2);
            dxHy = c1 * (wy[q + 2] - b0) + c2 * (b1 - b2);
        }
        if (vz) {
            dzHy = c1 * (wy[q + 2] - wy[q + 1]) + c2 * (wy[q + 3] - wy[q]);
            dzHx = c1 * (wx[q + 2] - wx[q + 1]) + c2 * (wx[q + 3] - wx[q]);
        }
        const T m = __ldg(M + c);
        const T esh_z = __ldg(P + 16 * nmax + k), ik_z = __ldg(P + 16 * nmax + 6 * nmax + k);
        T ex = Ex[c], ey = Ey[c], ez = Ez[c];

        T ca_x = T(1), cb_x = m, ca_y = T(1), cb_y = m, ca_z = T(1), cb_z = m;
        if (esh_x != T(0)) { const T h = esh_x * m; const T r = rcp(T(1) + h); ca_x = (T(1) - h) * r; cb_x = m * r; }
        if (esh_y != T(0)) { const T h = esh_y * m; const T r = rcp(T(1) + h); ca_y = (T(1) - h) * r; cb_y = m * r; }
        if (esh_z != T(0)) { const T h = esh_z * m; const T r = rcp(T(1) + h); ca_z = (T(1) - h) * r; cb_z = m * r; }
        if (in_box(a.upd[0], i, j, k)) ex = ca_x * ex + a.sgn * cb_x * (dyHz * ik_y - dzHy * ik_z);
        if (in_box(a.upd[1], i, j, k)) ey = ca_y * ey + a.sgn * cb_y * (dzHx * ik_z - dxHz * ik_x);
        if (in_box(a.upd[2], i, j, k)) ez = ca_z * ez + a.sgn * cb_z * (dxHy * ik_x - dyHx * ik_y);

        if (sx_col && k >= a.slab[0].other.lo[2] && k < a.slab[0].other.hi[2]) {
            T *__restrict__ q0 = a.psi[0][0];
            T *__restrict__ q1 = a.psi[0][1];
            const long long o = (long long)shot * a.pshot[0] + ((long long)k * a.ny + j) * a.slab[0].width + lx;
            const T be = __ldg(P + 2 * nmax + i), ced = __ldg(P + 3 * nmax + i);
            const T p0 = be * q0[o] + ced * dxHy;  // psi_Ezx
            const T p1 = be * q1[o] + ced * dxHz;  // psi_Eyx
            q0[o] = p0;
            q1[o] = p1;
            ez = ez + cb_z * p0;
            ey = ey - cb_y * p1;
        }
        if (sy_col && k >= a.slab[1].other.lo[2] && k < a.slab[1].other.hi[2]) {
            T *__restrict__ q0 = a.psi[1][0];
            T *__restrict__ q1 = a.psi[1][1];
            const long long o = (long long)shot * a.pshot[1] + ((long long)k * a.slab[1].width + ly) * a.px + i;
            const T be = __ldg(P + 8 * nmax + 2 * nmax + j), ced = __ldg(P + 8 * nmax + 3 * nmax + j);
            const T p0 = be * q0[o] + ced * dyHz;  // psi_Exy
            const T p1 = be * q1[o] + ced * dyHx;  // psi_Ezy
            q0[o] = p0;
            q1[o] = p1;
            ex = ex + cb_x * p0;
            ez = ez - cb_z * p1;
        }
        if (sz_col) {
            const int lz = slab_local(a.slab[2], k);
            if (lz >= 0) {
                T *__restrict__ q0 = a.psi[2][0];
                T *__restrict__ q1 = a.psi[2][1];
                const long long o = (long long)shot * a.pshot[2] + ((long long)lz * a.ny + j) * a.px + i;
                const T be = __ldg(P + 16 * nmax + 2 * nmax + k), ced = __ldg(P + 16 * nmax + 3 * nmax + k);
                const T p0 = be * q0[o] + ced * dzHx;  // psi_Eyz
                const T p1 = be * q1[o] + ced * dzHy;  // psi_Exz
                q0[o] = p0;
                q1[o] = p1;
                ey = ey + cb_y * p0;
                ex = ex - cb_x * p1;
            }
        }
        Ex[c] = ex;
        Ey[c] = ey;
        Ez[c] = ez;
        if (a.ring_k > 0) {
            T *__restrict__ r = a.ring + (long long)slot * 3 * a.ring_comp + sb + c;
            if (a.vmask & 1) r[0] = ex;
            if (a.vmask & 2) r[a.ring_comp] = ey;
            if (a.vmask & 4) r[2 * a.ring_comp] = ez;
        }
    }
}

template <typename T, int BX, int BY, int KZ>
__global__ void __launch_bounds__(BX *BY, ((KZ == 1 && sizeof(T) == 4) ? 1024 / (BX * BY) : 512 / (BX * BY)))
    h_phase_kernel(const PhaseArgs<T> a) {
    const int i = blockIdx.x * BX + threadIdx.x;
    const int j = blockIdx.y * BY + threadIdx.y;
    const int nzc = (a.nz + KZ - 1) / KZ;
    const int shot = blockIdx.z / nzc;
    const int kb = (blockIdx.z - shot * nzc) * KZ;
    if (i >= a.nx || j >= a.ny) return;

    const long long sb = (long long)shot * a.fshot;
    const T *__restrict__ Ex = a.f[0] + sb;
    const T *__restrict__ Ey = a.f[1] + sb;
    const T *__restrict__ Ez = a.f[2] + sb;
    T *__restrict__ Hx = a.f[3] + sb;
    T *__restrict__ Hy = a.f[4] + sb;
    T *__restrict__ Hz = a.f[5] + sb;
    const T *__restrict__ M = a.m;
    const T *__restrict__ DM = a.dtmu;
    const T *__restrict__ P = a.prof;
    const long long py = a.px, pz = a.plane;
    const int nz = a.nz, nmax = a.nmax;
    const T c1 = a.c1, c2 = a.c2, c2t = a.c2t;

    const T msh_x = __ldg(P + 1 * nmax + i), ik_x = __ldg(P + 7 * nmax + i);
    const T msh_y = __ldg(P + 8 * nmax + 1 * nmax + j), ik_y = __ldg(P + 8 * nmax + 7 * nmax + j);
    const bool vx = (i >= 1) && (i + 2 < a.nx);
    const bool vy = (j >= 1) && (j + 2 < a.ny);
    const int lx = slab_local(a.slab[0], i);
    const int ly = slab_local(a.slab[1], j);
    const bool sx_col = lx >= 0 && j >= a.slab[0].other.lo[1] && j < a.slab[0].other.hi[1];
    const bool sy_col = ly >= 0 && i >= a.slab[1].other.lo[0] && i < a.slab[1].other.hi[0];
    const bool sz_col = i >= a.slab[2].other.lo[0] && i < a.slab[2].other.hi[0] && j >= a.slab[2].other.lo[1] &&
                        j < a.slab[2].other.hi[1];
    const long long col = (long long)j * py + i;

    // z window: planes kb-1 .. kb+KZ+1 of Ex and Ey
    T wx[KZ + 3], wy[KZ + 3];
#pragma unroll
    for (int q = 0; q < KZ + 3; q++) {
        const int kk = kb - 1 + q;
        const bool ok = kk >= 0 && kk < nz;
        wx[q] = ok ? __ldg(Ex + kk * pz + col) : T(0);
        wy[q] = ok ? __ldg(Ey + kk * pz + col) : T(0);
    }

#pragma unroll
    for (int q = 0; q < KZ; q++) {
        const int k = kb + q;
        if (k >= nz) break;
        const long long c = k * pz + col;
        const bool vz = (k >= 1) && (k + 2 < nz);
        const T ez = __ldg(Ez + c);
        T dyEz = T(0), dyEx = T(0), dxEz = T(0), dxEy = T(0), dzEy = T(0), dzEx = T(0), dxEzt = T(0);
        if (vy) {
            const T a0 = __ldg(Ez + c + py), a1 = __ldg(Ez + c + 2 * py), a2 = __ldg(Ez + c - py);
            const T b0 = __ldg(Ex + c + py), b1 = __ldg(Ex + c + 2 * py), b2 = __ldg(Ex + c - py);
            dyEz = c1 * (a0 - ez) + c2 * (a1 - a2);
            dyEx = c1 * (b0 - wx[q + 1]) + c2 * (b1 - b2);
        }
        if (vx) {
            const T a0 = __ldg(Ez + c + 1), a1 = __ldg(Ez + c + 2), a2 = __ldg(Ez + c - 1);
            const T b0 = __ldg(Ey + c + 1), b1 = __ldg(Ey + c + 2), b2 = __ldg(Ey + c - 1);
            dxEz = c1 * (a0 - ez) + c2 * (a1 - a2);
            dxEzt = c1 * a0 - c2t * ez + c2 * a1 - c2 * a2;  // psi_Hyx stencil, cpu_cpml4.f90:400
            dxEy = c1 * (b0 - wy[q + 1]) + c2 * (b1 - b2);
        }
        if (vz) {
            dzEy = c1 * (wy[q + 2] - wy[q + 1]) + c2 * (wy[q + 3] - wy[q]);
            dzEx = c1 * (wx[q + 2] - wx[q + 1]) + c2 * (wx[q + 3] - wx[q]);
        }
        const T m = __ldg(M + c);
        const T dm = DM ? __ldg(DM + c) : a.dtmu0;
        const T msh_z = __ldg(P + 16 * nmax + 1 * nmax + k), ik_z = __ldg(P + 16 * nmax + 7 * nmax + k);
        T hx = Hx[c], hy = Hy[c], hz = Hz[c];

        T da_x = T(1), db_x = dm, da_y = T(1), db_y = dm, da_z = T(1), db_z = dm;
        if (msh_x != T(0)) { const T h = msh_x * m; const T r = rcp(T(1) + h); da_x = (T(1) - h) * r; db_x = dm * r; }
        if (msh_y != T(0)) { const T h = msh_y * m; const T r = rcp(T(1) + h); da_y = (T(1) - h) * r; db_y = dm * r; }
        if (msh_z != T(0)) { const T h = msh_z * m; const T r = rcp(T(1) + h); da_z = (T(1) - h) * r; db_z = dm * r; }
        if (in_box(a.upd[0], i, j, k)) hx = da_x * hx - a.sgn * db_x * (dyEz * ik_y - dzEy * ik_z);
        if (in_box(a.upd[1], i, j, k)) hy = da_y * hy - a.sgn * db_y * (dzEx * ik_z - dxEz * ik_x);
        if (in_box(a.upd[2], i, j, k)) hz = da_z * hz - a.sgn * db_z * (dxEy * ik_x - dyEx * ik_y);

        if (sx_col && k >= a.slab[0].other.lo[2] && k < a.slab[0].other.hi[2]) {
            T *__restrict__ q0 = a.psi[0][0];
            T *__restrict__ q1 = a.psi[0][1];
            const long long o = (long long)shot * a.pshot[0] + ((long long)k * a.ny + j) * a.slab[0].width + lx;
            const T bh = __ldg(P + 4 * nmax + i), chd = __ldg(P + 5 * nmax + i);
            const T p0 = bh * q0[o] + chd * dxEy;   // psi_Hzx
            const T p1 = bh * q1[o] + chd * dxEzt;  // psi_Hyx
            q0[o] = p0;
            q1[o] = p1;
            hz = hz - db_z * p0;
            hy = hy + db_y * p1;
        }
        if (sy_col && k >= a.slab[1].other.lo[2] && k < a.slab[1].other.hi[2]) {
            T *__restrict__ q0 = a.psi[1][0];
            T *__restrict__ q1 = a.psi[1][1];
            const long long o = (long long)shot * a.pshot[1] + ((long long)k * a.slab[1].width + ly) * a.px + i;
            const T bh = __ldg(P + 8 * nmax + 4 * nmax + j), chd = __ldg(P + 8 * nmax + 5 * nmax + j);
            const T p0 = bh * q0[o] + chd * dyEz;  // psi_Hxy
            const T p1 = bh * q1[o] + chd * dyEx;  // psi_Hzy
            q0[o] = p0;
            q1[o] = p1;
            hx = hx - db_x * p0;
            hz = hz + db_z * p1;
        }
        if (sz_col) {
            const int lz = slab_local(a.slab[2], k);
            if (lz >= 0) {
                T *__restrict__ q0 = a.psi[2][0];
                T *__restrict__ q1 = a.psi[2][1];
                const long long o = (long long)shot * a.pshot[2] + ((long long)lz * a.ny + j) * a.px + i;
                const T bh = __ldg(P + 16 * nmax + 4 * nmax + k), chd = __ldg(P + 16 * nmax + 5 * nmax + k);
                const T p0 = bh * q0[o] + chd * dzEx;  // psi_Hyz
                const T p1 = bh * q1[o] + chd * dzEy;  // psi_Hxz
                q0[o] = p0;
                q1[o] = p1;
                hy = hy - db_y * p0;
                hx = hx + db_x * p1;
            }
        }
        Hx[c] = hx;
        Hy[c] = hy;
        Hz[c] = hz;
    }
}

// Tile/depth variants the autotuner chooses from (BX, BY, KZ).
#define MITTET_STENCIL_VARIANTS(X) \
    X(32, 4, 1)                    \
    X(32, 8, 1)                    \
    X(64, 4, 1)                    \
    X(32, 16, 1)                   \
    X(32, 4, 2)                    \
    X(32, 8, 2)                    \
    X(64, 2, 2)                    \
    X(32, 4, 4)                    \
    X(32, 8, 4)

}  // namespace mittet
