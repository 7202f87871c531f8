// setup_host.h -- host-side set-up of one solve: CPML profiles, index ranges,
// reference time step.  Plain C++; shared by the CUDA library.
//
// Profiles restate init_cpml of the two reference flavours:
//   NCVER0027  ncver0027/cpu_cpml4.f90:20-240 (1-based, far side mirrored)
//   SATAN_I    satan_i/fwi3d_cpu_cpmlabc_v1.4.c:30-172 (0-based, x axis x optToMax,
//              float literals Rcoef=0.01f, aex_max=0.2f promoted to double)
// Ranges restate the loop bounds of
//   NCVER0027  e_field_cpml4/h_field_cpml4 (cpu_eh_field_cpml42.f90:127-151,222-246),
//              CPML_E4/CPML_H4 (cpu_cpml4.f90:281-359, 394-472)
//   SATAN_I    e/h_field_cpml42 (fwi3d_cpu_function_v1.4.c:1196-1281),
//              xe..zh_pml4 (fwi3d_cpu_cpmlabc_v1.4.c:402-679)
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace mittet {

struct Box {
    int lo[3], hi[3];
};

// A CPML slab group along one axis: a near interval [nlo,nhi) and a far
// interval [flo,fhi) on that axis, restricted to the `other` box on the two
// remaining axes.  Its psi are stored with `width` entries along the axis:
// the near cells at 0.., the far cells at fofs...  Along y and z (psi rows
// of px cells) the two intervals are packed (fofs = near cells); along x,
// where a psi row is only the slab cells of one grid row, each interval gets
// its own 32-byte-aligned half (fofs = width / 2, a multiple of 8 entries),
// so the near and far sides, computed by different CTAs, never share a DRAM
// sector.
struct Slab {
    int nlo, nhi, flo, fhi, width, fofs;
    Box other;
};

// Per-axis profile arrays used by the kernels.
enum ProfIdx { P_ESH = 0, P_MSH, P_BE, P_CED, P_BH, P_CHD, P_IKED, P_IKHD, P_COUNT };

struct Setup {
    int nx, ny, nz, nmax;
    Box upd[6];
    Slab se[3], sh[3];
    // [3 axes][P_COUNT][nmax]: esig/2, msig/2, be, ce/d, bh, ch/d, 1/ked, 1/khd
    std::vector<double> prof;
};

inline double prof_at(const Setup &s, int axis, int which, int i) {
    return s.prof[((size_t)axis * P_COUNT + which) * s.nmax + i];
}

struct CpmlConst {
    double nn, order, kappa_max, a_max, ma, rcoef, opt_to_max_x;
};

inline void profile_axis(int flavor, int n, double d, int ncpml, double cmax, double dt, bool is_x,
                         const CpmlConst &cc, double *esig, double *msig, double *be, double *ce,
                         double *bh, double *ch, double *ked, double *khd) {
    for (int i = 0; i < n; i++) {
        esig[i] = msig[i] = be[i] = ce[i] = bh[i] = ch[i] = 0.0;
        ked[i] = d;
        khd[i] = d;
    }
    const int nc = ncpml;
    if (flavor == 0) {
        const double delta = nc * d;
        const double sig_max = (cc.nn + cc.order + 1.0) * cmax * std::log(1.0 / cc.rcoef) / (2.0 * delta) *
                               (is_x ? cc.opt_to_max_x : 1.0);
        for (int ii = 1; ii <= nc; ii++) {
            const double q = ((double)nc - (double)ii) / ((double)nc - 1.0);
            const double qh = ((double)nc - (double)ii - 0.5) / ((double)nc - 1.0);
            const double es = sig_max * std::pow(q, cc.nn + cc.order);
            const double ms = sig_max * std::pow(qh, cc.nn + cc.order);  // negative at ii = ncpml
            const double ek = 1.0 + (cc.kappa_max - 1.0) * std::pow(q, cc.nn);
            const double mk = 1.0 + (cc.kappa_max - 1.0) * std::pow(qh, cc.nn);
            const double ae = cc.a_max * std::pow((double)ii / ((double)nc - 1.0), cc.ma);
            const double am = cc.a_max * std::pow(((double)ii + 0.5) / ((double)nc - 1.0), cc.ma);
            const double b_e = std::exp(-(es / ek + ae) * dt);
            const double b_h = std::exp(-(ms / mk + am) * dt);
            const double c_e = es * (b_e - 1.0) / (es + ek * ae) / ek;
            const double c_h = ms * (b_h - 1.0) / (ms + mk * am) / mk;
            const int a = ii - 1, b = n - ii;
            esig[a] = esig[b] = es;
            msig[a] = msig[b] = ms;
            be[a] = be[b] = b_e;
            bh[a] = bh[b] = b_h;
            ce[a] = ce[b] = c_e;
            ch[a] = ch[b] = c_h;
            ked[a] = ked[b] = ek * d;
            khd[a] = khd[b] = mk * d;
        }
    } else {
        const double Rcoef = (double)0.01f, nn = 3.0, order = 0.0, ma = 1.0, kappa_max = 1.0;
        const double aex_max = (double)0.2f;
        const double delta = nc * d;
        double esig_max = (nn + order + 1.0) * cmax * std::log(1.0 / Rcoef) / (2.0 * delta);
        if (is_x) esig_max = esig_max * 10.0;
        for (int i = 0; i < n; i++) {
            double es, ms, ek, mk, ae, am;
            if (i < nc) {
                es = esig_max * std::pow((double)(nc - i) / (double)(nc - 1.f), nn + order);
                ms = esig_max * std::pow((double)(nc - i - 0.5f) / (double)(nc - 1.f), nn + order);
                ek = 1.0 + (kappa_max - 1.0) * std::pow((double)(nc - i) / (double)(nc - 1.f), nn);
                mk = 1.0 + (kappa_max - 1.0) * std::pow((double)(nc - i - 0.5f) / (double)(nc - 1.f), nn);
                ae = aex_max * std::pow((double)i / (double)(nc - 1.f), ma);
                am = aex_max * std::pow((double)(i + 0.5f) / (double)(nc - 1.f), ma);
            } else if (i > n - nc - 1) {
                es = esig_max * std::pow((double)(i - n + 1.f + nc) / (double)(nc - 1.f), nn + order);
                ms = esig_max * std::pow((double)(i - n + 0.5f + nc) / (double)(nc - 1.f), nn + order);
                ek = 1.0 + (kappa_max - 1.0) * std::pow((double)(i - n + 1.0f + nc) / (double)(nc - 1.f), nn);
                mk = 1.0 + (kappa_max - 1.0) * std::pow((double)(i - n + 0.5f + nc) / (double)(nc - 1.f), nn);
                ae = aex_max * std::pow((double)(-i + n - 1.0f) / (double)(nc - 1.f), ma);
                am = aex_max * std::pow((double)(-i + n - 0.5f) / (double)(nc - 1.f), ma);
            } else {
                continue;
            }
            const double b_e = std::exp(-(es / ek + ae) * dt);
            const double b_h = std::exp(-(ms / mk + am) * dt);
            esig[i] = es;
            msig[i] = ms;
            be[i] = b_e;
            bh[i] = b_h;
            ce[i] = es * (b_e - 1.0) / (es + ek * ae) / ek;
            ch[i] = ms * (b_h - 1.0) / (ms + mk * am) / mk;
            ked[i] = ek * d;
            khd[i] = mk * d;
        }
    }
}

inline Box box(int x0, int y0, int z0, int x1, int y1, int z1) {
    Box b;
    b.lo[0] = x0; b.lo[1] = y0; b.lo[2] = z0;
    b.hi[0] = x1; b.hi[1] = y1; b.hi[2] = z1;
    return b;
}

inline void make_ranges(int flavor, int nx, int ny, int nz, int nc, Setup &s) {
    const int n3[3] = {nx, ny, nz};
    if (flavor == 0) {
        s.upd[0] = box(0, 2, 2, nx, ny - 1, nz - 1);
        s.upd[1] = box(2, 0, 2, nx - 1, ny, nz - 1);
        s.upd[2] = box(2, 2, 0, nx - 1, ny - 1, nz);
        s.upd[3] = box(0, 1, 1, nx, ny - 2, nz - 2);
        s.upd[4] = box(1, 0, 1, nx - 2, ny, nz - 2);
        s.upd[5] = box(1, 1, 0, nx - 2, ny - 2, nz);
        for (int a = 0; a < 3; a++) {
            s.se[a] = Slab{2, nc + 1, n3[a] - nc, n3[a] - 1, 0, 0, box(0, 0, 0, nx, ny, nz)};
            s.sh[a] = Slab{1, nc, n3[a] - nc - 1, n3[a] - 2, 0, 0, box(0, 0, 0, nx, ny, nz)};
        }
    } else {
        s.upd[0] = box(1, 2, 2, nx - 1, ny - 1, nz - 1);
        s.upd[1] = box(2, 1, 2, nx - 1, ny - 1, nz - 1);
        s.upd[2] = box(2, 2, 1, nx - 1, ny - 1, nz - 1);
        s.upd[3] = box(1, 1, 1, nx - 1, ny - 2, nz - 2);
        s.upd[4] = box(1, 1, 1, nx - 2, ny - 1, nz - 2);
        s.upd[5] = box(1, 1, 1, nx - 2, ny - 2, nz - 1);
        const Box oth = box(0, 0, 0, nx - 1, ny - 1, nz - 1);
        s.se[0] = Slab{2, nc - 1, nx - nc + 1, nx - 2, 0, 0, oth};
        s.se[1] = Slab{2, nc, ny - nc + 1, ny - 2, 0, 0, oth};
        s.se[2] = Slab{2, nc, nz - nc + 1, nz - 2, 0, 0, oth};
        s.sh[0] = Slab{1, nc - 1, nx - nc, nx - 2, 0, 0, oth};
        s.sh[1] = Slab{1, nc - 1, ny - nc, ny - 2, 0, 0, oth};
        s.sh[2] = Slab{1, nc - 1, nz - nc, nz - 2, 0, 0, oth};
    }
    for (int a = 0; a < 3; a++) {
        Slab *g[2] = {&s.se[a], &s.sh[a]};
        for (Slab *q : g) {
            if (q->nhi < q->nlo) q->nhi = q->nlo;
            if (q->fhi < q->flo) q->fhi = q->flo;
            const int near = q->nhi - q->nlo, far = q->fhi - q->flo;
            if (a == 0) {
                const int half = (std::max(near, far) + 7) / 8 * 8;
                q->fofs = half;
                q->width = 2 * half;
            } else {
                q->fofs = near;
                q->width = near + far;
            }
        }
    }
}

// Every stencil read of every range must stay inside the grid.  E reads
// offsets -2..+1 along its derivative axes, H reads -1..+2.  Returns false if
// a range would read outside (the grid is then too small for the flavour).
inline bool ranges_in_bounds(const Setup &s) {
    const int n3[3] = {s.nx, s.ny, s.nz};
    // derivative axes per component: Ex(y,z) Ey(z,x) Ez(x,y) and likewise for H
    const int dax[6][2] = {{1, 2}, {2, 0}, {0, 1}, {1, 2}, {2, 0}, {0, 1}};
    for (int c = 0; c < 6; c++) {
        const Box &b = s.upd[c];
        for (int a = 0; a < 3; a++)
            if (b.lo[a] < 0 || b.hi[a] > n3[a]) return false;
        bool empty = false;
        for (int a = 0; a < 3; a++) empty |= b.hi[a] <= b.lo[a];
        if (empty) continue;
        for (int q = 0; q < 2; q++) {
            const int a = dax[c][q];
            const int lo_off = c < 3 ? -2 : -1, hi_off = c < 3 ? 1 : 2;
            if (b.lo[a] + lo_off < 0 || b.hi[a] - 1 + hi_off > n3[a] - 1) return false;
        }
    }
    for (int a = 0; a < 3; a++) {
        const Slab *g[2] = {&s.se[a], &s.sh[a]};
        for (int t = 0; t < 2; t++) {
            const Slab *q = g[t];
            const int lo_off = t == 0 ? -2 : -1, hi_off = t == 0 ? 1 : 2;
            if (q->nhi > q->nlo && (q->nlo + lo_off < 0 || q->nhi - 1 + hi_off > n3[a] - 1)) return false;
            if (q->fhi > q->flo && (q->flo + lo_off < 0 || q->fhi - 1 + hi_off > n3[a] - 1)) return false;
            if (q->nhi > q->flo && q->fhi > q->flo && q->nhi > q->nlo) return false;  // overlapping slabs
            for (int b = 0; b < 3; b++)
                if (q->other.lo[b] < 0 || q->other.hi[b] > n3[b]) return false;
        }
    }
    return true;
}

inline void build_setup(int flavor, int nx, int ny, int nz, double dx, double dy, double dz, int ncpml,
                        double cmax, double dt, const CpmlConst &cc, Setup &s) {
    s.nx = nx; s.ny = ny; s.nz = nz;
    // profile row stride, a multiple of 4 so x profiles load as aligned vectors
    s.nmax = (std::max(nx, std::max(ny, nz)) + 3) / 4 * 4;
    s.prof.assign((size_t)3 * P_COUNT * s.nmax, 0.0);
    const int n3[3] = {nx, ny, nz};
    const double d3[3] = {dx, dy, dz};
    std::vector<double> es, ms, be, ce, bh, ch, ked, khd;
    for (int a = 0; a < 3; a++) {
        const int n = n3[a];
        es.assign(n, 0); ms.assign(n, 0); be.assign(n, 0); ce.assign(n, 0);
        bh.assign(n, 0); ch.assign(n, 0); ked.assign(n, 0); khd.assign(n, 0);
        profile_axis(flavor, n, d3[a], ncpml, cmax, dt, a == 0, cc, es.data(), ms.data(), be.data(),
                     ce.data(), bh.data(), ch.data(), ked.data(), khd.data());
        for (int i = 0; i < n; i++) {
            double *p = &s.prof[(size_t)a * P_COUNT * s.nmax];
            p[P_ESH * s.nmax + i] = es[i] * 0.5;
            p[P_MSH * s.nmax + i] = ms[i] * 0.5;
            p[P_BE * s.nmax + i] = be[i];
            p[P_CED * s.nmax + i] = ce[i] / d3[a];
            p[P_BH * s.nmax + i] = bh[i];
            p[P_CHD * s.nmax + i] = ch[i] / d3[a];
            p[P_IKED * s.nmax + i] = 1.0 / ked[i];
            p[P_IKHD * s.nmax + i] = 1.0 / khd[i];
        }
    }
    make_ranges(flavor, nx, ny, nz, ncpml, s);
}

}  // namespace mittet
