/*
 * mittet_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 CPU restatement of the reference's Mittet fictitious-wave FDTD hot path.
 * It is the checker for the CUDA library: only tests/, the smoke check and the
 * CPU-baseline leg of bench.py load it.  Nothing in the product links it.
 *
 * Two flavours of the reference exist and both are restated here:
 *
 *  NCVER0027 (Fortran, canonical forward driver)
 *    constants      ncver0027/cpu_parameter_wafe.f90:24-132
 *    CPML profiles  ncver0027/cpu_cpml4.f90:8-248 (init_cpml), mirrored far side
 *    coefficients   ncver0027/cpu_eh_field_cpml42.f90:8-57 (media_coeff)
 *    E update       ncver0027/cpu_eh_field_cpml42.f90:114-158 (e_field_cpml4)
 *    H update       ncver0027/cpu_eh_field_cpml42.f90:210-253 (h_field_cpml4)
 *    sign-flipped   ncver0027/cpu_eh_field_cpml42.f90:161-204,257-300 (*bp)
 *    psi_E          ncver0027/cpu_cpml4.f90:271-361 (CPML_E4)
 *    psi_H          ncver0027/cpu_cpml4.f90:384-474 (CPML_H4), incl. the
 *                   psi_Hyx stencil typo at :400 and :413 (switchable)
 *    source         ncver0027/cpu_waveform.f90:26,46-50 (magnetic, pre-E)
 *    step order     ncver0027/cpu_main.f90:99-141
 *    sampling       ncver0027/cpu_output.f90:20-55 (after the H half step)
 *
 *  SATAN_I (C, FWI code)
 *    CPML profiles  satan_i/fwi3d_cpu_cpmlabc_v1.4.c:7-175 (x axis x optToMax)
 *    coefficients   satan_i/fwi3d_cpu_function_v1.4.c:325-435 (media_coeff_3d)
 *    E/H update     satan_i/fwi3d_cpu_function_v1.4.c:1184-1290
 *    psi            satan_i/fwi3d_cpu_cpmlabc_v1.4.c:402-679
 *    source         satan_i/fwi3d_cpu_function_v1.4.c:514-529 (electric, post-E)
 *    step order     satan_i/fwi3d_cpu_function_v1.4.c:2528-2536 (fwdpropagation)
 *    sampling       satan_i/fwi3d_cpu_function_v1.4.c:765-780 (output)
 *
 * The DFT (f_to_d) restates ncver0027/cpu_f_to_d_e.f90:134-160 and
 * ncver0027/cpu_f_to_d_h.f90:134-167 (the H factor sqrt(-2 w0/(i w))).
 *
 * Parity pin: the SATAN_I flavour is checked bit for bit against the
 * reference's own C kernels compiled from their sources (oracle/ref_satan_driver.c);
 * the NCVER0027 flavour shares every loop body and differs only in the
 * constants, profile formulae and index ranges restated from the Fortran.
 *
 * All fields are real: the Fortran stores complex(8) but every input is real,
 * so the imaginary parts stay exactly zero.
 *
 * Index convention: 0-based, x fastest, c = (k*ny + j)*nx + i (the satan_i
 * layout and Fortran column-major order).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <complex.h>

enum { FLAVOR_NCVER0027 = 0, FLAVOR_SATAN_I = 1 };
enum { SRC_MAGNETIC = 0, SRC_ELECTRIC = 1 };
enum { C_EX = 0, C_EY, C_EZ, C_HX, C_HY, C_HZ };

typedef struct {
    int32_t nx, ny, nz, ncpml;
    int32_t flavor;          /* FLAVOR_* */
    int32_t psi_hyx_typo;    /* 1: reproduce cpu_cpml4.f90:400,413 */
    int32_t e_sign, h_sign;  /* +1 normal, -1 for the "bp" variants */
    double dx, dy, dz, dt, omega0, c1, c2;
    double cmax;             /* fastest fictitious velocity, for sig_max */
    double nn, order, kappa_max, a_max, ma, rcoef, opt_to_max_x;
} orc_params;

/* 1-D CPML profiles of one axis: esig, msig, be, ce, bh, ch, ked, khd */
typedef struct { double *esig, *msig, *be, *ce, *bh, *ch, *ked, *khd; } prof1d;

/* Index ranges, 0-based half-open. */
typedef struct { int lo[3], hi[3]; } box3;
typedef struct { int nlo, nhi, flo, fhi; box3 other; } slab;

static int inbox(const box3 *b, int i, int j, int k) {
    return i >= b->lo[0] && i < b->hi[0] && j >= b->lo[1] && j < b->hi[1] &&
           k >= b->lo[2] && k < b->hi[2];
}

/* ---------------------------------------------------------------- profiles */

/* ncver0027/cpu_cpml4.f90:20-91 for one axis of length n, spacing d.
 * Fortran index ii = i+1.  Near side ii=1..ncpml, far side mirrored
 * (ii' = n-(ii-1)), interior zero / kappa one.  Note msig at ii=ncpml is
 * sig_max*(-0.5/(ncpml-1))**3 < 0 (pow of a negative base, integer exponent). */
static void profile_ncver(const orc_params *p, int n, double d, int is_z, prof1d *o) {
    const double delta = p->ncpml * d;
    const double sig_max = (p->nn + p->order + 1.0) * p->cmax * log(1.0 / p->rcoef) / (2.0 * delta);
    const int nc = p->ncpml;
    for (int i = 0; i < n; i++) {
        o->esig[i] = 0.0; o->msig[i] = 0.0; o->be[i] = 0.0; o->bh[i] = 0.0;
        o->ce[i] = 0.0; o->ch[i] = 0.0; o->ked[i] = d; o->khd[i] = d;
    }
    for (int ii = 1; ii <= nc; ii++) {
        double esig = sig_max * pow(((double)nc - (double)ii) / ((double)nc - 1.0), p->nn + p->order);
        double msig = sig_max * pow(((double)nc - (double)ii - 0.5) / ((double)nc - 1.0), p->nn + p->order);
        double ek = 1.0 + (p->kappa_max - 1.0) * pow(((double)nc - (double)ii) / ((double)nc - 1.0), p->nn);
        double mk = 1.0 + (p->kappa_max - 1.0) * pow(((double)nc - (double)ii - 0.5) / ((double)nc - 1.0), p->nn);
        double ae = p->a_max * pow(((double)ii) / ((double)nc - 1.0), p->ma);
        double am = p->a_max * pow(((double)ii + 0.5) / ((double)nc - 1.0), p->ma);
        double be = exp(-(esig / ek + ae) * p->dt);
        double bh = exp(-(msig / mk + am) * p->dt);
        double ce = esig * (be - 1.0) / (esig + ek * ae) / ek;
        double ch = msig * (bh - 1.0) / (msig + mk * am) / mk;
        int a = ii - 1, b = n - ii; /* near, mirrored far (0-based) */
        o->esig[a] = o->esig[b] = esig; o->msig[a] = o->msig[b] = msig;
        o->be[a] = o->be[b] = be; o->bh[a] = o->bh[b] = bh;
        o->ce[a] = o->ce[b] = ce; o->ch[a] = o->ch[b] = ch;
        o->ked[a] = o->ked[b] = ek * d; o->khd[a] = o->khd[b] = mk * d;
    }
    (void)is_z; /* the stray khdz(ncpml+1) assignment at :224 is overwritten at :239 */
}

/* satan_i/fwi3d_cpu_cpmlabc_v1.4.c:7-175.  Float literals are kept as floats
 * (Rcoef=0.01f, aex_max=0.2f) and promoted exactly as the C code does. */
static void profile_satan(const orc_params *p, int n, double d, int is_x, prof1d *o) {
    const double Rcoef = 0.01f, nn = 3.f, order = 0.f, ma = 1.f, kappa_max = 1.f, aex_max = 0.2f;
    const double optToMax = 10.0;
    const int nc = p->ncpml;
    double delta = nc * d;
    double esig_max = (nn + order + 1.f) * p->cmax * log(1.f / Rcoef) / (2.f * delta);
    if (is_x) esig_max = esig_max * optToMax;
    for (int i = 0; i < n; i++) {
        double esig, msig, ek, mk, ae, am, be, bh, ce, ch;
        if (i < nc) {
            esig = esig_max * pow((double)(nc - i) / (double)(nc - 1.f), nn + order);
            msig = esig_max * pow((double)(nc - i - 0.5f) / (double)(nc - 1.f), nn + order);
            ek = 1.f + (kappa_max - 1.f) * pow((double)(nc - i) / (double)(nc - 1.f), nn);
            mk = 1.f + (kappa_max - 1.f) * pow((double)(nc - i - 0.5f) / (double)(nc - 1.f), nn);
            ae = aex_max * pow((double)(i) / (double)(nc - 1.f), ma);
            am = aex_max * pow((double)(i + 0.5f) / (double)(nc - 1.f), ma);
        } else if (i > (n - nc - 1)) {
            esig = esig_max * pow((double)(i - n + 1.f + nc) / (double)(nc - 1.f), nn + order);
            msig = esig_max * pow((double)(i - n + 0.5f + nc) / (double)(nc - 1.f), nn + order);
            ek = 1.f + (kappa_max - 1.f) * pow((double)(i - n + 1.0f + nc) / (double)(nc - 1.f), nn);
            mk = 1.f + (kappa_max - 1.f) * pow((double)(i - n + 0.5f + nc) / (double)(nc - 1.f), nn);
            ae = aex_max * pow((double)(-i + n - 1.0f) / (double)(nc - 1.f), ma);
            am = aex_max * pow((double)(-i + n - 0.5f) / (double)(nc - 1.f), ma);
        } else {
            o->esig[i] = o->msig[i] = 0.0; o->be[i] = o->ce[i] = 0.0; o->bh[i] = o->ch[i] = 0.0;
            o->ked[i] = 1.0 * d; o->khd[i] = 1.0 * d;
            continue;
        }
        be = exp(-(esig / ek + ae) * p->dt);
        bh = exp(-(msig / mk + am) * p->dt);
        ce = esig * (be - 1.f) / (esig + ek * ae) / ek;
        ch = msig * (bh - 1.f) / (msig + mk * am) / mk;
        o->esig[i] = esig; o->msig[i] = msig; o->be[i] = be; o->bh[i] = bh;
        o->ce[i] = ce; o->ch[i] = ch; o->ked[i] = ek * d; o->khd[i] = mk * d;
    }
}

/* ------------------------------------------------------------------ ranges */

static void ranges_ncver(int nx, int ny, int nz, int nc, box3 upd[6], slab se[3], slab sh[3]) {
    /* ncver0027/cpu_eh_field_cpml42.f90:127-151 and :222-246 */
    box3 ex = {{0, 2, 2}, {nx, ny - 1, nz - 1}};
    box3 ey = {{2, 0, 2}, {nx - 1, ny, nz - 1}};
    box3 ez = {{2, 2, 0}, {nx - 1, ny - 1, nz}};
    box3 hx = {{0, 1, 1}, {nx, ny - 2, nz - 2}};
    box3 hy = {{1, 0, 1}, {nx - 2, ny, nz - 2}};
    box3 hz = {{1, 1, 0}, {nx - 2, ny - 2, nz}};
    upd[0] = ex; upd[1] = ey; upd[2] = ez; upd[3] = hx; upd[4] = hy; upd[5] = hz;
    int n3[3] = {nx, ny, nz};
    for (int a = 0; a < 3; a++) {
        box3 all = {{0, 0, 0}, {nx, ny, nz}};
        /* CPML_E4 cpu_cpml4.f90:283,296: 3..ncpml+1 and n-ncpml+1..n-1 (1-based) */
        se[a].nlo = 2; se[a].nhi = nc + 1; se[a].flo = n3[a] - nc; se[a].fhi = n3[a] - 1; se[a].other = all;
        /* CPML_H4 cpu_cpml4.f90:396,409: 2..ncpml and n-ncpml..n-2 (1-based) */
        sh[a].nlo = 1; sh[a].nhi = nc; sh[a].flo = n3[a] - nc - 1; sh[a].fhi = n3[a] - 2; sh[a].other = all;
    }
}

static void ranges_satan(int ix, int iy, int iz, int nc, box3 upd[6], slab se[3], slab sh[3]) {
    /* satan_i/fwi3d_cpu_function_v1.4.c:1196-1281 */
    box3 ex = {{1, 2, 2}, {ix - 1, iy - 1, iz - 1}};
    box3 ey = {{2, 1, 2}, {ix - 1, iy - 1, iz - 1}};
    box3 ez = {{2, 2, 1}, {ix - 1, iy - 1, iz - 1}};
    box3 hx = {{1, 1, 1}, {ix - 1, iy - 2, iz - 2}};
    box3 hy = {{1, 1, 1}, {ix - 2, iy - 1, iz - 2}};
    box3 hz = {{1, 1, 1}, {ix - 2, iy - 2, iz - 1}};
    upd[0] = ex; upd[1] = ey; upd[2] = ez; upd[3] = hx; upd[4] = hy; upd[5] = hz;
    box3 oth = {{0, 0, 0}, {ix - 1, iy - 1, iz - 1}};
    /* satan_i/fwi3d_cpu_cpmlabc_v1.4.c:415,433 (x), 465,483 (y), 515,534 (z) */
    se[0].nlo = 2; se[0].nhi = nc - 1; se[0].flo = ix - nc + 1; se[0].fhi = ix - 2;
    se[1].nlo = 2; se[1].nhi = nc;     se[1].flo = iy - nc + 1; se[1].fhi = iy - 2;
    se[2].nlo = 2; se[2].nhi = nc;     se[2].flo = iz - nc + 1; se[2].fhi = iz - 2;
    /* :565,583 (x), 614,632 (y), 663,681 (z) */
    sh[0].nlo = 1; sh[0].nhi = nc - 1; sh[0].flo = ix - nc; sh[0].fhi = ix - 2;
    sh[1].nlo = 1; sh[1].nhi = nc - 1; sh[1].flo = iy - nc; sh[1].fhi = iy - 2;
    sh[2].nlo = 1; sh[2].nhi = nc - 1; sh[2].flo = iz - nc; sh[2].fhi = iz - 2;
    for (int a = 0; a < 3; a++) { se[a].other = oth; sh[a].other = oth; }
}

static int inslab(const slab *s, int axis, int i, int j, int k) {
    int v = axis == 0 ? i : (axis == 1 ? j : k);
    if (!((v >= s->nlo && v < s->nhi) || (v >= s->flo && v < s->fhi))) return 0;
    return inbox(&s->other, i, j, k);
}

/* Exported so tests can inspect the restated profiles and ranges. */
int orc_profiles(const orc_params *p, double *out /* [3][8][nmax] */, int nmax) {
    int n3[3] = {p->nx, p->ny, p->nz};
    double d3[3] = {p->dx, p->dy, p->dz};
    for (int a = 0; a < 3; a++) {
        if (n3[a] > nmax) return -1;
        double *b = out + (size_t)a * 8 * nmax;
        prof1d o = {b, b + nmax, b + 2 * nmax, b + 3 * nmax, b + 4 * nmax, b + 5 * nmax, b + 6 * nmax, b + 7 * nmax};
        if (p->flavor == FLAVOR_SATAN_I) profile_satan(p, n3[a], d3[a], a == 0, &o);
        else profile_ncver(p, n3[a], d3[a], a == 2, &o);
    }
    return 0;
}

int orc_ranges(const orc_params *p, int32_t *out /* 6*6 upd + 6*10 slabs */) {
    box3 upd[6]; slab se[3], sh[3];
    if (p->flavor == FLAVOR_SATAN_I) ranges_satan(p->nx, p->ny, p->nz, p->ncpml, upd, se, sh);
    else ranges_ncver(p->nx, p->ny, p->nz, p->ncpml, upd, se, sh);
    int w = 0;
    for (int c = 0; c < 6; c++) { for (int a = 0; a < 3; a++) out[w++] = upd[c].lo[a]; for (int a = 0; a < 3; a++) out[w++] = upd[c].hi[a]; }
    slab *all[6] = {&se[0], &se[1], &se[2], &sh[0], &sh[1], &sh[2]};
    for (int s = 0; s < 6; s++) {
        out[w++] = all[s]->nlo; out[w++] = all[s]->nhi; out[w++] = all[s]->flo; out[w++] = all[s]->fhi;
        for (int a = 0; a < 3; a++) out[w++] = all[s]->other.lo[a];
        for (int a = 0; a < 3; a++) out[w++] = all[s]->other.hi[a];
    }
    return 0;
}

/* ---------------------------------------------------------------- forward */

typedef struct {
    int nx, ny, nz; size_t n;
    double *f[6];       /* Ex Ey Ez Hx Hy Hz */
    double *psi[12];    /* E: zx yx | xy zy | yz xz ; H: yx zx | xy zy | yz xz */
    double *ca[3], *cb[3], *da[3], *db[3];
    prof1d pr[3];
    double *prbuf;
    box3 upd[6]; slab se[3], sh[3];
} orc_state;

#define IDX(i, j, k) (((size_t)(k) * ny + (j)) * nx + (i))

static int state_init(orc_state *s, const orc_params *p, const double *sigma, const double *mu) {
    int nx = p->nx, ny = p->ny, nz = p->nz;
    s->nx = nx; s->ny = ny; s->nz = nz; s->n = (size_t)nx * ny * nz;
    size_t n = s->n;
    for (int c = 0; c < 6; c++) { s->f[c] = calloc(n, sizeof(double)); if (!s->f[c]) return -1; }
    for (int c = 0; c < 12; c++) { s->psi[c] = calloc(n, sizeof(double)); if (!s->psi[c]) return -1; }
    for (int a = 0; a < 3; a++) {
        s->ca[a] = malloc(n * sizeof(double)); s->cb[a] = malloc(n * sizeof(double));
        s->da[a] = malloc(n * sizeof(double)); s->db[a] = malloc(n * sizeof(double));
        if (!s->ca[a] || !s->cb[a] || !s->da[a] || !s->db[a]) return -1;
    }
    int nmax = nx > ny ? nx : ny; nmax = nmax > nz ? nmax : nz;
    s->prbuf = malloc(sizeof(double) * 24 * nmax);
    orc_profiles(p, s->prbuf, nmax);
    for (int a = 0; a < 3; a++) {
        double *b = s->prbuf + (size_t)a * 8 * nmax;
        prof1d o = {b, b + nmax, b + 2 * nmax, b + 3 * nmax, b + 4 * nmax, b + 5 * nmax, b + 6 * nmax, b + 7 * nmax};
        s->pr[a] = o;
    }
    if (p->flavor == FLAVOR_SATAN_I) ranges_satan(nx, ny, nz, p->ncpml, s->upd, s->se, s->sh);
    else ranges_ncver(nx, ny, nz, p->ncpml, s->upd, s->se, s->sh);

    /* media_coeff: ncver0027/cpu_eh_field_cpml42.f90:26-56 and
     * satan_i/fwi3d_cpu_function_v1.4.c:336,412-426 (identical arithmetic
     * once the float literals 2.f, 1.0f are promoted). */
    const double dt = p->dt;
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                size_t c = IDX(i, j, k);
                double eps2 = sigma[c] / 2.0 / p->omega0;
                double es[3] = {s->pr[0].esig[i], s->pr[1].esig[j], s->pr[2].esig[k]};
                double ms[3] = {s->pr[0].msig[i], s->pr[1].msig[j], s->pr[2].msig[k]};
                for (int a = 0; a < 3; a++) {
                    s->ca[a][c] = (1.0 - ((es[a] * dt) / (2.0 * eps2))) / (1.0 + ((es[a] * dt) / (2.0 * eps2)));
                    s->cb[a][c] = dt / eps2 / (1.0 + (es[a] * dt) / (2.0 * eps2));
                    s->da[a][c] = (1.0 - ((ms[a] * dt) / (2.0 * eps2))) / (1.0 + ((ms[a] * dt) / (2.0 * eps2)));
                    s->db[a][c] = dt / mu[c] / (1.0 + (ms[a] * dt) / (2.0 * eps2));
                }
            }
    return 0;
}

static void state_free(orc_state *s) {
    for (int c = 0; c < 6; c++) free(s->f[c]);
    for (int c = 0; c < 12; c++) free(s->psi[c]);
    for (int a = 0; a < 3; a++) { free(s->ca[a]); free(s->cb[a]); free(s->da[a]); free(s->db[a]); }
    free(s->prbuf);
}

/* E half step: e_field_cpml4 then CPML_E4 (same loop bodies in both flavours). */
static void e_phase(orc_state *s, const orc_params *p) {
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const double c1 = p->c1, c2 = p->c2, sg = (double)p->e_sign;
    double *Ex = s->f[0], *Ey = s->f[1], *Ez = s->f[2];
    const double *Hx = s->f[3], *Hy = s->f[4], *Hz = s->f[5];
    const size_t sx = 1, sy = (size_t)nx, sz = (size_t)nx * ny;
    const double *kedx = s->pr[0].ked, *kedy = s->pr[1].ked, *kedz = s->pr[2].ked;
    box3 *u = s->upd;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                size_t c = IDX(i, j, k);
                if (inbox(&u[0], i, j, k))
                    Ex[c] = s->ca[0][c] * Ex[c] + sg * s->cb[0][c] *
                        ((c1 * Hz[c] - c1 * Hz[c - sy] + c2 * Hz[c + sy] - c2 * Hz[c - 2 * sy]) / kedy[j] -
                         (c1 * Hy[c] - c1 * Hy[c - sz] + c2 * Hy[c + sz] - c2 * Hy[c - 2 * sz]) / kedz[k]);
                if (inbox(&u[1], i, j, k))
                    Ey[c] = s->ca[1][c] * Ey[c] + sg * s->cb[1][c] *
                        ((c1 * Hx[c] - c1 * Hx[c - sz] + c2 * Hx[c + sz] - c2 * Hx[c - 2 * sz]) / kedz[k] -
                         (c1 * Hz[c] - c1 * Hz[c - sx] + c2 * Hz[c + sx] - c2 * Hz[c - 2 * sx]) / kedx[i]);
                if (inbox(&u[2], i, j, k))
                    Ez[c] = s->ca[2][c] * Ez[c] + sg * s->cb[2][c] *
                        ((c1 * Hy[c] - c1 * Hy[c - sx] + c2 * Hy[c + sx] - c2 * Hy[c - 2 * sx]) / kedx[i] -
                         (c1 * Hx[c] - c1 * Hx[c - sy] + c2 * Hx[c + sy] - c2 * Hx[c - 2 * sy]) / kedy[j]);
            }
    /* CPML_E4: x slabs, then y slabs, then z slabs (each updates two fields) */
    const double dx = p->dx, dy = p->dy, dz = p->dz;
    double *pEzx = s->psi[0], *pEyx = s->psi[1], *pExy = s->psi[2], *pEzy = s->psi[3], *pEyz = s->psi[4], *pExz = s->psi[5];
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                if (!inslab(&s->se[0], 0, i, j, k)) continue;
                size_t c = IDX(i, j, k);
                double be = s->pr[0].be[i], ce = s->pr[0].ce[i];
                pEzx[c] = be * pEzx[c] + ce * (c1 * Hy[c] - c1 * Hy[c - sx] + c2 * Hy[c + sx] - c2 * Hy[c - 2 * sx]) / dx;
                pEyx[c] = be * pEyx[c] + ce * (c1 * Hz[c] - c1 * Hz[c - sx] + c2 * Hz[c + sx] - c2 * Hz[c - 2 * sx]) / dx;
                Ez[c] = Ez[c] + s->cb[2][c] * pEzx[c];
                Ey[c] = Ey[c] - s->cb[1][c] * pEyx[c];
            }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                if (!inslab(&s->se[1], 1, i, j, k)) continue;
                size_t c = IDX(i, j, k);
                double be = s->pr[1].be[j], ce = s->pr[1].ce[j];
                pExy[c] = be * pExy[c] + ce * (c1 * Hz[c] - c1 * Hz[c - sy] + c2 * Hz[c + sy] - c2 * Hz[c - 2 * sy]) / dy;
                pEzy[c] = be * pEzy[c] + ce * (c1 * Hx[c] - c1 * Hx[c - sy] + c2 * Hx[c + sy] - c2 * Hx[c - 2 * sy]) / dy;
                Ex[c] = Ex[c] + s->cb[0][c] * pExy[c];
                Ez[c] = Ez[c] - s->cb[2][c] * pEzy[c];
            }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                if (!inslab(&s->se[2], 2, i, j, k)) continue;
                size_t c = IDX(i, j, k);
                double be = s->pr[2].be[k], ce = s->pr[2].ce[k];
                pEyz[c] = be * pEyz[c] + ce * (c1 * Hx[c] - c1 * Hx[c - sz] + c2 * Hx[c + sz] - c2 * Hx[c - 2 * sz]) / dz;
                pExz[c] = be * pExz[c] + ce * (c1 * Hy[c] - c1 * Hy[c - sz] + c2 * Hy[c + sz] - c2 * Hy[c - 2 * sz]) / dz;
                Ey[c] = Ey[c] + s->cb[1][c] * pEyz[c];
                Ex[c] = Ex[c] - s->cb[0][c] * pExz[c];
            }
}

/* H half step: h_field_cpml4 then CPML_H4. */
static void h_phase(orc_state *s, const orc_params *p) {
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const double c1 = p->c1, c2 = p->c2, sg = (double)p->h_sign;
    const double *Ex = s->f[0], *Ey = s->f[1], *Ez = s->f[2];
    double *Hx = s->f[3], *Hy = s->f[4], *Hz = s->f[5];
    const size_t sx = 1, sy = (size_t)nx, sz = (size_t)nx * ny;
    const double *khdx = s->pr[0].khd, *khdy = s->pr[1].khd, *khdz = s->pr[2].khd;
    box3 *u = s->upd;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                size_t c = IDX(i, j, k);
                if (inbox(&u[3], i, j, k))
                    Hx[c] = s->da[0][c] * Hx[c] - sg * s->db[0][c] *
                        ((c1 * Ez[c + sy] - c1 * Ez[c] + c2 * Ez[c + 2 * sy] - c2 * Ez[c - sy]) / khdy[j] -
                         (c1 * Ey[c + sz] - c1 * Ey[c] + c2 * Ey[c + 2 * sz] - c2 * Ey[c - sz]) / khdz[k]);
                if (inbox(&u[4], i, j, k))
                    Hy[c] = s->da[1][c] * Hy[c] - sg * s->db[1][c] *
                        ((c1 * Ex[c + sz] - c1 * Ex[c] + c2 * Ex[c + 2 * sz] - c2 * Ex[c - sz]) / khdz[k] -
                         (c1 * Ez[c + sx] - c1 * Ez[c] + c2 * Ez[c + 2 * sx] - c2 * Ez[c - sx]) / khdx[i]);
                if (inbox(&u[5], i, j, k))
                    Hz[c] = s->da[2][c] * Hz[c] - sg * s->db[2][c] *
                        ((c1 * Ey[c + sx] - c1 * Ey[c] + c2 * Ey[c + 2 * sx] - c2 * Ey[c - sx]) / khdx[i] -
                         (c1 * Ex[c + sy] - c1 * Ex[c] + c2 * Ex[c + 2 * sy] - c2 * Ex[c - sy]) / khdy[j]);
            }
    const double dx = p->dx, dy = p->dy, dz = p->dz;
    double *pHyx = s->psi[6], *pHzx = s->psi[7], *pHxy = s->psi[8], *pHzy = s->psi[9], *pHyz = s->psi[10], *pHxz = s->psi[11];
    const double c2t = p->psi_hyx_typo ? c2 : c1; /* cpu_cpml4.f90:400: c1*Ez(i+1)-c2*Ez(i) */
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                if (!inslab(&s->sh[0], 0, i, j, k)) continue;
                size_t c = IDX(i, j, k);
                double bh = s->pr[0].bh[i], ch = s->pr[0].ch[i];
                pHzx[c] = bh * pHzx[c] + ch * (c1 * Ey[c + sx] - c1 * Ey[c] + c2 * Ey[c + 2 * sx] - c2 * Ey[c - sx]) / dx;
                pHyx[c] = bh * pHyx[c] + ch * (c1 * Ez[c + sx] - c2t * Ez[c] + c2 * Ez[c + 2 * sx] - c2 * Ez[c - sx]) / dx;
                Hz[c] = Hz[c] - s->db[2][c] * pHzx[c];
                Hy[c] = Hy[c] + s->db[1][c] * pHyx[c];
            }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                if (!inslab(&s->sh[1], 1, i, j, k)) continue;
                size_t c = IDX(i, j, k);
                double bh = s->pr[1].bh[j], ch = s->pr[1].ch[j];
                pHxy[c] = bh * pHxy[c] + ch * (c1 * Ez[c + sy] - c1 * Ez[c] + c2 * Ez[c + 2 * sy] - c2 * Ez[c - sy]) / dy;
                pHzy[c] = bh * pHzy[c] + ch * (c1 * Ex[c + sy] - c1 * Ex[c] + c2 * Ex[c + 2 * sy] - c2 * Ex[c - sy]) / dy;
                Hx[c] = Hx[c] - s->db[0][c] * pHxy[c];
                Hz[c] = Hz[c] + s->db[2][c] * pHzy[c];
            }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                if (!inslab(&s->sh[2], 2, i, j, k)) continue;
                size_t c = IDX(i, j, k);
                double bh = s->pr[2].bh[k], ch = s->pr[2].ch[k];
                pHyz[c] = bh * pHyz[c] + ch * (c1 * Ex[c + sz] - c1 * Ex[c] + c2 * Ex[c + 2 * sz] - c2 * Ex[c - sz]) / dz;
                pHxz[c] = bh * pHxz[c] + ch * (c1 * Ey[c + sz] - c1 * Ey[c] + c2 * Ey[c + 2 * sz] - c2 * Ey[c - sz]) / dz;
                Hy[c] = Hy[c] - s->db[1][c] * pHyz[c];
                Hx[c] = Hx[c] + s->db[0][c] * pHxz[c];
            }
}

/*
 * Forward solve of one shot.
 *  src_cell: 0-based linear cell index; src_comp: C_*; src_kind: SRC_*;
 *  wavelet[n] = s(n*dt), n = 0..nt.
 *  Magnetic (ncver0027/cpu_waveform.f90:46-50), applied before the E step:
 *      F -= amp * wavelet[n+1] * dt / mu / (dx dy dz)
 *  Electric (satan_i/fwi3d_cpu_function_v1.4.c:526-527), after the E step:
 *      F -= amp * (wavelet[n] + wavelet[n+1]) / 2 * dt * 2 w0 / sigma / (dx dy dz)
 *  traces[r*nt + n] = field after step n (n = 0..nt-1).
 *  final_fields (nullable): 6*n doubles, the fields after the last step.
 */
int orc_forward(const orc_params *p, const double *sigma, const double *mu,
                int nsrc, const int64_t *src_cell, const int32_t *src_comp,
                const int32_t *src_kind, const double *src_amp,
                int nt, const double *wavelet,
                int nrec, const int64_t *rec_cell, const int32_t *rec_comp,
                double *traces, double *final_fields) {
    orc_state s;
    memset(&s, 0, sizeof(s));
    if (state_init(&s, p, sigma, mu)) { state_free(&s); return -1; }
    const double vol = p->dx * p->dy * p->dz;
    for (int n = 0; n < nt; n++) {
        for (int q = 0; q < nsrc; q++) {
            if (src_kind[q] != SRC_MAGNETIC) continue;
            int64_t c = src_cell[q];
            s.f[src_comp[q]][c] = s.f[src_comp[q]][c] - src_amp[q] * wavelet[n + 1] * p->dt / mu[c] / p->dx / p->dy / p->dz;
        }
        e_phase(&s, p);
        for (int q = 0; q < nsrc; q++) {
            if (src_kind[q] != SRC_ELECTRIC) continue;
            int64_t c = src_cell[q];
            s.f[src_comp[q]][c] -= src_amp[q] * (wavelet[n] + wavelet[n + 1]) / 2.f * p->dt * 2.f * p->omega0 / sigma[c] / p->dx / p->dy / p->dz;
        }
        (void)vol;
        h_phase(&s, p);
        for (int r = 0; r < nrec; r++) traces[(size_t)r * nt + n] = s.f[rec_comp[r]][rec_cell[r]];
    }
    if (final_fields)
        for (int c = 0; c < 6; c++) memcpy(final_fields + (size_t)c * s.n, s.f[c], s.n * sizeof(double));
    state_free(&s);
    return 0;
}

/*
 * f_to_d damped DFT, ncver0027/cpu_f_to_d_e.f90:140-148:
 *   X(w) = sum_{n=0}^{nt-1} x[n] * dt * exp((i-1) * sqrt(w0*w) * n*dt)
 * With h_factor, ncver0027/cpu_f_to_d_h.f90:146-148 multiplies every term by
 * sqrt(-2 w0/(i w)) (principal branch; w = 0 gives a non-finite value, as in
 * the reference's k = 0 row).
 * out is interleaved complex: out[2*f], out[2*f+1].
 */
void orc_dft(int nt, double dt, double omega0, const double *x, int nf, const double *omega,
             int h_factor, double *out) {
#pragma omp parallel for schedule(static)
    for (int f = 0; f < nf; f++) {
        double complex acc = 0.0;
        double complex hf = 1.0;
        if (h_factor) hf = csqrt(-2.0 * omega0 / I / omega[f]);
        double sw = sqrt(omega0 * omega[f]);
        for (int n = 0; n < nt; n++) {
            double complex term = x[n] * dt * cexp((I - 1.0) * sw * n * dt);
            acc = h_factor ? acc + hf * term : acc + term;
        }
        out[2 * f] = creal(acc);
        out[2 * f + 1] = cimag(acc);
    }
}

/* ======================================================================
 * Discrete adjoint gradient d(misfit)/d(sigma) of one shot.
 *
 * No counterpart in the reference (satan_i forms its gradient from
 * frequency-domain reciprocity fields, satan_i/fwi3d_cpu_function_v1.4.c:
 * 2246-2384); this is the exact derivative of the restated forward path
 * above, written here in scatter form (each forward operation's transpose
 * applied in reverse order) to check the GPU's gather-form adjoint.
 *
 *   misfit = 1/2 sum_{r,f} |S_rf - obs_rf|^2,  S_rf = sum_n d_r[n] W_rf[n],
 *   W_rf[n] = hf_r(f) dt exp((i-1) sqrt(w0 w_f) n dt),
 *   hf = sqrt(-2 w0/(i w)) for H receivers when hfac, else 1.
 * Adjoint source at receiver r, step n: a_r[n] = Re(conj(S_rf - obs_rf) W_rf[n]).
 * sigma enters through ca, cb (every cell), da, db (CPML cells only) and the
 * electric source gain; the gradient is returned for every cell.
 * ====================================================================== */

static void dplus_t(double *lam, size_t c, size_t s, double c1, double c2, double mu) {
    /* transpose of D+(F)[c] = c1 (F[c+s]-F[c]) + c2 (F[c+2s]-F[c-s]) */
    lam[c + s] += c1 * mu; lam[c] -= c1 * mu; lam[c + 2 * s] += c2 * mu; lam[c - s] -= c2 * mu;
}
static void dtypo_t(double *lam, size_t c, size_t s, double c1, double c2, double c2t, double mu) {
    /* transpose of c1 F[c+s] - c2t F[c] + c2 F[c+2s] - c2 F[c-s] */
    lam[c + s] += c1 * mu; lam[c] -= c2t * mu; lam[c + 2 * s] += c2 * mu; lam[c - s] -= c2 * mu;
}
static void dminus_t(double *lam, size_t c, size_t s, double c1, double c2, double mu) {
    /* transpose of D(F)[c] = c1 (F[c]-F[c-s]) + c2 (F[c+s]-F[c-2s]) */
    lam[c] += c1 * mu; lam[c - s] -= c1 * mu; lam[c + s] += c2 * mu; lam[c - 2 * s] -= c2 * mu;
}

int orc_gradient(const orc_params *p, const double *sigma, const double *mu,
                 int nsrc, const int64_t *src_cell, const int32_t *src_comp,
                 const int32_t *src_kind, const double *src_amp,
                 int nt, const double *wavelet,
                 int nrec, const int64_t *rec_cell, const int32_t *rec_comp,
                 int nf, const double *omega, int hfac, const double *obs,
                 double *misfit, double *grad, double *spec) {
    orc_state s;
    memset(&s, 0, sizeof(s));
    if (state_init(&s, p, sigma, mu)) { state_free(&s); return -1; }
    const int nx = s.nx, ny = s.ny, nz = s.nz;
    const size_t n = s.n, sx = 1, sy = (size_t)nx, sz = (size_t)nx * ny;
    const double vol = p->dx * p->dy * p->dz;
    double *hist = malloc(sizeof(double) * 6 * n * (size_t)(nt + 1));
    double *tr = malloc(sizeof(double) * (size_t)nrec * nt);
    if (!hist || !tr) { free(hist); free(tr); state_free(&s); return -1; }
    memset(hist, 0, sizeof(double) * 6 * n);
    /* forward, keeping every state (E, H after each step) */
    for (int t = 0; t < nt; t++) {
        for (int q = 0; q < nsrc; q++) {
            if (src_kind[q] != SRC_MAGNETIC) continue;
            int64_t c = src_cell[q];
            s.f[src_comp[q]][c] = s.f[src_comp[q]][c] - src_amp[q] * wavelet[t + 1] * p->dt / mu[c] / p->dx / p->dy / p->dz;
        }
        e_phase(&s, p);
        for (int q = 0; q < nsrc; q++) {
            if (src_kind[q] != SRC_ELECTRIC) continue;
            int64_t c = src_cell[q];
            s.f[src_comp[q]][c] -= src_amp[q] * (wavelet[t] + wavelet[t + 1]) / 2.f * p->dt * 2.f * p->omega0 / sigma[c] / p->dx / p->dy / p->dz;
        }
        h_phase(&s, p);
        for (int r = 0; r < nrec; r++) tr[(size_t)r * nt + t] = s.f[rec_comp[r]][rec_cell[r]];
        for (int c = 0; c < 6; c++) memcpy(hist + ((size_t)(t + 1) * 6 + c) * n, s.f[c], n * sizeof(double));
    }
    /* spectra, residual, misfit, adjoint sources */
    double complex *R = malloc(sizeof(double complex) * (size_t)nrec * nf);
    double *asrc = malloc(sizeof(double) * (size_t)nrec * nt);
    double J = 0.0;
    for (int r = 0; r < nrec; r++) {
        for (int f = 0; f < nf; f++) {
            double complex hf = 1.0;
            if (hfac && rec_comp[r] >= 3) hf = csqrt(-2.0 * p->omega0 / I / omega[f]);
            const double sw = sqrt(p->omega0 * omega[f]);
            double complex acc = 0.0;
            for (int t = 0; t < nt; t++) acc += hf * (tr[(size_t)r * nt + t] * p->dt * cexp((I - 1.0) * sw * t * p->dt));
            const double complex res = acc - (obs[2 * ((size_t)r * nf + f)] + I * obs[2 * ((size_t)r * nf + f) + 1]);
            R[(size_t)r * nf + f] = res;
            J += 0.5 * creal(res * conj(res));
            if (spec) { spec[2 * ((size_t)r * nf + f)] = creal(acc); spec[2 * ((size_t)r * nf + f) + 1] = cimag(acc); }
        }
        for (int t = 0; t < nt; t++) {
            double a = 0.0;
            for (int f = 0; f < nf; f++) {
                double complex hf = 1.0;
                if (hfac && rec_comp[r] >= 3) hf = csqrt(-2.0 * p->omega0 / I / omega[f]);
                const double sw = sqrt(p->omega0 * omega[f]);
                const double complex W = hf * p->dt * cexp((I - 1.0) * sw * t * p->dt);
                a += creal(conj(R[(size_t)r * nf + f]) * W);
            }
            asrc[(size_t)r * nt + t] = a;
        }
    }
    *misfit = J;

    /* adjoint sweep */
    double *lam[6], *lpsE[6], *lpsH[6];
    for (int c = 0; c < 6; c++) {
        lam[c] = calloc(n, sizeof(double)); lpsE[c] = calloc(n, sizeof(double)); lpsH[c] = calloc(n, sizeof(double));
    }
    memset(grad, 0, n * sizeof(double));
    double *H0 = malloc(sizeof(double) * 3 * n), *E1 = malloc(sizeof(double) * 3 * n);
    const double c1 = p->c1, c2 = p->c2, c2t = p->psi_hyx_typo ? p->c2 : p->c1;
    const double se = (double)p->e_sign, sh = (double)p->h_sign;
    const double dt = p->dt;
    for (int t = nt - 1; t >= 0; t--) {
        const double *Eh0 = hist + ((size_t)t * 6) * n, *Hh0 = hist + ((size_t)t * 6 + 3) * n;
        const double *Eh1 = hist + ((size_t)(t + 1) * 6) * n, *Hh1 = hist + ((size_t)(t + 1) * 6 + 3) * n;
        /* forward states of this step: H before the H phase (magnetic injection applied),
         * E after the E phase (electric injection undone) */
        memcpy(H0, Hh0, sizeof(double) * 3 * n);
        memcpy(E1, Eh1, sizeof(double) * 3 * n);
        for (int q = 0; q < nsrc; q++) {
            const int64_t c = src_cell[q];
            if (src_kind[q] == SRC_MAGNETIC && src_comp[q] >= 3)
                H0[(size_t)(src_comp[q] - 3) * n + c] -= src_amp[q] * wavelet[t + 1] * dt / mu[c] / p->dx / p->dy / p->dz;
            if (src_kind[q] == SRC_ELECTRIC && src_comp[q] < 3)
                E1[(size_t)src_comp[q] * n + c] += src_amp[q] * (wavelet[t] + wavelet[t + 1]) / 2.f * dt * 2.f * p->omega0 / sigma[c] / p->dx / p->dy / p->dz;
        }
        /* sampling adjoint */
        for (int r = 0; r < nrec; r++) lam[rec_comp[r]][rec_cell[r]] += asrc[(size_t)r * nt + t];

        /* ---- H phase transpose ---- */
        double *lEx = lam[0], *lEy = lam[1], *lEz = lam[2], *lHx = lam[3], *lHy = lam[4], *lHz = lam[5];
        /* gradient of the H phase (CPML cells): uses lam of H after the phase */
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    const size_t c = IDX(i, j, k);
                    const double w2 = 2.0 * p->omega0;
                    const double ms[3] = {s.pr[0].msig[i], s.pr[1].msig[j], s.pr[2].msig[k]};
                    for (int a = 0; a < 3; a++) {
                        if (ms[a] == 0.0) continue;
                        const double h = ms[a] * dt * p->omega0 / sigma[c];
                        (void)w2;
                        const double da = s.da[a][c];
                        const double dda = 2.0 * h / (sigma[c] * (1.0 + h) * (1.0 + h));
                        const double rdb = h / (sigma[c] * (1.0 + h));
                        const int in = inbox(&s.upd[3 + a], i, j, k);
                        const double h0 = H0[(size_t)a * n + c], h1 = Hh1[(size_t)a * n + c];
                        grad[c] += lam[3 + a][c] * ((in ? dda * h0 : 0.0) + rdb * (h1 - (in ? da * h0 : h0)));
                    }
                }
        /* z slabs, y slabs, x slabs (reverse of CPML_H4), then the main update */
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    const size_t c = IDX(i, j, k);
                    if (inslab(&s.sh[2], 2, i, j, k)) {
                        const double bh = s.pr[2].bh[k], chd = s.pr[2].ch[k] / p->dz;
                        const double lxz = lpsH[5][c] + s.db[0][c] * lHx[c];
                        const double lyz = lpsH[4][c] - s.db[1][c] * lHy[c];
                        lpsH[5][c] = bh * lxz; lpsH[4][c] = bh * lyz;
                        dplus_t(lEy, c, sz, c1, c2, chd * lxz);
                        dplus_t(lEx, c, sz, c1, c2, chd * lyz);
                    }
                    if (inslab(&s.sh[1], 1, i, j, k)) {
                        const double bh = s.pr[1].bh[j], chd = s.pr[1].ch[j] / p->dy;
                        const double lxy = lpsH[2][c] - s.db[0][c] * lHx[c];
                        const double lzy = lpsH[3][c] + s.db[2][c] * lHz[c];
                        lpsH[2][c] = bh * lxy; lpsH[3][c] = bh * lzy;
                        dplus_t(lEz, c, sy, c1, c2, chd * lxy);
                        dplus_t(lEx, c, sy, c1, c2, chd * lzy);
                    }
                    if (inslab(&s.sh[0], 0, i, j, k)) {
                        const double bh = s.pr[0].bh[i], chd = s.pr[0].ch[i] / p->dx;
                        const double lzx = lpsH[1][c] - s.db[2][c] * lHz[c];
                        const double lyx = lpsH[0][c] + s.db[1][c] * lHy[c];
                        lpsH[1][c] = bh * lzx; lpsH[0][c] = bh * lyx;
                        dplus_t(lEy, c, sx, c1, c2, chd * lzx);
                        dtypo_t(lEz, c, sx, c1, c2, c2t, chd * lyx);
                    }
                }
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    const size_t c = IDX(i, j, k);
                    const double iky = 1.0 / s.pr[1].khd[j], ikz = 1.0 / s.pr[2].khd[k], ikx = 1.0 / s.pr[0].khd[i];
                    if (inbox(&s.upd[3], i, j, k)) {
                        const double w = -sh * s.db[0][c] * lHx[c];
                        dplus_t(lEz, c, sy, c1, c2, w * iky);
                        dplus_t(lEy, c, sz, c1, c2, -w * ikz);
                        lHx[c] *= s.da[0][c];
                    }
                    if (inbox(&s.upd[4], i, j, k)) {
                        const double w = -sh * s.db[1][c] * lHy[c];
                        dplus_t(lEx, c, sz, c1, c2, w * ikz);
                        dplus_t(lEz, c, sx, c1, c2, -w * ikx);
                        lHy[c] *= s.da[1][c];
                    }
                    if (inbox(&s.upd[5], i, j, k)) {
                        const double w = -sh * s.db[2][c] * lHz[c];
                        dplus_t(lEy, c, sx, c1, c2, w * ikx);
                        dplus_t(lEx, c, sy, c1, c2, -w * iky);
                        lHz[c] *= s.da[2][c];
                    }
                }
        /* ---- electric source transpose: sigma enters through the gain ---- */
        for (int q = 0; q < nsrc; q++) {
            if (src_kind[q] != SRC_ELECTRIC) continue;
            const int64_t c = src_cell[q];
            const double g = src_amp[q] * (wavelet[t] + wavelet[t + 1]) / 2.0 * dt * 2.0 * p->omega0 / sigma[c] / vol;
            grad[c] += lam[src_comp[q]][c] * g / sigma[c];
        }
        /* ---- E phase transpose ---- */
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    const size_t c = IDX(i, j, k);
                    const double es[3] = {s.pr[0].esig[i], s.pr[1].esig[j], s.pr[2].esig[k]};
                    for (int a = 0; a < 3; a++) {
                        const double h = es[a] * dt * p->omega0 / sigma[c];
                        const double ca = s.ca[a][c];
                        const double dca = 2.0 * h / (sigma[c] * (1.0 + h) * (1.0 + h));
                        const double rcb = -1.0 / (sigma[c] * (1.0 + h));
                        const int in = inbox(&s.upd[a], i, j, k);
                        const double e0 = Eh0[(size_t)a * n + c], e1 = E1[(size_t)a * n + c];
                        grad[c] += lam[a][c] * ((in ? dca * e0 : 0.0) + rcb * (e1 - (in ? ca * e0 : e0)));
                    }
                }
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    const size_t c = IDX(i, j, k);
                    if (inslab(&s.se[2], 2, i, j, k)) {
                        const double be = s.pr[2].be[k], ced = s.pr[2].ce[k] / p->dz;
                        const double lyz = lpsE[4][c] + s.cb[1][c] * lEy[c];
                        const double lxz = lpsE[5][c] - s.cb[0][c] * lEx[c];
                        lpsE[4][c] = be * lyz; lpsE[5][c] = be * lxz;
                        dminus_t(lHx, c, sz, c1, c2, ced * lyz);
                        dminus_t(lHy, c, sz, c1, c2, ced * lxz);
                    }
                    if (inslab(&s.se[1], 1, i, j, k)) {
                        const double be = s.pr[1].be[j], ced = s.pr[1].ce[j] / p->dy;
                        const double lxy = lpsE[2][c] + s.cb[0][c] * lEx[c];
                        const double lzy = lpsE[3][c] - s.cb[2][c] * lEz[c];
                        lpsE[2][c] = be * lxy; lpsE[3][c] = be * lzy;
                        dminus_t(lHz, c, sy, c1, c2, ced * lxy);
                        dminus_t(lHx, c, sy, c1, c2, ced * lzy);
                    }
                    if (inslab(&s.se[0], 0, i, j, k)) {
                        const double be = s.pr[0].be[i], ced = s.pr[0].ce[i] / p->dx;
                        const double lzx = lpsE[0][c] + s.cb[2][c] * lEz[c];
                        const double lyx = lpsE[1][c] - s.cb[1][c] * lEy[c];
                        lpsE[0][c] = be * lzx; lpsE[1][c] = be * lyx;
                        dminus_t(lHy, c, sx, c1, c2, ced * lzx);
                        dminus_t(lHz, c, sx, c1, c2, ced * lyx);
                    }
                }
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    const size_t c = IDX(i, j, k);
                    const double iky = 1.0 / s.pr[1].ked[j], ikz = 1.0 / s.pr[2].ked[k], ikx = 1.0 / s.pr[0].ked[i];
                    if (inbox(&s.upd[0], i, j, k)) {
                        const double w = se * s.cb[0][c] * lEx[c];
                        dminus_t(lHz, c, sy, c1, c2, w * iky);
                        dminus_t(lHy, c, sz, c1, c2, -w * ikz);
                        lEx[c] *= s.ca[0][c];
                    }
                    if (inbox(&s.upd[1], i, j, k)) {
                        const double w = se * s.cb[1][c] * lEy[c];
                        dminus_t(lHx, c, sz, c1, c2, w * ikz);
                        dminus_t(lHz, c, sx, c1, c2, -w * ikx);
                        lEy[c] *= s.ca[1][c];
                    }
                    if (inbox(&s.upd[2], i, j, k)) {
                        const double w = se * s.cb[2][c] * lEz[c];
                        dminus_t(lHy, c, sx, c1, c2, w * ikx);
                        dminus_t(lHx, c, sy, c1, c2, -w * iky);
                        lEz[c] *= s.ca[2][c];
                    }
                }
    }
    for (int c = 0; c < 6; c++) { free(lam[c]); free(lpsE[c]); free(lpsH[c]); }
    free(H0); free(E1); free(hist); free(tr); free(R); free(asrc);
    state_free(&s);
    return 0;
}
