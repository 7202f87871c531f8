/*
 * ref_satan_driver.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Runs the reference's own satan_i functions, compiled from their sources
 * (satan_i/fwi3d_cpu_function_v1.4.c, fwi3d_cpu_cpmlabc_v1.4.c,
 * fwi3d_cpu_lattice_v1.4.c), on inputs given in a binary file, and writes
 * their results to a binary file.  It replaces only the reference's text-file
 * drivers (satan_i/fwi3d_cpu_rec2rec_v1.4.c:16-66 and
 * fwi3d_cpu_inv_fwi_v1.4.c:16-113, which read ./data/*.dat); every number
 * below is computed by the reference's functions.  They write text dumps
 * under ./data, so run it in a scratch directory that has a data/ directory.
 *
 *   satan_ref [fwd] in out [nseg]
 *     The forward time loop: fwdpropagation() (function.c:2528-2536) with the
 *     source component selectable as in ThreeCfwdpropagation() (:2539-2550).
 *     input:  int32 ix iy iz ncpml nt scomp spx spy spz nrec {rpx rpy rpz rcomp}*nrec
 *             int32 nvol  (only when the mode word "fwd" is given)
 *             double dx dy dz omega_0 minval maxval sigma[ix*iy*iz] wavelet[nt+1]
 *     output: double dt cmax traces[nrec][nt] fields[6][ix*iy*iz]
 *             and, when nvol > 0, EcalX_ff EcalY_ff EcalZ_ff [nvol-1][n] complex:
 *             the full-volume transform laplaceToFreq_2 (function.c:2091-2200)
 *             of the E history copytoEcal (:1652-1686) keeps, w = 1 .. nvol-1
 *             (startF = 1, upperF = nvol), it = nt + 1 samples (the last one
 *             zero, as the reference never writes it), with JX_f = delta / dt
 *             and signalTrue = delta, so EcalX_ff = EX_w / sqrt(-2 w0/(i w)).
 *     Timing mode (nseg): nseg segments of nt steps each (the wavelet then
 *     holds nseg*nt+1 samples); output the wall time of every segment.
 *
 *   satan_ref ftod in out
 *     laplaceToFreq (function.c:1976-2089) on given traces, one receiver per
 *     call (its spectra arrays hold one receiver), then once over all of them
 *     so that it writes its spectrum_*_000_RRR.dat files.
 *     input:  int32 it nrec upperF; double dt omega_0 traces[nrec][3][it] jx[it]
 *     output: complex EX_w EY_w EZ_w JX_w, [nrec][4][it]
 *
 *   satan_ref gamma in out
 *     residualE(0), sensitivity(), conv_GdelE(), calc_gamma()
 *     (function.c:2202-2384) on given spectra.
 *     input:  int32 ix iy iz ncpml rec_num upperF {px py pz}*rec_num
 *             double dx dy dz
 *             complex Exobs Eyobs Ezobs [rec][upperF],
 *                     EcalX_ff EcalY_ff EcalZ_ff [upperF][n],
 *                     EcalX_bb EcalY_bb EcalZ_bb [rec][3][upperF][n]
 *     output: double err_sum; complex delEx_f delEy_f delEz_f [rec][upperF];
 *             double sense[n]; complex EcalX_back EcalY_back EcalZ_back
 *             [upperF][n]; double grad[n]
 *
 *   satan_ref update in out
 *     calc_phi(), calc_alpha(0), update_para2(0) (function.c:2565-2603,
 *     2757-2832), writing sig_tmp.dat, gradient_000.dat and sig_000.dat.
 *     input:  int32 ix iy iz ncpml iseabed rec_num upperF {px py pz}*rec_num
 *             double dx dy dz minval maxval sig[n] grad[n]
 *             complex delEx_f delEy_f delEz_f [rec][upperF],
 *                     EcalX_ffL EcalY_ffL EcalZ_ffL [upperF][n] (shot 0),
 *                     EcalX_ff2 EcalY_ff2 EcalZ_ff2 [upperF][n]
 *     output: double scaler k1re k1im k2re k2im alpha sig2[n] sig[n]
 */
#include <complex.h>
#include <omp.h>
#include <string.h>
#include "fwi3d_cpu_header1_v1.4.h"

static void rd(void *p, size_t sz, size_t n, FILE *f) {
    if (n && fread(p, sz, n, f) != n) { fprintf(stderr, "short read\n"); exit(2); }
}
static void *zalloc(size_t bytes) {
    void *p = calloc(bytes ? bytes : 1, 1);
    if (!p) { fprintf(stderr, "out of memory\n"); exit(3); }
    return p;
}
static double _Complex *rdc(size_t count, FILE *f) {
    double _Complex *p = zalloc(sizeof(double _Complex) * count);
    rd(p, sizeof(double _Complex), count, f);
    return p;
}
static void read_positions(int nrec, FILE *f) {
    int32_t *pos = zalloc(sizeof(int32_t) * 3 * (nrec > 0 ? nrec : 1));
    rd(pos, 4, 3 * (size_t)nrec, f);
    rec_px = zalloc(sizeof(int) * (nrec + 1));
    rec_py = zalloc(sizeof(int) * (nrec + 1));
    rec_pz = zalloc(sizeof(int) * (nrec + 1));
    for (int r = 0; r < nrec; r++) { rec_px[r] = pos[3 * r]; rec_py[r] = pos[3 * r + 1]; rec_pz[r] = pos[3 * r + 2]; }
    free(pos);
}

static int mode_ftod(FILE *fi, FILE *fo) {
    int32_t hdr[3];
    rd(hdr, 4, 3, fi);
    it = hdr[0];
    const int nrec = hdr[1];
    upperF = hdr[2];
    double dh[2];
    rd(dh, 8, 2, fi);
    dt = dh[0];
    omega_0 = dh[1];
    fmax_w = 1.0;  /* enters only t0 and beta, which laplaceToFreq computes and never uses */
    double *tr = zalloc(sizeof(double) * (size_t)nrec * 3 * it);
    rd(tr, 8, (size_t)nrec * 3 * it, fi);
    double *jx = zalloc(sizeof(double) * it);
    rd(jx, 8, it, fi);
    EX_f = zalloc(sizeof(double) * it); EY_f = zalloc(sizeof(double) * it); EZ_f = zalloc(sizeof(double) * it);
    EX_w = zalloc(sizeof(double _Complex) * it); EY_w = zalloc(sizeof(double _Complex) * it);
    EZ_w = zalloc(sizeof(double _Complex) * it); JX_w = zalloc(sizeof(double _Complex) * it);
    GX_w = zalloc(sizeof(double _Complex) * it); GY_w = zalloc(sizeof(double _Complex) * it);
    GZ_w = zalloc(sizeof(double _Complex) * it);
    JX_f = zalloc(sizeof(double _Complex) * it);
    for (int k = 0; k < (int)it; k++) JX_f[k] = jx[k];
    signalTrue = zalloc(sizeof(double) * it);
    signalTrue[0] = 1.0;
    double *ax = zalloc(sizeof(double) * (size_t)nrec * it), *ay = zalloc(sizeof(double) * (size_t)nrec * it),
           *az = zalloc(sizeof(double) * (size_t)nrec * it);
    for (int r = 0; r < nrec; r++)
        for (int k = 0; k < (int)it; k++) {
            ax[(size_t)r * it + k] = tr[((size_t)r * 3 + 0) * it + k];
            ay[(size_t)r * it + k] = tr[((size_t)r * 3 + 1) * it + k];
            az[(size_t)r * it + k] = tr[((size_t)r * 3 + 2) * it + k];
        }
    double _Complex *out = zalloc(sizeof(double _Complex) * (size_t)nrec * 4 * it);
    for (int r = 0; r < nrec; r++) {
        rec_num = 1;
        all_recEX = ax + (size_t)r * it;
        all_recEY = ay + (size_t)r * it;
        all_recEZ = az + (size_t)r * it;
        laplaceToFreq(100 + r);
        memcpy(out + ((size_t)r * 4 + 0) * it, EX_w, sizeof(double _Complex) * it);
        memcpy(out + ((size_t)r * 4 + 1) * it, EY_w, sizeof(double _Complex) * it);
        memcpy(out + ((size_t)r * 4 + 2) * it, EZ_w, sizeof(double _Complex) * it);
        memcpy(out + ((size_t)r * 4 + 3) * it, JX_w, sizeof(double _Complex) * it);
    }
    rec_num = nrec;
    all_recEX = ax;
    all_recEY = ay;
    all_recEZ = az;
    laplaceToFreq(0);
    fwrite(out, sizeof(double _Complex), (size_t)nrec * 4 * it, fo);
    return 0;
}

static int mode_gamma(FILE *fi, FILE *fo) {
    int32_t hdr[6];
    rd(hdr, 4, 6, fi);
    ix = hdr[0]; iy = hdr[1]; iz = hdr[2]; ncpml = hdr[3]; rec_num = hdr[4]; upperF = hdr[5];
    n = ix * iy * iz;
    read_positions(rec_num, fi);
    double dh[3];
    rd(dh, 8, 3, fi);
    dx = dh[0]; dy = dh[1]; dz = dh[2];
    const size_t ns = (size_t)rec_num * upperF, nf = (size_t)upperF * n, nb = (size_t)rec_num * 3 * upperF * n;
    Exobs = rdc(ns, fi); Eyobs = rdc(ns, fi); Ezobs = rdc(ns, fi);
    EcalX_ff = rdc(nf, fi); EcalY_ff = rdc(nf, fi); EcalZ_ff = rdc(nf, fi);
    EcalX_bb = rdc(nb, fi); EcalY_bb = rdc(nb, fi); EcalZ_bb = rdc(nb, fi);
    delEx_f = zalloc(sizeof(double _Complex) * ns);
    delEy_f = zalloc(sizeof(double _Complex) * ns);
    delEz_f = zalloc(sizeof(double _Complex) * ns);
    EcalX_back = zalloc(sizeof(double _Complex) * nf);
    EcalY_back = zalloc(sizeof(double _Complex) * nf);
    EcalZ_back = zalloc(sizeof(double _Complex) * nf);
    sense = zalloc(sizeof(double) * n);
    grad = zalloc(sizeof(double) * n);
    err_sum = zalloc(sizeof(double) * MAXITR);
    residualE(0);
    sensitivity();
    conv_GdelE();
    calc_gamma();
    fwrite(&err_sum[0], 8, 1, fo);
    fwrite(delEx_f, sizeof(double _Complex), ns, fo);
    fwrite(delEy_f, sizeof(double _Complex), ns, fo);
    fwrite(delEz_f, sizeof(double _Complex), ns, fo);
    fwrite(sense, 8, n, fo);
    fwrite(EcalX_back, sizeof(double _Complex), nf, fo);
    fwrite(EcalY_back, sizeof(double _Complex), nf, fo);
    fwrite(EcalZ_back, sizeof(double _Complex), nf, fo);
    fwrite(grad, 8, n, fo);
    return 0;
}

static int mode_update(FILE *fi, FILE *fo) {
    int32_t hdr[7];
    rd(hdr, 4, 7, fi);
    ix = hdr[0]; iy = hdr[1]; iz = hdr[2]; ncpml = hdr[3]; iseabed = hdr[4]; rec_num = hdr[5]; upperF = hdr[6];
    n = ix * iy * iz;
    read_positions(rec_num, fi);
    double dh[5];
    rd(dh, 8, 5, fi);
    dx = dh[0]; dy = dh[1]; dz = dh[2]; minval = dh[3]; maxval = dh[4];
    sig = zalloc(sizeof(double) * n);
    rd(sig, 8, n, fi);
    grad = zalloc(sizeof(double) * n);
    rd(grad, 8, n, fi);
    sig2 = zalloc(sizeof(double) * n);
    grad_p = zalloc(sizeof(double) * n);
    const size_t ns = (size_t)rec_num * upperF, nf = (size_t)upperF * n;
    delEx_f = rdc(ns, fi); delEy_f = rdc(ns, fi); delEz_f = rdc(ns, fi);
    EcalX_ffL = rdc(nf, fi); EcalY_ffL = rdc(nf, fi); EcalZ_ffL = rdc(nf, fi);
    EcalX_ff2 = rdc(nf, fi); EcalY_ff2 = rdc(nf, fi); EcalZ_ff2 = rdc(nf, fi);
    k1 = k2 = 0;
    calc_phi();
    calc_alpha(0);
    update_para2(0);
    const double head[6] = {scaler, creal(k1), cimag(k1), creal(k2), cimag(k2), alpha};
    fwrite(head, 8, 6, fo);
    fwrite(sig2, 8, n, fo);
    fwrite(sig, 8, n, fo);
    return 0;
}

static int mode_fwd(int argc, char **argv, int with_vol) {
    const int nseg = argc == 4 ? atoi(argv[3]) : 0;
    FILE *fi = fopen(argv[1], "rb");
    if (!fi) return 2;
    int32_t hdr[10];
    rd(hdr, 4, 10, fi);
    ix = hdr[0]; iy = hdr[1]; iz = hdr[2]; ncpml = hdr[3];
    int nt = hdr[4], scomp = hdr[5];
    shot_num = 1;
    shot_px = malloc(sizeof(int)); shot_py = malloc(sizeof(int)); shot_pz = malloc(sizeof(int));
    shot_px[0] = hdr[6]; shot_py[0] = hdr[7]; shot_pz[0] = hdr[8];
    rec_num = hdr[9];
    int32_t *rec = malloc(sizeof(int32_t) * 4 * (rec_num > 0 ? rec_num : 1));
    rd(rec, 4, 4 * (size_t)rec_num, fi);
    rec_px = malloc(sizeof(int) * (rec_num + 1)); rec_py = malloc(sizeof(int) * (rec_num + 1)); rec_pz = malloc(sizeof(int) * (rec_num + 1));
    for (int r = 0; r < rec_num; r++) { rec_px[r] = rec[4 * r]; rec_py[r] = rec[4 * r + 1]; rec_pz[r] = rec[4 * r + 2]; }
    int32_t nvol = 0;
    if (with_vol) rd(&nvol, 4, 1, fi);
    double dh[6];
    rd(dh, 8, 6, fi);
    dx = dh[0]; dy = dh[1]; dz = dh[2]; omega_0 = dh[3]; minval = dh[4]; maxval = dh[5];
    const int nsteps_total = nseg > 0 ? nseg * nt : nt;
    it = nsteps_total + 1;
    init_eh_field_3d();
    rd(sig, 8, (size_t)n, fi);
    signalX = malloc(sizeof(double) * it);
    rd(signalX, 8, (size_t)it, fi);
    fclose(fi);

    lattice_time_3d();
    init_cpml();
    media_coeff_3d();
    set_zero_eh();

    double *F[6] = {EX, EY, EZ, HX, HY, HZ};
    if (nseg > 0) {
        double *tseg = malloc(sizeof(double) * nseg);
        int step = 0;
        for (int s = 0; s < nseg; s++) {
            double t0 = omp_get_wtime();
            for (int q = 0; q < nt; q++, step++) {
                e_field_cpml42(EX, EY, EZ, HX, HY, HZ);
                epml_abcs4(EX, EY, EZ, HX, HY, HZ);
                if (scomp == 0) read_source_3d(EX, signalX, 0, step);
                if (scomp == 1) read_source_3d(EY, signalX, 0, step);
                if (scomp == 2) read_source_3d(EZ, signalX, 0, step);
                h_field_cpml42(EX, EY, EZ, HX, HY, HZ);
                hpml_abcs4(EX, EY, EZ, HX, HY, HZ);
            }
            tseg[s] = omp_get_wtime() - t0;
        }
        FILE *fo = fopen(argv[2], "wb");
        fwrite(tseg, 8, (size_t)nseg, fo);
        fclose(fo);
        return 0;
    }
    if (nvol > 0) {
        EcalX_b = zalloc(sizeof(double _Complex) * (size_t)n * it);
        EcalY_b = zalloc(sizeof(double _Complex) * (size_t)n * it);
        EcalZ_b = zalloc(sizeof(double _Complex) * (size_t)n * it);
    }
    double *tr = malloc(sizeof(double) * (size_t)nt * (rec_num > 0 ? rec_num : 1));
    for (int step = 0; step < nt; step++) {
        e_field_cpml42(EX, EY, EZ, HX, HY, HZ);
        epml_abcs4(EX, EY, EZ, HX, HY, HZ);
        if (scomp == 0) read_source_3d(EX, signalX, 0, step);
        if (scomp == 1) read_source_3d(EY, signalX, 0, step);
        if (scomp == 2) read_source_3d(EZ, signalX, 0, step);
        h_field_cpml42(EX, EY, EZ, HX, HY, HZ);
        hpml_abcs4(EX, EY, EZ, HX, HY, HZ);
        if (nvol > 0) copytoEcal(EX, EY, EZ, step);
        for (int r = 0; r < rec_num; r++) {
            int ijk = ix * iy * (rec_pz[r] - 1) + ix * (rec_py[r] - 1) + rec_px[r] - 1;
            tr[(size_t)r * nt + step] = F[rec[4 * r + 3]][ijk];
        }
    }
    FILE *fo = fopen(argv[2], "wb");
    fwrite(&dt, 8, 1, fo);
    fwrite(&cmax, 8, 1, fo);
    fwrite(tr, 8, (size_t)nt * rec_num, fo);
    for (int c = 0; c < 6; c++) fwrite(F[c], 8, (size_t)n, fo);
    if (nvol > 0) {
        startF = 1;
        upperF = nvol;
        fmax_w = 1.0;  /* enters only t0 and beta, which laplaceToFreq_2 never uses */
        JX_f = zalloc(sizeof(double _Complex) * it);
        JX_f[0] = 1.0 / dt;
        signalTrue = zalloc(sizeof(double) * it);
        signalTrue[0] = 1.0;
        const size_t nf = (size_t)upperF * n;
        EcalX_ff = zalloc(sizeof(double _Complex) * nf); EcalY_ff = zalloc(sizeof(double _Complex) * nf);
        EcalZ_ff = zalloc(sizeof(double _Complex) * nf);
        EcalX_ffL = zalloc(sizeof(double _Complex) * nf); EcalY_ffL = zalloc(sizeof(double _Complex) * nf);
        EcalZ_ffL = zalloc(sizeof(double _Complex) * nf);
        laplaceToFreq_2(0);
        fwrite(EcalX_ff + n, sizeof(double _Complex), nf - n, fo);
        fwrite(EcalY_ff + n, sizeof(double _Complex), nf - n, fo);
        fwrite(EcalZ_ff + n, sizeof(double _Complex), nf - n, fo);
    }
    fclose(fo);
    return 0;
}

int main(int argc, char **argv) {
    if (argc >= 2 && (!strcmp(argv[1], "ftod") || !strcmp(argv[1], "gamma") || !strcmp(argv[1], "update"))) {
        if (argc != 4) { fprintf(stderr, "usage: %s %s input.bin output.bin\n", argv[0], argv[1]); return 2; }
        FILE *fi = fopen(argv[2], "rb"), *fo = fopen(argv[3], "wb");
        if (!fi || !fo) return 2;
        int rc = !strcmp(argv[1], "ftod") ? mode_ftod(fi, fo) : !strcmp(argv[1], "gamma") ? mode_gamma(fi, fo)
                                                                                          : mode_update(fi, fo);
        fclose(fi);
        fclose(fo);
        return rc;
    }
    int with_vol = 0;
    if (argc >= 2 && !strcmp(argv[1], "fwd")) {
        with_vol = 1;
        argv++;
        argc--;
    }
    if (argc != 3 && argc != 4) { fprintf(stderr, "usage: %s [fwd] input.bin output.bin [nseg]\n", argv[0]); return 2; }
    return mode_fwd(argc, argv, with_vol);
}
