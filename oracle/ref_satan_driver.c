/*
 * ref_satan_driver.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Runs the reference's own satan_i forward kernels, compiled from their
 * sources (satan_i/fwi3d_cpu_function_v1.4.c, fwi3d_cpu_cpmlabc_v1.4.c,
 * fwi3d_cpu_lattice_v1.4.c), on inputs given in a binary file, and writes the
 * receiver traces and final fields.  It replaces only the reference's
 * text-file driver (satan_i/fwi3d_cpu_rec2rec_v1.4.c:16-66, which reads
 * ./data/*.dat): the time loop below is the reference's fwdpropagation()
 * (satan_i/fwi3d_cpu_function_v1.4.c:2528-2536) with the source component
 * selectable as in ThreeCfwdpropagation() (:2539-2550).
 * The reference functions write coefficient dumps under ./data, so run it in
 * a scratch directory that has a data/ subdirectory.
 *
 * input:  int32 ix iy iz ncpml nt scomp spx spy spz nrec {rpx rpy rpz rcomp}*nrec
 *         double dx dy dz omega_0 minval maxval sigma[ix*iy*iz] wavelet[nt+1]
 * output: double dt cmax traces[nrec][nt] fields[6][ix*iy*iz]
 *
 * Timing mode (argv[3] = nseg): the loop runs nseg segments of nt steps each
 * (the wavelet then holds nseg*nt+1 samples) and the output is the wall time
 * of every segment (double[nseg]); set-up is outside the timed segments.
 */
#include <omp.h>
#include "fwi3d_cpu_header1_v1.4.h"

static void rd(void *p, size_t sz, size_t n, FILE *f) {
    if (fread(p, sz, n, f) != n) { fprintf(stderr, "short read\n"); exit(2); }
}

int main(int argc, char **argv) {
    if (argc != 3 && argc != 4) { fprintf(stderr, "usage: %s input.bin output.bin [nseg]\n", argv[0]); return 2; }
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
    double *tr = malloc(sizeof(double) * (size_t)nt * (rec_num > 0 ? rec_num : 1));
    for (int step = 0; step < nt; step++) {
        e_field_cpml42(EX, EY, EZ, HX, HY, HZ);
        epml_abcs4(EX, EY, EZ, HX, HY, HZ);
        if (scomp == 0) read_source_3d(EX, signalX, 0, step);
        if (scomp == 1) read_source_3d(EY, signalX, 0, step);
        if (scomp == 2) read_source_3d(EZ, signalX, 0, step);
        h_field_cpml42(EX, EY, EZ, HX, HY, HZ);
        hpml_abcs4(EX, EY, EZ, HX, HY, HZ);
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
    fclose(fo);
    return 0;
}
