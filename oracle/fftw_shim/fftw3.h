/*
 * fftw3.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Minimal stand-in for the FFTW3 interface (FFTW 3.x; the reference pins no
 * version: satan_i/Makefile:13 links -lfftw3) so the reference's satan_i C
 * sources compile here without the library.  It declares only the calls the
 * reference makes (satan_i/fwi3d_cpu_function_v1.4.c:1506-1555) and
 * implements them as a naive O(N^2) DFT with FFTW's published conventions:
 * FFTW_FORWARD = -1 (exp(-2 pi i jk/N)), FFTW_BACKWARD = +1, unnormalised.
 */
#ifndef MITTET_FFTW_SHIM_H
#define MITTET_FFTW_SHIM_H
#include <stddef.h>
/* FFTW's documented rule: with <complex.h> included first, fftw_complex is the
 * native C99 complex type; otherwise double[2].  Same memory layout. */
#if defined(_Complex_I) && defined(complex) && defined(I)
typedef double _Complex fftw_complex;
#else
typedef double fftw_complex[2];
#endif
typedef struct shim_plan_s *fftw_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
#endif
