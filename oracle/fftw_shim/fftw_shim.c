/* TEST INFRASTRUCTURE ONLY: naive DFT behind the fftw3.h stand-in. */
#include <math.h>
#include <stdlib.h>
#include "fftw3.h"

typedef double shim_c2[2];

struct shim_plan_s { int n, sign; shim_c2 *in, *out; };

void *fftw_malloc(size_t n) { return malloc(n); }
void fftw_free(void *p) { free(p); }

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
    (void)flags;
    fftw_plan p = (fftw_plan)malloc(sizeof(*p));
    p->n = n; p->sign = sign; p->in = (shim_c2 *)in; p->out = (shim_c2 *)out;
    return p;
}

void fftw_execute(const fftw_plan p) {
    const int n = p->n;
    shim_c2 *tmp = (shim_c2 *)malloc(sizeof(shim_c2) * (size_t)n);
    const double two_pi = 6.283185307179586476925286766559;
    for (int k = 0; k < n; k++) {
        double re = 0.0, im = 0.0;
        for (int j = 0; j < n; j++) {
            /* reduce jk mod n first so the angle stays small and exact */
            long long m = ((long long)j * k) % n;
            double a = p->sign * two_pi * (double)m / (double)n;
            double c = cos(a), s = sin(a);
            re += p->in[j][0] * c - p->in[j][1] * s;
            im += p->in[j][0] * s + p->in[j][1] * c;
        }
        tmp[k][0] = re; tmp[k][1] = im;
    }
    for (int k = 0; k < n; k++) { p->out[k][0] = tmp[k][0]; p->out[k][1] = tmp[k][1]; }
    free(tmp);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
