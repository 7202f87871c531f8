// gamma.cu -- mittet_satan_gamma(): satan_i's frequency-domain gradient
// formula on the GPU.
//
// satan_i forms its FWI gradient from frequency-domain fields
// (satan_i/fwi3d_cpu_function_v1.4.c):
//   residualE   (:2202-2244)  dE_d[rec][w] = obs_d[rec][w] - E_ff,d[w](receiver cell),
//                             err_sum += |dE_x| + |dE_y| + |dE_z|
//   sensitivity (:2246-2290)  sense = sum_rec sum_dir sum_w sum_c |E_ff,c[w] E_bb,c[rec][dir][w]|
//   conv_GdelE  (:2292-2349)  E_back,c[w] = sum_rec sum_dir E_bb,c[rec][dir][w] conj(dE_dir[rec][w])
//   calc_gamma  (:2351-2384)  grad += Re(sum_w sum_c E_ff,c[w] E_back,c[w]) / sense
//                             on k, j, i in [ncpml, n - ncpml)
// Each of the three per-cell loops reads the whole E_bb volume set (nrec x 3
// x 3 x nf complex volumes); here they are one pass: one thread per cell
// reads every E_bb value of its cell once (coalesced, cell index fastest in
// every array), accumulates sense and the three E_back values of a
// frequency in registers, and adds the frequency's gamma term.  The kernel
// is HBM-bound: 16 bytes per E_bb value, 3 x 16 per E_ff value, plus the
// optional E_back write.  All arithmetic is FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/mittet.h"

namespace mittet {
void set_last_error(const char *msg);  // defined in mittet_capi.cu
}

namespace {

int gfail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    mittet::set_last_error(buf);
    return code;
}

struct GBuf {
    void *p = nullptr;
    ~GBuf() {
        if (p) cudaFree(p);
    }
};

#define GCK(call)                                                                                        \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) {                                                                         \
            cudaGetLastError();                                                                          \
            return gfail(e_ == cudaErrorMemoryAllocation ? MITTET_ERR_OOM : MITTET_ERR_CUDA, "%s: %s", #call, \
                         cudaGetErrorString(e_));                                                        \
        }                                                                                                \
    } while (0)

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmul_conj(double2 a, double2 b) {  // a * conj(b)
    return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// residualE: one thread per (component, receiver, frequency).
__global__ void residual_e_kernel(const double2 *__restrict__ obs, const double2 *__restrict__ eff,
                                  const long long *__restrict__ rcell, int nrec, int nf, long long n,
                                  double2 *__restrict__ de) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= 3 * nrec * nf) return;
    const int c = q / (nrec * nf), r = (q / nf) % nrec, w = q % nf;
    const double2 e = eff[((long long)c * nf + w) * n + rcell[r]];
    const double2 o = obs[q];
    de[q] = make_double2(o.x - e.x, o.y - e.y);
}

// sensitivity + conv_GdelE + calc_gamma, one thread per cell.
//   eff  [3][nf][n], ebb [3][nrec][3][nf][n], de [3][nrec][nf]
__global__ void __launch_bounds__(256) satan_gamma_kernel(const double2 *__restrict__ eff,
                                                          const double2 *__restrict__ ebb,
                                                          const double2 *__restrict__ de, int nrec, int nf,
                                                          int nx, int ny, int nz, int ncpml, int normalize,
                                                          double *__restrict__ sense_out,
                                                          double2 *__restrict__ back_out,
                                                          double *__restrict__ grad) {
    const long long n = (long long)nx * ny * nz;
    const long long bstride = (long long)nrec * 3 * nf * n;  // one component's E_bb block
    for (long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x; cell < n;
         cell += (long long)gridDim.x * blockDim.x) {
        double sense = 0.0, gsum = 0.0;
        for (int w = 0; w < nf; w++) {
            double2 f[3], b[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                f[c] = eff[((long long)c * nf + w) * n + cell];
                b[c] = make_double2(0.0, 0.0);
            }
            for (int r = 0; r < nrec; r++)
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    const double2 dd = de[((long long)d * nrec + r) * nf + w];
                    const long long o = (((long long)r * 3 + d) * nf + w) * n + cell;
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const double2 g = ebb[c * bstride + o];
                        const double2 p = cmul(f[c], g);
                        sense += hypot(p.x, p.y);
                        const double2 t = cmul_conj(g, dd);
                        b[c].x += t.x;
                        b[c].y += t.y;
                    }
                }
            double re = 0.0;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                re += f[c].x * b[c].x - f[c].y * b[c].y;
                if (back_out) back_out[((long long)c * nf + w) * n + cell] = b[c];
            }
            gsum += re;
        }
        if (sense_out) sense_out[cell] = sense;
        const int i = (int)(cell % nx), j = (int)((cell / nx) % ny), k = (int)(cell / ((long long)nx * ny));
        if (i >= ncpml && i < nx - ncpml && j >= ncpml && j < ny - ncpml && k >= ncpml && k < nz - ncpml)
            grad[cell] += normalize ? gsum / sense : gsum;
    }
}

}  // namespace

extern "C" int mittet_satan_gamma(int32_t device, const mittet_grid *g, int32_t nrec, const int32_t *rec_pos,
                                  int32_t nf, const double *obs, const double *e_ff, const double *e_bb,
                                  int32_t normalize, double *err_sum, double *de_out, double *sense,
                                  double *e_back, double *grad) {
    if (!g || !e_ff || !e_bb || !grad || nrec < 0 || nf <= 0 || (nrec > 0 && (!rec_pos || (!obs && !de_out))))
        return gfail(MITTET_ERR_INVALID_ARG, "bad satan_gamma arguments");
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    if (nx <= 0 || ny <= 0 || nz <= 0 || g->ncpml < 0) return gfail(MITTET_ERR_INVALID_ARG, "bad grid");
    const long long n = (long long)nx * ny * nz;
    std::vector<long long> rc((size_t)(nrec > 0 ? nrec : 1));
    for (int r = 0; r < nrec; r++) {
        const int px = rec_pos[3 * r], py = rec_pos[3 * r + 1], pz = rec_pos[3 * r + 2];
        if (px < 1 || px > nx || py < 1 || py > ny || pz < 1 || pz > nz)
            return gfail(MITTET_ERR_INVALID_ARG, "receiver %d outside the grid", r);
        rc[r] = ((long long)(pz - 1) * ny + (py - 1)) * nx + (px - 1);
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return gfail(MITTET_ERR_CUDA, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return gfail(MITTET_ERR_INVALID_ARG, "device %d out of range", device);
    GCK(cudaSetDevice(device));
    const size_t nff = (size_t)3 * nf * n, nbb = (size_t)3 * nrec * 3 * nf * n, nde = (size_t)3 * nrec * nf;
    GBuf dff, dbb, dobs, dde, drc, dsense, dback, dgrad;
    GCK(cudaMalloc(&dff.p, nff * 16));
    GCK(cudaMalloc(&dbb.p, (nbb ? nbb : 1) * 16));
    GCK(cudaMalloc(&dobs.p, (nde ? nde : 1) * 16));
    GCK(cudaMalloc(&dde.p, (nde ? nde : 1) * 16));
    GCK(cudaMalloc(&drc.p, rc.size() * 8));
    GCK(cudaMalloc(&dgrad.p, (size_t)n * 8));
    if (sense) GCK(cudaMalloc(&dsense.p, (size_t)n * 8));
    if (e_back) GCK(cudaMalloc(&dback.p, nff * 16));
    GCK(cudaMemcpy(dff.p, e_ff, nff * 16, cudaMemcpyHostToDevice));
    if (nbb) GCK(cudaMemcpy(dbb.p, e_bb, nbb * 16, cudaMemcpyHostToDevice));
    if (nde && obs) GCK(cudaMemcpy(dobs.p, obs, nde * 16, cudaMemcpyHostToDevice));
    if (nde && !obs) GCK(cudaMemcpy(dde.p, de_out, nde * 16, cudaMemcpyHostToDevice));  // residual given
    GCK(cudaMemcpy(drc.p, rc.data(), rc.size() * 8, cudaMemcpyHostToDevice));
    GCK(cudaMemcpy(dgrad.p, grad, (size_t)n * 8, cudaMemcpyHostToDevice));
    if (nde && obs) {
        residual_e_kernel<<<(int)((nde + 255) / 256), 256>>>((const double2 *)dobs.p, (const double2 *)dff.p,
                                                            (const long long *)drc.p, nrec, nf, n, (double2 *)dde.p);
        GCK(cudaGetLastError());
    }
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 8);
    satan_gamma_kernel<<<blocks, 256>>>((const double2 *)dff.p, (const double2 *)dbb.p, (const double2 *)dde.p, nrec,
                                        nf, nx, ny, nz, g->ncpml, normalize ? 1 : 0, (double *)dsense.p,
                                        (double2 *)dback.p, (double *)dgrad.p);
    GCK(cudaGetLastError());
    GCK(cudaMemcpy(grad, dgrad.p, (size_t)n * 8, cudaMemcpyDeviceToHost));
    if (sense) GCK(cudaMemcpy(sense, dsense.p, (size_t)n * 8, cudaMemcpyDeviceToHost));
    if (e_back) GCK(cudaMemcpy(e_back, dback.p, nff * 16, cudaMemcpyDeviceToHost));
    std::vector<double> dh(2 * (nde ? nde : 1));
    if (nde) GCK(cudaMemcpy(dh.data(), dde.p, nde * 16, cudaMemcpyDeviceToHost));
    if (de_out && nde && obs) memcpy(de_out, dh.data(), nde * 16);
    if (err_sum) {
        // residualE's sum over receivers, frequencies and x, y, z in its own order
        double s = 0.0;
        for (int r = 0; r < nrec; r++)
            for (int w = 0; w < nf; w++)
                for (int c = 0; c < 3; c++) {
                    const size_t q = ((size_t)c * nrec + r) * nf + w;
                    s += std::hypot(dh[2 * q], dh[2 * q + 1]);
                }
        *err_sum = s;
    }
    return MITTET_OK;
}
