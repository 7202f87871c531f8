// mittet_noalloc.cu -- mittet_forward_noalloc(): a forward solve that
// allocates nothing.
//
// Who needs it: host code that must not call cudaMalloc/cudaFree.  cudaFree
// (and often cudaMalloc) synchronises the whole device, which stalls every
// other stream of a latency-bound serving process; and hosts whose device
// memory is owned by another allocator (a framework's caching allocator, a
// fixed per-process budget) cannot take memory behind its back.  For them this entry point keeps every intermediate buffer of the
// solve (fields, CPML psi slabs, model words, profiles, receiver traces) in
// one file-scope __device__ array of fixed size, and takes its inputs and
// outputs from the caller.  It launches the same stencil kernels as
// mittet_forward() (the general body over the whole grid), FP32 fields with
// an FP64 f_to_d of the receiver traces, one shot.
//
// Limits: the array holds MITTET_NOALLOC_SCRATCH_BYTES (32 MiB) and every
// GPU that loads the library holds it until the process exits; grids are at
// most 256 cells per axis, at most 64 source points, 2048 receivers, 256
// frequencies, and the padded layout of the solve must fit the array
// (roughly 96^3 cells with a few hundred receivers for a few thousand steps).
// Calls share the array and keep the last call's contents; everything that
// must start at zero is cleared at the start of each call.  Calls that
// overlap on the GPU (issued on different streams without ordering between
// them) race on the array.  The first call on a device looks up the array's
// device address for that device; make that first call before any stream
// capture.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/mittet.h"
#include "kernels.cuh"
#include "setup_host.h"

namespace mittet {
void set_last_error(const char *msg);  // defined in mittet_capi.cu
}

using namespace mittet;

#define MITTET_NOALLOC_SCRATCH_BYTES (32u << 20)

static __device__ __align__(256) unsigned char g_noalloc_scratch[MITTET_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int NA_MAX_AXIS = 256, NA_MAX_POINTS = 64, NA_MAX_REC = 2048, NA_MAX_FREQ = 256, NA_MAX_DEV = 64;
constexpr int NA_VX = 2, NA_BX = 32, NA_BY = 4, NA_ZC = 4;

std::mutex g_na_mu;
void *g_na_ptr[NA_MAX_DEV] = {nullptr};

int na_fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    set_last_error(buf);
    return code;
}

// Device address of the scratch array on the current device (looked up once
// per device with that device current).
int na_scratch(int dev, unsigned char **out) {
    if (dev < 0 || dev >= NA_MAX_DEV) return na_fail(MITTET_ERR_INVALID_ARG, "device %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (!g_na_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return na_fail(MITTET_ERR_CUDA, "cudaGetSymbolAddress of the scratch array: %s", cudaGetErrorString(e));
        g_na_ptr[dev] = p;
    }
    *out = (unsigned char *)g_na_ptr[dev];
    return MITTET_OK;
}

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

__global__ void na_model_kernel(const double *__restrict__ sig, int nx, int ny, int nz, int px, double two_w0_dt,
                                float *__restrict__ m) {
    const long long n = (long long)nx * ny * nz;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % nx);
        m[(e / nx) * px + i] = (float)(two_w0_dt / sig[e]);
    }
}

// Electric point gains need sigma at the source cell: g = amp dt 2 w0 / sigma / (dx dy dz).
__global__ void na_gain_kernel(SrcPoint *pts, const double *__restrict__ sig, const long long *__restrict__ cell,
                               const double *__restrict__ amp, int npts, double dt, double w0, double mu0, double vol) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npts) return;
    pts[q].g = pts[q].kind == 0 ? amp[q] * dt / mu0 / vol : amp[q] * dt * 2.0 * w0 / sig[cell[q]] / vol;
}

}  // namespace

extern "C" int mittet_forward_noalloc(const mittet_grid *g, const mittet_phys *ph, const double *sigma_dev,
                                      int32_t npoint, const mittet_point_source *pts, int32_t nt,
                                      const double *wavelet_dev, int32_t nrec, const mittet_receiver *rec,
                                      int32_t nf, const double *omega, int32_t h_factor, double *rec_fd_dev,
                                      void *stream) {
    if (!g || !ph || !sigma_dev || !pts || !wavelet_dev || !rec || !omega || !rec_fd_dev)
        return na_fail(MITTET_ERR_INVALID_ARG, "null argument");
    const int nx = g->nx, ny = g->ny, nz = g->nz, nc = g->ncpml;
    if (nx < 8 || ny < 8 || nz < 8 || nx > NA_MAX_AXIS || ny > NA_MAX_AXIS || nz > NA_MAX_AXIS)
        return na_fail(MITTET_ERR_INVALID_ARG, "grid must have 8..%d cells per axis here", NA_MAX_AXIS);
    if (nc < 2 || 2 * nc + 4 > std::min(nx, std::min(ny, nz)))
        return na_fail(MITTET_ERR_INVALID_ARG, "ncpml %d does not fit the grid", nc);
    if (!(g->dx > 0 && g->dy > 0 && g->dz > 0 && ph->dt > 0 && ph->omega0 > 0 && ph->cmax > 0 && ph->mu0 > 0))
        return na_fail(MITTET_ERR_INVALID_ARG, "cell sizes, dt, omega0, cmax and mu0 must be positive");
    if (ph->precision != MITTET_FP32) return na_fail(MITTET_ERR_INVALID_ARG, "this entry point runs FP32 fields only");
    if (ph->flavor != MITTET_FLAVOR_NCVER0027 && ph->flavor != MITTET_FLAVOR_SATAN_I)
        return na_fail(MITTET_ERR_INVALID_ARG, "unknown flavor %d", ph->flavor);
    if (ph->check_cfl) {
        const double dmin = std::min(g->dx, std::min(g->dy, g->dz));
        const double lim = dmin / ph->cmax / std::sqrt(3.0) / 1.16667;
        if (ph->dt > lim * (1.0 + 1e-12)) return na_fail(MITTET_ERR_CFL, "dt %.6e exceeds the (2,4) Taylor limit %.6e", ph->dt, lim);
    }
    if (npoint <= 0 || npoint > NA_MAX_POINTS) return na_fail(MITTET_ERR_INVALID_ARG, "1..%d source points", NA_MAX_POINTS);
    if (nrec <= 0 || nrec > NA_MAX_REC) return na_fail(MITTET_ERR_INVALID_ARG, "1..%d receivers", NA_MAX_REC);
    if (nf <= 0 || nf > NA_MAX_FREQ) return na_fail(MITTET_ERR_INVALID_ARG, "1..%d frequencies", NA_MAX_FREQ);
    if (nt <= 0) return na_fail(MITTET_ERR_INVALID_ARG, "nt must be positive");

    // ---- host set-up on the stack (no heap, no device allocation)
    Setup su;
    su.nx = nx; su.ny = ny; su.nz = nz;
    su.nmax = (std::max(nx, std::max(ny, nz)) + 3) / 4 * 4;
    make_ranges(ph->flavor, nx, ny, nz, nc, su);
    if (!ranges_in_bounds(su)) return na_fail(MITTET_ERR_INVALID_ARG, "grid too small for the flavour's index ranges");
    const int ps = su.nmax;
    static_assert(NA_MAX_AXIS % 4 == 0, "profile stride");
    float prof[3 * P_COUNT * NA_MAX_AXIS];
    {
        const int n3[3] = {nx, ny, nz};
        const double d3[3] = {g->dx, g->dy, g->dz};
        const CpmlConst cc{ph->cpml_nn, ph->cpml_order, ph->cpml_kappa_max, ph->cpml_a_max, ph->cpml_ma, ph->cpml_rcoef,
                           ph->cpml_opt_to_max_x};
        double es[NA_MAX_AXIS], ms[NA_MAX_AXIS], be[NA_MAX_AXIS], ce[NA_MAX_AXIS], bh[NA_MAX_AXIS], ch[NA_MAX_AXIS],
            ked[NA_MAX_AXIS], khd[NA_MAX_AXIS];
        memset(prof, 0, sizeof(float) * 3 * P_COUNT * ps);
        for (int a = 0; a < 3; a++) {
            profile_axis(ph->flavor, n3[a], d3[a], nc, ph->cmax, ph->dt, a == 0, cc, es, ms, be, ce, bh, ch, ked, khd);
            float *p = prof + (size_t)a * P_COUNT * ps;
            for (int i = 0; i < n3[a]; i++) {
                p[P_ESH * ps + i] = (float)(es[i] * 0.5);
                p[P_MSH * ps + i] = (float)(ms[i] * 0.5);
                p[P_BE * ps + i] = (float)be[i];
                p[P_CED * ps + i] = (float)(ce[i] / d3[a]);
                p[P_BH * ps + i] = (float)bh[i];
                p[P_CHD * ps + i] = (float)(ch[i] / d3[a]);
                p[P_IKED * ps + i] = (float)(1.0 / ked[i]);
                p[P_IKHD * ps + i] = (float)(1.0 / khd[i]);
            }
        }
    }
    const int px = (nx + 31) / 32 * 32;
    const long long plane = (long long)px * ny, fshot = plane * nz;
    size_t pe[3], ph_[3];
    for (int a = 0; a < 3; a++) {
        const Slab *gr[2] = {&su.se[a], &su.sh[a]};
        for (int t = 0; t < 2; t++) {
            const Slab &s = *gr[t];
            const size_t n = a == 0 ? (size_t)nz * ny * s.width : (a == 1 ? (size_t)nz * s.width * px : (size_t)s.width * ny * px);
            (t == 0 ? pe : ph_)[a] = n;
        }
    }
    // ---- scratch layout
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off = align256(off + bytes); return o; };
    const size_t o_prof = take(sizeof(float) * 3 * P_COUNT * ps);
    const size_t o_tmap = take(sizeof(TileMap));
    const size_t o_m = take(sizeof(float) * fshot);
    size_t o_f[6];
    for (int c = 0; c < 6; c++) o_f[c] = take(sizeof(float) * fshot);
    size_t o_pe[3][2], o_ph[3][2];
    for (int a = 0; a < 3; a++)
        for (int w = 0; w < 2; w++) {
            o_pe[a][w] = take(sizeof(float) * pe[a]);
            o_ph[a][w] = take(sizeof(float) * ph_[a]);
        }
    const size_t o_pts = take(sizeof(SrcPoint) * npoint);
    const size_t o_cell = take(sizeof(long long) * npoint);
    const size_t o_amp = take(sizeof(double) * npoint);
    const size_t o_roff = take(sizeof(long long) * nrec);
    const size_t o_rcomp = take(sizeof(int) * nrec);
    const size_t o_rish = take(nrec);
    const size_t o_om = take(sizeof(double) * nf);
    const size_t o_tr = take(sizeof(float) * (size_t)nrec * nt);
    const size_t o_step = take(sizeof(int));
    const size_t need = off;
    if (need > MITTET_NOALLOC_SCRATCH_BYTES)
        return na_fail(MITTET_ERR_INVALID_ARG, "this solve needs %zu bytes of scratch; the static array holds %u", need,
                       (unsigned)MITTET_NOALLOC_SCRATCH_BYTES);

    // ---- small descriptor arrays, staged on the stack
    SrcPoint sp[NA_MAX_POINTS];
    long long scell[NA_MAX_POINTS];
    double samp[NA_MAX_POINTS];
    bool has_mag = false, has_ele = false;
    for (int q = 0; q < npoint; q++) {
        const mittet_point_source &p = pts[q];
        if (p.shot != 0) return na_fail(MITTET_ERR_INVALID_ARG, "point %d: this entry point solves shot 0 only", q);
        if (p.ix < 1 || p.ix > nx || p.iy < 1 || p.iy > ny || p.iz < 1 || p.iz > nz)
            return na_fail(MITTET_ERR_INVALID_ARG, "point %d outside the grid", q);
        if (p.comp < 0 || p.comp > 5 || (p.kind != MITTET_SRC_MAGNETIC && p.kind != MITTET_SRC_ELECTRIC) ||
            !std::isfinite(p.amp))
            return na_fail(MITTET_ERR_INVALID_ARG, "point %d: bad component, kind or amplitude", q);
        sp[q].off = ((long long)(p.iz - 1) * ny + (p.iy - 1)) * px + (p.ix - 1);
        sp[q].comp = p.comp;
        sp[q].kind = p.kind;
        sp[q].g = 0.0;
        scell[q] = ((long long)(p.iz - 1) * ny + (p.iy - 1)) * nx + (p.ix - 1);
        samp[q] = p.amp;
        has_mag |= p.kind == MITTET_SRC_MAGNETIC;
        has_ele |= p.kind == MITTET_SRC_ELECTRIC;
    }
    long long roff[NA_MAX_REC];
    int rcomp[NA_MAX_REC];
    unsigned char rish[NA_MAX_REC];
    for (int r = 0; r < nrec; r++) {
        const mittet_receiver &q = rec[r];
        if (q.ix < 1 || q.ix > nx || q.iy < 1 || q.iy > ny || q.iz < 1 || q.iz > nz || q.comp < 0 || q.comp > 5)
            return na_fail(MITTET_ERR_INVALID_ARG, "receiver %d outside the grid or bad component", r);
        roff[r] = ((long long)(q.iz - 1) * ny + (q.iy - 1)) * px + (q.ix - 1);
        rcomp[r] = q.comp;
        rish[r] = q.comp >= 3;
    }
    for (int f = 0; f < nf; f++)
        if (!(omega[f] >= 0) || !std::isfinite(omega[f])) return na_fail(MITTET_ERR_INVALID_ARG, "omega[%d] invalid", f);
    TileMap tm;
    memset(&tm, 0, sizeof(tm));
    tm.nbox = 1;
    tm.zc = NA_ZC;
    tm.pbox[kParts] = 1;  // one general box: part 4 (edges body) covers the grid
    tm.kind[0] = 7;
    tm.hi[0][0] = nx; tm.hi[0][1] = ny; tm.hi[0][2] = nz;
    tm.ntx[0] = (nx + NA_BX * NA_VX - 1) / (NA_BX * NA_VX);
    tm.nty[0] = (ny + NA_BY - 1) / NA_BY;
    tm.start[1] = tm.ntx[0] * tm.nty[0] * ((nz + NA_ZC - 1) / NA_ZC);

    // ---- device work, all on the caller's stream, all inside the array
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return na_fail(MITTET_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    unsigned char *base = nullptr;
    int rc = na_scratch(dev, &base);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
#define NA_CK(call)                                                                                     \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) return na_fail(MITTET_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)
    NA_CK(cudaMemcpyAsync(base + o_prof, prof, sizeof(float) * 3 * P_COUNT * ps, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(base + o_tmap, &tm, sizeof(tm), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(base + o_pts, sp, sizeof(SrcPoint) * npoint, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(base + o_cell, scell, sizeof(long long) * npoint, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(base + o_amp, samp, sizeof(double) * npoint, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(base + o_roff, roff, sizeof(long long) * nrec, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(base + o_rcomp, rcomp, sizeof(int) * nrec, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(base + o_rish, rish, nrec, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(base + o_om, omega, sizeof(double) * nf, cudaMemcpyHostToDevice, st));
    // zero what must start at zero: model padding, fields, psi, traces, step counter
    NA_CK(cudaMemsetAsync(base + o_m, 0, sizeof(float) * fshot, st));
    for (int c = 0; c < 6; c++) NA_CK(cudaMemsetAsync(base + o_f[c], 0, sizeof(float) * fshot, st));
    for (int a = 0; a < 3; a++)
        for (int w = 0; w < 2; w++) {
            NA_CK(cudaMemsetAsync(base + o_pe[a][w], 0, sizeof(float) * pe[a], st));
            NA_CK(cudaMemsetAsync(base + o_ph[a][w], 0, sizeof(float) * ph_[a], st));
        }
    NA_CK(cudaMemsetAsync(base + o_tr, 0, sizeof(float) * (size_t)nrec * nt, st));
    NA_CK(cudaMemsetAsync(base + o_step, 0, sizeof(int), st));

    na_model_kernel<<<256, 256, 0, st>>>(sigma_dev, nx, ny, nz, px, 2.0 * ph->omega0 * ph->dt, (float *)(base + o_m));
    na_gain_kernel<<<1, NA_MAX_POINTS, 0, st>>>((SrcPoint *)(base + o_pts), sigma_dev, (const long long *)(base + o_cell),
                                                (const double *)(base + o_amp), npoint, ph->dt, ph->omega0, ph->mu0,
                                                g->dx * g->dy * g->dz);

    PhaseArgs<float> pa[2];
    for (int t = 0; t < 2; t++) {
        PhaseArgs<float> &a = pa[t];
        memset(&a, 0, sizeof(a));
        for (int c = 0; c < 6; c++) a.f[c] = a.fo[c] = (float *)(base + o_f[c]);
        for (int ax = 0; ax < 3; ax++)
            for (int w = 0; w < 2; w++) a.psi[ax][w] = (float *)(base + (t == 0 ? o_pe[ax][w] : o_ph[ax][w]));
        a.m = (const float *)(base + o_m);
        a.dtmu = nullptr;
        a.dtmu0 = (float)(ph->dt / ph->mu0);
        a.prof = (const float *)(base + o_prof);
        a.nmax = ps;
        a.nx = nx; a.ny = ny; a.nz = nz; a.px = px;
        a.plane = plane;
        a.fshot = fshot;
        for (int ax = 0; ax < 3; ax++) {
            const Slab &s = t == 0 ? su.se[ax] : su.sh[ax];
            a.pshot[ax] = (long long)(t == 0 ? pe[ax] : ph_[ax]);
            a.slab[ax].nlo = s.nlo; a.slab[ax].nhi = s.nhi; a.slab[ax].flo = s.flo; a.slab[ax].fhi = s.fhi;
            a.slab[ax].width = s.width;
            a.slab[ax].fofs = s.fofs;
            for (int b = 0; b < 3; b++) {
                a.slab[ax].other.lo[b] = s.other.lo[b];
                a.slab[ax].other.hi[b] = s.other.hi[b];
                a.upd[ax].lo[b] = su.upd[(t == 0 ? 0 : 3) + ax].lo[b];
                a.upd[ax].hi[b] = su.upd[(t == 0 ? 0 : 3) + ax].hi[b];
            }
        }
        a.c1 = (float)ph->c1;
        a.c2 = (float)ph->c2;
        a.c2t = (float)(ph->psi_hyx_typo ? ph->c2 : ph->c1);
        a.sgn = (float)(t == 0 ? ph->e_sign : ph->h_sign);
        a.ik[0] = (float)(1.0 / g->dx);
        a.ik[1] = (float)(1.0 / g->dy);
        a.ik[2] = (float)(1.0 / g->dz);
        a.ring = nullptr;
        a.ring_k = 0;
        a.d_step = (const int *)(base + o_step);
    }
    InjectArgs<float> ia;
    memset(&ia, 0, sizeof(ia));
    for (int c = 0; c < 6; c++) ia.f[c] = (float *)(base + o_f[c]);
    ia.pts = (const SrcPoint *)(base + o_pts);
    ia.npts = npoint;
    ia.wave = wavelet_dev;
    ia.d_step = (const int *)(base + o_step);
    InjectArgs<float> ia_m = ia, ia_e = ia;
    ia_m.kind = 0;
    ia_e.kind = 1;
    SampleArgs<float> sa;
    memset(&sa, 0, sizeof(sa));
    for (int c = 0; c < 6; c++) sa.f[c] = (const float *)(base + o_f[c]);
    sa.rec_off = (const long long *)(base + o_roff);
    sa.rec_comp = (const int *)(base + o_rcomp);
    sa.nrec = nrec;
    sa.nshot = 1;
    sa.fshot = fshot;
    sa.traces = (float *)(base + o_tr);
    sa.nt = nt;
    sa.d_step = (int *)(base + o_step);
    const TileMap *dtm = (const TileMap *)(base + o_tmap);
    const dim3 grid(tm.start[1], 1), block(NA_BX, NA_BY);
    for (int s = 0; s < nt; s++) {
        if (has_mag) inject_kernel<float><<<1, 128, 0, st>>>(ia_m);
        e_part_kernel<float, NA_VX, NA_BX, NA_BY, 7><<<grid, block, 0, st>>>(pa[0], dtm, 0, 0, 1);
        if (has_ele) inject_kernel<float><<<1, 128, 0, st>>>(ia_e);
        h_part_kernel<float, NA_VX, NA_BX, NA_BY, 7><<<grid, block, 0, st>>>(pa[1], dtm, 0, 0, 1);
        sample_kernel<float><<<1, 1024, 0, st>>>(sa);
    }
    trace_dft_kernel<float><<<nf, 256, 0, st>>>((const float *)(base + o_tr), nrec, nt, (const double *)(base + o_om), nf,
                                                ph->dt, ph->omega0, (const unsigned char *)(base + o_rish), nrec,
                                                h_factor ? 1 : 0, (double2 *)rec_fd_dev);
    NA_CK(cudaGetLastError());
#undef NA_CK
    return MITTET_OK;
}
