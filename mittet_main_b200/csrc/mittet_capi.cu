// mittet_capi.cu -- the C ABI declared in include/mittet.h.
//
// A handle owns: the CPML profiles and ranges (host set-up), the resident
// model (m = 2 w0 dt / sigma, optional dt/mu), the batched fields and compact
// psi slabs of all shots, the receiver traces, and (optionally) the
// full-volume DFT ring and accumulators.  mittet_forward() runs the time loop
// as one CUDA graph of G steps replayed nt/G times, then the f_to_d
// transform of the receiver traces.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <array>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "../../include/mittet.h"
#include "kernels.cuh"
#include "persistent.cuh"
#include "tma_interior.cuh"
#include "adjoint.cuh"
#include "setup_host.h"

using namespace mittet;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(call)                                                                                     \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) {                                                                     \
            if (e_ == cudaErrorMemoryAllocation) {                                                   \
                cudaGetLastError();                                                                  \
                return fail(MITTET_ERR_OOM, "%s: %s", #call, cudaGetErrorString(e_));                \
            }                                                                                        \
            return fail(MITTET_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
        }                                                                                            \
    } while (0)

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    cudaError_t ensure(size_t b) {
        if (b <= bytes && p) return cudaSuccess;
        release();
        cudaError_t e = cudaMalloc(&p, b ? b : 16);
        if (e == cudaSuccess) bytes = b;
        return e;
    }
    template <typename T>
    T *as() const { return (T *)p; }
};

DBox to_dbox(const Box &b) {
    DBox d;
    for (int a = 0; a < 3; a++) { d.lo[a] = b.lo[a]; d.hi[a] = b.hi[a]; }
    return d;
}
DSlab to_dslab(const Slab &s) {
    DSlab d;
    d.nlo = s.nlo; d.nhi = s.nhi; d.flo = s.flo; d.fhi = s.fhi; d.width = s.width; d.fofs = s.fofs;
    d.other = to_dbox(s.other);
    return d;
}

}  // namespace

namespace mittet {
// Lets the other translation unit of the library report through mittet_last_error.
void set_last_error(const char *msg) { g_err = msg; }
}  // namespace mittet

struct mittet_handle_s {
    mittet_grid g{};
    mittet_phys ph{};
    Setup su;
    int px = 0;
    long long plane = 0, fshot = 0;
    bool fp64 = false;
    size_t esz = 4;
    cudaStream_t st = nullptr;
    // side streams and events of the concurrent phase parts (fork/join,
    // captured as parallel branches of the step graph)
    cudaStream_t pst[kParts] = {nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[kParts] = {nullptr};

    DevBuf prof, m, dtmu;
    bool has_model = false, has_mu = false;
    std::vector<double> sigma_h;  // host copy of the model (source scaling)
    std::vector<double> mu_h;

    int nshot = 0;
    std::vector<mittet_point_source> pts;
    DevBuf d_pts;
    int npts = 0;
    bool has_mag = false, has_ele = false;

    int nt_wave = -1;
    DevBuf wave;

    int nrec = 0;
    std::vector<mittet_receiver> recs;
    DevBuf rec_off, rec_comp, rec_is_h;

    std::vector<double> omega;
    int hfac = 1;
    DevBuf d_omega;

    uint32_t vmask = 0;
    int ring_k = kFlushRing;  // ring depth = steps per graph and per volume-DFT flush
    int var_e[kParts] = {0};   // stencil variant (index into variants<T>()) of the interior,
    int var_h[kParts] = {0};   // x/y/z face and edge launches of each phase;
                               // var[0] = -1 - c selects TMA interior config c
    TmaMaps tma_maps[2];       // tensor maps of the E and H interior (current buffers)
    int tma_spin = kMbarSpinLimit;  // polls before a TMA wait gives up (MITTET_TMA_SPIN_LIMIT)
    int tma_nown[2] = {0, 0};
    bool tma_ok = false;
    int ibox[2][6] = {{0}};    // interior box of each phase: lo xyz, hi xyz
    bool has_ibox[2] = {false, false};
    int ldg_int[2] = {0, 0};   // best plain-load interior variant of each phase
    int merge_b[2] = {-1, -1}; // variant of the merged boundary launch of each phase (-1: four part launches)
    int band[2] = {0, 0};      // z planes per band of the interior + x-face band launch (0: part launches)
    // forward layout of each phase: kLayoutParts, kLayoutOneBox (the grid as
    // one general box) or kLayoutCoreRows (interior and x faces as parts, the
    // y- and z-slab rows whole as general boxes)
    int layout[2] = {0, 0};
    int tm_layout[2] = {0, 0};  // the layout the uploaded tile maps have
    DevBuf tmaps;              // TileMap per (variant, phase), device copy
    std::vector<TileMap> tmaps_host;
    DevBuf adj_tmaps;          // one-cell tile maps (32 x 8 x 1) of the E and H phase: the adjoint own kernels
    TileMap adj_tm_host[2];
    int ptile[64][kParts + 1] = {{0}};  // per (variant, phase): part p is tiles [ptile[p], ptile[p+1])
    bool tuned = false;
    DevBuf ring, acc;
    DevBuf stage_sigma, stage_mu;  // FP64 model stage of uploads (kept: a freed buffer would synchronise the device)
    bool model_dev = false;        // the model came from device memory: sigma_h / mu_h are empty, the stage holds it
    std::vector<double> wt_host;  // volume-DFT weights [n][f] (re, im)
    // Work buffers of mittet_gradient, kept for the next call on this handle
    // (an FWI loop calls it once per iteration; allocating and freeing ~100
    // GB each time costs up to a second).  mittet_release_gradient_buffers
    // frees them.
    struct GradBufs {
        DevBuf obs, R, mis, asrc, asp, fl[6], pe[3][2], pH[3][2], hist, ck, lam[6], lpe[3][2], lph[3][2], mu[7],
            gacc, gred, gpts;
        template <typename F>
        void each(F f) {
            for (DevBuf *b : {&obs, &R, &mis, &asrc, &asp, &hist, &ck, &gacc, &gred, &gpts}) f(*b);
            for (int c = 0; c < 6; c++) { f(fl[c]); f(lam[c]); }
            for (int c = 0; c < 7; c++) f(mu[c]);
            for (int a = 0; a < 3; a++)
                for (int w = 0; w < 2; w++) { f(pe[a][w]); f(pH[a][w]); f(lpe[a][w]); f(lph[a][w]); }
        }
        size_t held() {
            size_t n = 0;
            each([&](DevBuf &b) { n += b.bytes; });
            return n;
        }
        void release() {
            each([](DevBuf &b) { b.release(); });
        }
    } gb;

    DevBuf fields[6], psiE[3][2], psiH[3][2];
    int alloc_shots = -1;
    DevBuf traces, spectra, d_step, d_flag;
    int last_nt = 0;
    int64_t launches = 0;

    // persistent launch (persistent.cuh): the stencil variant whose tile
    // maps and thread shape it uses (-1: the stepped graph of part kernels),
    // whether the choice was made for the current tuning, its grid size and
    // barrier words
    int persist_vi = -1;
    bool persist_decided = false;
    int persist_grid = 0;
    DevBuf bar;

    // cached CUDA graph of G steps
    cudaGraphExec_t gexec = nullptr;
    int graph_steps = 0;
    int64_t graph_launches = 0;
    int graph_key_shots = -1;
    long long graph_key = -1;
};

namespace {

int set_device(mittet_handle *h) {
    CK(cudaSetDevice(h->ph.device));
    return MITTET_OK;
}

size_t psi_elems(const mittet_handle *h, const Slab &s, int axis) {
    const size_t ny = h->g.ny, nz = h->g.nz, px = h->px;
    if (axis == 0) return nz * ny * (size_t)s.width;
    if (axis == 1) return nz * (size_t)s.width * px;
    return (size_t)s.width * ny * px;
}

void drop_graph(mittet_handle *h) {
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    h->gexec = nullptr;
    h->graph_steps = 0;
    h->tuned = false;  // the shot count or ring may have changed
    h->persist_decided = false;
}

int ensure_state(mittet_handle *h) {
    const int ns = h->nshot;
    if (h->alloc_shots != ns) {
        drop_graph(h);
        const size_t fbytes = (size_t)ns * h->fshot * h->esz;
        for (int c = 0; c < 6; c++) CK(h->fields[c].ensure(fbytes));
        for (int a = 0; a < 3; a++)
            for (int w = 0; w < 2; w++) {
                CK(h->psiE[a][w].ensure((size_t)ns * psi_elems(h, h->su.se[a], a) * h->esz));
                CK(h->psiH[a][w].ensure((size_t)ns * psi_elems(h, h->su.sh[a], a) * h->esz));
            }
        h->alloc_shots = ns;
    }
    for (int c = 0; c < 6; c++) CK(cudaMemsetAsync(h->fields[c].p, 0, (size_t)ns * h->fshot * h->esz, h->st));
    for (int a = 0; a < 3; a++)
        for (int w = 0; w < 2; w++) {
            CK(cudaMemsetAsync(h->psiE[a][w].p, 0, (size_t)ns * psi_elems(h, h->su.se[a], a) * h->esz, h->st));
            CK(cudaMemsetAsync(h->psiH[a][w].p, 0, (size_t)ns * psi_elems(h, h->su.sh[a], a) * h->esz, h->st));
        }
    return MITTET_OK;
}

template <typename T>
PhaseArgs<T> phase_args(mittet_handle *h, bool e_phase) {
    PhaseArgs<T> a;
    memset(&a, 0, sizeof(a));
    for (int c = 0; c < 6; c++) a.f[c] = a.fo[c] = h->fields[c].as<T>();
    for (int ax = 0; ax < 3; ax++)
        for (int w = 0; w < 2; w++) a.psi[ax][w] = (e_phase ? h->psiE : h->psiH)[ax][w].as<T>();
    a.m = h->m.as<T>();
    a.dtmu = h->has_mu ? h->dtmu.as<T>() : nullptr;
    a.dtmu0 = (T)(h->ph.dt / h->ph.mu0);
    a.prof = h->prof.as<T>();
    a.nmax = h->su.nmax;
    a.nx = h->g.nx; a.ny = h->g.ny; a.nz = h->g.nz; a.px = h->px;
    a.plane = h->plane; a.fshot = h->fshot;
    for (int ax = 0; ax < 3; ax++) {
        const Slab &s = e_phase ? h->su.se[ax] : h->su.sh[ax];
        a.pshot[ax] = (long long)psi_elems(h, s, ax);
        a.slab[ax] = to_dslab(s);
        a.upd[ax] = to_dbox(h->su.upd[(e_phase ? 0 : 3) + ax]);
    }
    a.c1 = (T)h->ph.c1;
    a.c2 = (T)h->ph.c2;
    a.c2t = (T)(h->ph.psi_hyx_typo ? h->ph.c2 : h->ph.c1);
    a.sgn = (T)(e_phase ? h->ph.e_sign : h->ph.h_sign);
    a.ik[0] = (T)(1.0 / h->g.dx);
    a.ik[1] = (T)(1.0 / h->g.dy);
    a.ik[2] = (T)(1.0 / h->g.dz);
    a.d_step = h->d_step.as<int>();
    if (e_phase && h->vmask) {
        a.ring = h->ring.as<T>();
        a.ring_k = h->ring_k;
        a.vmask = (int)h->vmask;
        a.ring_comp = ring_comp_of((long long)h->nshot * h->fshot);
    }
    return a;
}

// Stencil variants (VX x cells per thread, BX x BY threads, ZC z planes per
// tile, BZ threads along z: 0 = each thread marches ZC planes) the autotuner
// picks from; k[phase][part] are the kernels of the five bodies.
template <typename T>
using PartKernel = void (*)(PhaseArgs<T>, const TileMap *, int, int, int);
template <typename T>
struct Variant {
    int vx, bx, by, zc, bz;
    PartKernel<T> k[2][kParts];
};

#define MITTET_PARTS(PH, T, vx, bx, by, bz)                                                            \
    {PH##_part_kernel<T, vx, bx, by, 0, bz>, PH##_part_kernel<T, vx, bx, by, 1, bz>,                   \
     PH##_part_kernel<T, vx, bx, by, 2, bz>, PH##_part_kernel<T, vx, bx, by, 4, bz>,                   \
     PH##_part_kernel<T, vx, bx, by, 7, bz>}

template <typename T>
const std::vector<Variant<T>> &variants();

// the handle's ptile table holds 64 (variant, phase) slots
#define MITTET_COUNT(vx, bx, by, zc, bz) +1
static_assert(0 MITTET_STENCIL_VARIANTS_F32(MITTET_COUNT) <= 32 && 0 MITTET_STENCIL_VARIANTS_F64(MITTET_COUNT) <= 32,
              "more stencil variants than the ptile table holds");
#undef MITTET_COUNT

template <>
const std::vector<Variant<float>> &variants<float>() {
    static const std::vector<Variant<float>> v = {
#define MITTET_X(vx, bx, by, zc, bz) \
    {vx, bx, by, zc, bz, {MITTET_PARTS(e, float, vx, bx, by, bz), MITTET_PARTS(h, float, vx, bx, by, bz)}},
        MITTET_STENCIL_VARIANTS_F32(MITTET_X)
#undef MITTET_X
    };
    return v;
}
template <>
const std::vector<Variant<double>> &variants<double>() {
    static const std::vector<Variant<double>> v = {
#define MITTET_X(vx, bx, by, zc, bz) \
    {vx, bx, by, zc, bz, {MITTET_PARTS(e, double, vx, bx, by, bz), MITTET_PARTS(h, double, vx, bx, by, bz)}},
        MITTET_STENCIL_VARIANTS_F64(MITTET_X)
#undef MITTET_X
    };
    return v;
}

// Interior box of one phase: per axis, the run of indices around the centre
// where the general body reduces to the plain update (no CPML profile, no
// psi slab, inside every component's update range, derivative defined).
void interior_box(const mittet_handle *h, bool e, int lo[3], int hi[3]) {
    const Setup &su = h->su;
    const int n3[3] = {h->g.nx, h->g.ny, h->g.nz};
    const double d3[3] = {h->g.dx, h->g.dy, h->g.dz};
    for (int a = 0; a < 3; a++) {
        const int n = n3[a];
        const Slab &sl = e ? su.se[a] : su.sh[a];
        auto ok = [&](int v) {
            const double sig = prof_at(su, a, e ? P_ESH : P_MSH, v);
            const double ik = prof_at(su, a, e ? P_IKED : P_IKHD, v);
            if (sig != 0.0 || ik != 1.0 / d3[a]) return false;
            if ((v >= sl.nlo && v < sl.nhi) || (v >= sl.flo && v < sl.fhi)) return false;
            for (int c = 0; c < 3; c++) {
                const Box &b = su.upd[(e ? 0 : 3) + c];
                if (v < b.lo[a] || v >= b.hi[a]) return false;
            }
            return e ? (v >= 2 && v + 1 < n) : (v >= 1 && v + 2 < n);
        };
        const int mid = n / 2;
        if (!ok(mid)) { lo[a] = hi[a] = 0; continue; }
        int l = mid, r = mid + 1;
        while (l - 1 >= 0 && ok(l - 1)) l--;
        while (r < n && ok(r)) r++;
        lo[a] = l;
        hi[a] = r;
    }
}

enum Layout { kLayoutParts = 0, kLayoutOneBox = 1, kLayoutCoreRows = 2 };

TileMap make_tilemap(const mittet_handle *h, bool e, int vx, int bx, int by, int zc, int layout = kLayoutParts) {
    TileMap t;
    memset(&t, 0, sizeof(t));
    t.zc = zc;
    const int nx = h->g.nx, ny = h->g.ny, nz = h->g.nz;
    const int TX = bx * vx;
    int lo[3], hi[3];
    interior_box(h, e, lo, hi);
    // The boxes do not depend on the variant.  x box edges are multiples of
    // 32 cells, so every box owns whole 128-byte lines of each row (rows
    // start 128-byte aligned): a 16-cell CPML slab sharing its lines with
    // interior cells that another launch reads makes DRAM move each line
    // twice (measured: 16-cell row segments run at 2.6 TB/s, 32-cell ones at
    // 5.0).  The general x body then also covers the interior cells up to the
    // next multiple of 32.  Grids whose interior would keep less than 64
    // cells of x that way use multiples of 4 (every vector width divides
    // them).  Partial tiles in x and y are masked and the last z chunk of a
    // box is cut at the box edge.
    // MITTET_X_ALIGN_MIN: the narrowest line-aligned interior kept (default 64 cells)
    static const int align_min = [] {
        const char *v = std::getenv("MITTET_X_ALIGN_MIN");
        return v ? std::max(1, std::atoi(v)) : 64;
    }();
    int X0 = (lo[0] + 31) / 32 * 32, X1 = hi[0] / 32 * 32;
    if (X1 - X0 < align_min) {
        X0 = (lo[0] + 3) / 4 * 4;
        X1 = hi[0] / 4 * 4;
    }
    const int Y0 = lo[1], Y1 = hi[1];
    const int Z0 = lo[2], Z1 = hi[2];
    auto add = [&](int kind, int x0, int y0, int z0, int x1, int y1, int z1) {
        if (x1 <= x0 || y1 <= y0 || z1 <= z0) return;
        const int q = t.nbox++;
        t.kind[q] = kind;
        t.lo[q][0] = x0; t.lo[q][1] = y0; t.lo[q][2] = z0;
        t.hi[q][0] = x1; t.hi[q][1] = y1; t.hi[q][2] = z1;
        t.ntx[q] = (x1 - x0 + TX - 1) / TX;
        t.nty[q] = (y1 - y0 + by - 1) / by;
        const int nzt = (z1 - z0 + zc - 1) / zc;
        t.start[q + 1] = t.start[q] + t.ntx[q] * t.nty[q] * nzt;
    };
    // kLayoutOneBox: the whole grid as one general box (part 4), the layout
    // the autotuner may choose for grids that are mostly CPML slab
    if (X1 > X0 && Y1 > Y0 && Z1 > Z0 && layout == kLayoutCoreRows) {
        t.pbox[0] = t.nbox;
        add(0, X0, Y0, Z0, X1, Y1, Z1);
        t.pbox[1] = t.nbox;
        add(1, 0, Y0, Z0, X0, Y1, Z1);   // x faces
        add(1, X1, Y0, Z0, nx, Y1, Z1);
        t.pbox[2] = t.pbox[3] = t.pbox[4] = t.nbox;
        add(7, 0, 0, 0, nx, ny, Z0);     // z-slab planes, whole
        add(7, 0, 0, Z1, nx, ny, nz);
        add(7, 0, 0, Z0, nx, Y0, Z1);    // y-slab rows of the interior z range, whole
        add(7, 0, Y1, Z0, nx, ny, Z1);
    } else if (X1 > X0 && Y1 > Y0 && Z1 > Z0 && layout != kLayoutOneBox) {
        t.pbox[0] = t.nbox;
        add(0, X0, Y0, Z0, X1, Y1, Z1);
        t.pbox[1] = t.nbox;
        add(1, 0, Y0, Z0, X0, Y1, Z1);   // x faces
        add(1, X1, Y0, Z0, nx, Y1, Z1);
        t.pbox[2] = t.nbox;
        add(2, X0, 0, Z0, X1, Y0, Z1);   // y faces
        add(2, X0, Y1, Z0, X1, ny, Z1);
        t.pbox[3] = t.nbox;
        add(4, X0, Y0, 0, X1, Y1, Z0);   // z faces
        add(4, X0, Y0, Z1, X1, Y1, nz);
        t.pbox[4] = t.nbox;
        const int zr[2][2] = {{0, Z0}, {Z1, nz}};
        for (int zz = 0; zz < 2; zz++) {  // rings around the z faces
            const int za = zr[zz][0], zb = zr[zz][1];
            add(7, 0, 0, za, nx, Y0, zb);
            add(7, 0, Y1, za, nx, ny, zb);
            add(7, 0, Y0, za, X0, Y1, zb);
            add(7, X1, Y0, za, nx, Y1, zb);
        }
        add(7, 0, 0, Z0, X0, Y0, Z1);     // vertical edges
        add(7, X1, 0, Z0, nx, Y0, Z1);
        add(7, 0, Y1, Z0, X0, ny, Z1);
        add(7, X1, Y1, Z0, nx, ny, Z1);
    } else {
        add(7, 0, 0, 0, nx, ny, nz);
    }
    t.pbox[kParts] = t.nbox;  // without an interior every box is part 4 (pbox[0..4] = 0)
    return t;
}

template <typename T>
int upload_tilemaps(mittet_handle *h) {
    const auto &vs = variants<T>();
    std::vector<TileMap> maps(2 * vs.size());
    for (size_t v = 0; v < vs.size(); v++) {
        maps[2 * v] = make_tilemap(h, true, vs[v].vx, vs[v].bx, vs[v].by, vs[v].zc, h->layout[0]);
        maps[2 * v + 1] = make_tilemap(h, false, vs[v].vx, vs[v].bx, vs[v].by, vs[v].zc, h->layout[1]);
        for (int p = 0; p < 2; p++) {
            const TileMap &t = maps[2 * v + p];
            for (int q = 0; q <= kParts; q++) h->ptile[2 * v + p][q] = t.start[t.pbox[q]];
        }
    }
    h->tm_layout[0] = h->layout[0];
    h->tm_layout[1] = h->layout[1];
    for (int p = 0; p < 2; p++) {  // the interior box of the partitioned layout (the adjoint's boxes too)
        const TileMap t = make_tilemap(h, p == 0, vs[0].vx, vs[0].bx, vs[0].by, vs[0].zc);
        h->has_ibox[p] = t.pbox[1] > t.pbox[0];
        for (int q = 0; q < 3; q++) {
            h->ibox[p][q] = t.lo[0][q];
            h->ibox[p][3 + q] = t.hi[0][q];
        }
    }
    h->tmaps_host = maps;
    CK(h->tmaps.ensure(maps.size() * sizeof(TileMap)));
    CK(cudaMemcpy(h->tmaps.p, maps.data(), maps.size() * sizeof(TileMap), cudaMemcpyHostToDevice));
    drop_graph(h);
    h->adj_tm_host[0] = make_tilemap(h, true, 1, 32, 8, 1);
    h->adj_tm_host[1] = make_tilemap(h, false, 1, 32, 8, 1);
    CK(h->adj_tmaps.ensure(2 * sizeof(TileMap)));
    CK(cudaMemcpy(h->adj_tmaps.p, h->adj_tm_host, 2 * sizeof(TileMap), cudaMemcpyHostToDevice));
    return MITTET_OK;
}

// The adjoint own kernels of one phase over its five parts (one-cell tiles,
// the forward's boxes, so each part drops the CPML logic of the axes it is
// interior along), concurrently on the part streams like a forward phase.
template <typename T>
void launch_adj_own(mittet_handle *h, bool e, const AdjArgs<T> &a, int nshot) {
    using K = void (*)(AdjArgs<T>, const TileMap *, int, int, int);
    static const K ke[kParts] = {adj_e_own_part_kernel<T, 0>, adj_e_own_part_kernel<T, 1>,
                                 adj_e_own_part_kernel<T, 2>, adj_e_own_part_kernel<T, 4>,
                                 adj_e_own_part_kernel<T, 7>};
    static const K kh[kParts] = {adj_h_own_part_kernel<T, 0>, adj_h_own_part_kernel<T, 1>,
                                 adj_h_own_part_kernel<T, 2>, adj_h_own_part_kernel<T, 4>,
                                 adj_h_own_part_kernel<T, 7>};
    const TileMap &tm = h->adj_tm_host[e ? 0 : 1];
    const TileMap *dtm = h->adj_tmaps.as<TileMap>() + (e ? 0 : 1);
    cudaEventRecord(h->ev_fork, h->st);
    for (int p = 1; p < kParts; p++) cudaStreamWaitEvent(h->pst[p], h->ev_fork, 0);
    for (int p = kParts - 1; p >= 0; p--) {
        const int first = tm.start[tm.pbox[p]], last = tm.start[tm.pbox[p + 1]];
        if (last <= first) continue;
        cudaStream_t st = p == 0 ? h->st : h->pst[p];
        (e ? ke : kh)[p]<<<dim3(last - first, nshot), dim3(32, 8), 0, st>>>(a, dtm, first, tm.pbox[p], tm.pbox[p + 1]);
    }
    for (int p = 1; p < kParts; p++) {
        cudaEventRecord(h->ev_join[p], h->pst[p]);
        cudaStreamWaitEvent(h->st, h->ev_join[p], 0);
    }
}

// ------------------------------------------------- TMA-staged interior
// Configurations of interior_tma_kernel the autotuner may pick for part 0:
// tile TX x TY (TX = 64 FP32 / 32 FP64 cells, TY = 8 rows), ring depth of
// the E and H phases, z planes per CTA.
template <typename T>
struct TmaShape {
    static constexpr int TX = sizeof(T) == 4 ? 64 : 32, TY = 8;
};

template <typename T>
struct TmaCfg {
    int zc;
    bool own_smem;  // own-cell tiles staged by TMA (else loaded by the threads)
    int se, sh;     // ring depth of the E and H kernels
    void (*ek)(PhaseArgs<T>, TmaTiling, TmaMaps, int, int *);
    void (*hk)(PhaseArgs<T>, TmaTiling, TmaMaps, int, int *);
    size_t smem(bool e) const {
        using S = TmaShape<T>;
        return own_smem ? TmaStage<T, S::TX, S::TY, 4>::bytes(e ? se : sh)
                        : TmaStage<T, S::TX, S::TY, 0>::bytes(e ? se : sh);
    }
};

template <typename T>
const std::vector<TmaCfg<T>> &tma_cfgs() {
    constexpr int TX = TmaShape<T>::TX, TY = TmaShape<T>::TY;
#define MITTET_TMA(ZC, OWN, SE, SH) \
    {ZC, OWN, SE, SH, interior_tma_kernel<T, TX, TY, SE, true, OWN>, interior_tma_kernel<T, TX, TY, SH, false, OWN>}
    static const std::vector<TmaCfg<T>> v = {
        MITTET_TMA(8, true, 4, 5),  MITTET_TMA(16, true, 4, 5),  MITTET_TMA(32, true, 4, 5),
        MITTET_TMA(8, false, 6, 6), MITTET_TMA(16, false, 6, 6), MITTET_TMA(32, false, 6, 6),
    };
#undef MITTET_TMA
    return v;
}

PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// 3-D map of one padded field array [nzs][ny][px] with a bx x by x 1 box.
bool encode_map(CUtensorMap *m, const void *base, bool fp64, int px, int ny, long long nzs, int bx, int by) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = tma_encoder();
    if (!fn || !base) return false;
    const cuuint64_t esz = fp64 ? 8 : 4;
    const cuuint64_t dims[3] = {(cuuint64_t)px, (cuuint64_t)ny, (cuuint64_t)nzs};
    const cuuint64_t strides[2] = {(cuuint64_t)px * esz, (cuuint64_t)px * ny * esz};
    const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    return fn(m, fp64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void *>(base),
              dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Encodes the tensor maps of both phases for the handle's current field and
// model buffers; a change of any map invalidates the captured graph.
template <typename T>
int build_tma_maps(mittet_handle *h) {
    using S = TmaShape<T>;
    static std::once_flag attr_once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(attr_once, [] {
        for (const auto &c : tma_cfgs<T>()) {
            cudaError_t e1 = cudaFuncSetAttribute(c.ek, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem(true));
            cudaError_t e2 = cudaFuncSetAttribute(c.hk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem(false));
            if (e1 != cudaSuccess) attr_err = e1;
            if (e2 != cudaSuccess) attr_err = e2;
        }
    });
    const char *mode = std::getenv("MITTET_INTERIOR");
    if (attr_err != cudaSuccess || (mode && std::string(mode) == "ldg")) {
        h->tma_ok = false;
        return MITTET_OK;
    }
    const int px = h->px, ny = h->g.ny, nz = h->g.nz, TX = S::TX, TY = S::TY, PA = TX + 8;
    const long long nzs = (long long)nz * h->nshot;
    const bool f64 = h->fp64;
    TmaMaps me, mh;
    memset(&me, 0, sizeof(me));
    memset(&mh, 0, sizeof(mh));
    auto F = [&](int c) { return h->fields[c].p; };
    bool ok = encode_map(&me.map[0], F(5), f64, px, ny, nzs, PA, TY + 3) &&   // Hz, x and y halo
              encode_map(&me.map[1], F(4), f64, px, ny, nzs, PA, TY) &&       // Hy, x halo
              encode_map(&me.map[2], F(3), f64, px, ny, nzs, TX, TY + 3) &&   // Hx, y halo
              encode_map(&me.map[3], h->m.p, f64, px, ny, nz, TX, TY) &&      // m
              encode_map(&me.map[4], F(0), f64, px, ny, nzs, TX, TY) &&
              encode_map(&me.map[5], F(1), f64, px, ny, nzs, TX, TY) &&
              encode_map(&me.map[6], F(2), f64, px, ny, nzs, TX, TY) &&
              encode_map(&mh.map[0], F(2), f64, px, ny, nzs, PA, TY + 3) &&   // Ez, x and y halo
              encode_map(&mh.map[1], F(1), f64, px, ny, nzs, PA, TY) &&       // Ey, x halo
              encode_map(&mh.map[2], F(0), f64, px, ny, nzs, TX, TY + 3) &&   // Ex, y halo
              encode_map(&mh.map[3], F(3), f64, px, ny, nzs, TX, TY) &&
              encode_map(&mh.map[4], F(4), f64, px, ny, nzs, TX, TY) &&
              encode_map(&mh.map[5], F(5), f64, px, ny, nzs, TX, TY);
    if (ok && h->has_mu) ok = encode_map(&mh.map[6], h->dtmu.p, f64, px, ny, nz, TX, TY);
    if (ok && (!h->tma_ok || memcmp(&me, &h->tma_maps[0], sizeof(me)) || memcmp(&mh, &h->tma_maps[1], sizeof(mh))))
        drop_graph(h);
    h->tma_ok = ok;
    h->tma_maps[0] = me;
    h->tma_maps[1] = mh;
    h->tma_nown[0] = 4;
    h->tma_nown[1] = h->has_mu ? 4 : 3;
    return MITTET_OK;
}

// The interior of one phase with TMA config ci.
template <typename T>
int launch_tma(mittet_handle *h, bool e, int ci, const PhaseArgs<T> &a, cudaStream_t st) {
    using S = TmaShape<T>;
    const int p = e ? 0 : 1;
    if (!h->has_ibox[p] || h->layout[p] == kLayoutOneBox) return 0;
    const TmaCfg<T> &c = tma_cfgs<T>()[ci];
    const int *ib = h->ibox[p];
    TmaTiling tl;
    tl.x0 = ib[0]; tl.y0 = ib[1]; tl.z0 = ib[2];
    tl.x1 = ib[3]; tl.y1 = ib[4]; tl.z1 = ib[5];
    tl.ntx = (tl.x1 - tl.x0 + S::TX - 1) / S::TX;
    tl.nty = (tl.y1 - tl.y0 + S::TY - 1) / S::TY;
    tl.zc = c.zc;
    tl.spin_limit = h->tma_spin;
    const int nzc = (tl.z1 - tl.z0 + c.zc - 1) / c.zc;
    const dim3 grid(tl.ntx * tl.nty * nzc, h->nshot), block(S::TX / 2, S::TY);
    const size_t smem = c.smem(e);
    (e ? c.ek : c.hk)<<<grid, block, smem, st>>>(a, tl, h->tma_maps[p], h->tma_nown[p], h->d_flag.as<int>());
    return 1;
}

// True when a phase's arguments are the handle's own buffers (the ones the
// tensor maps describe).
template <typename T>
bool tma_usable(const mittet_handle *h, const PhaseArgs<T> &a) {
    return h->tma_ok && a.f[0] == h->fields[0].as<T>() && a.fo[0] == a.f[0] && a.f[3] == h->fields[3].as<T>() &&
           a.fo[3] == a.f[3] && a.m == h->m.as<T>();
}

template <typename T>
using BoundaryKernel = void (*)(PhaseArgs<T>, const TileMap *, int, int, int);

// The merged boundary kernels (stencil.cuh boundary_kernel), by thread shape.
template <typename T>
BoundaryKernel<T> boundary_kernel_for(int vx, int bx, int by, bool e) {
    if (vx == 2 && bx == 32 && by == 4) return e ? boundary_kernel<T, 2, 32, 4, true> : boundary_kernel<T, 2, 32, 4, false>;
    if (vx == 2 && bx == 16 && by == 8) return e ? boundary_kernel<T, 2, 16, 8, true> : boundary_kernel<T, 2, 16, 8, false>;
    if (vx == 2 && bx == 8 && by == 16) return e ? boundary_kernel<T, 2, 8, 16, true> : boundary_kernel<T, 2, 8, 16, false>;
    return nullptr;
}

// The four boundary parts of a phase as one launch of variant vi's tiles.
template <typename T>
int launch_boundary(mittet_handle *h, bool e, int vi, const PhaseArgs<T> &a, cudaStream_t st) {
    const Variant<T> &v = variants<T>()[vi];
    BoundaryKernel<T> k = boundary_kernel_for<T>(v.vx, v.bx, v.by, e);
    const int slot = 2 * vi + (e ? 0 : 1);
    const int first = h->ptile[slot][1], last = h->ptile[slot][kParts];
    if (!k || last <= first) return 0;
    const TileMap &th = h->tmaps_host[slot];
    k<<<dim3(last - first, h->nshot), dim3(v.bx, v.by), 0, st>>>(a, h->tmaps.as<TileMap>() + slot, first, th.pbox[1],
                                                                   th.pbox[kParts]);
    return 1;
}

// The interior and x faces of a phase as one band launch (stencil.cuh
// band_kernel): 128-thread CTAs, interior tiles of 64 (FP32) or 32 (FP64)
// cells, x-face tiles of 32 cells, zc planes per band.
template <typename T>
struct BandShape {
    static constexpr int VXI = sizeof(T) == 4 ? 4 : 2, VXF = 2, BX = 16, BY = 8;
};

template <typename T>
int launch_band(mittet_handle *h, bool e, int zc, const PhaseArgs<T> &a, cudaStream_t st) {
    using S = BandShape<T>;
    const int p = e ? 0 : 1;
    if (!h->has_ibox[p] || h->layout[p] == kLayoutOneBox || zc <= 0) return 0;
    const int *ib = h->ibox[p];
    BandMap bm;
    bm.x0 = ib[0]; bm.y0 = ib[1]; bm.z0 = ib[2];
    bm.x1 = ib[3]; bm.y1 = ib[4]; bm.z1 = ib[5];
    bm.nx = h->g.nx;
    bm.zc = zc;
    const int wf = S::BX * S::VXF, wi = S::BX * S::VXI;
    bm.ntl = (bm.x0 + wf - 1) / wf;
    bm.nti = (bm.x1 - bm.x0 + wi - 1) / wi;
    bm.ntr = (bm.nx - bm.x1 + wf - 1) / wf;
    bm.nty = (bm.y1 - bm.y0 + S::BY - 1) / S::BY;
    const int nzc = (bm.z1 - bm.z0 + zc - 1) / zc;
    const dim3 grid((bm.ntl + bm.nti + bm.ntr) * bm.nty * nzc, h->nshot), block(S::BX, S::BY);
    if (e)
        band_kernel<T, S::VXI, S::VXF, S::BX, S::BY, true><<<grid, block, 0, st>>>(a, bm);
    else
        band_kernel<T, S::VXI, S::VXF, S::BX, S::BY, false><<<grid, block, 0, st>>>(a, bm);
    return 1;
}
constexpr int kBandZc[3] = {4, 8, 16};  // band depths the autotuner tries

// One part of a phase (0 interior, 1 faces, 2 edges and corners) with
// variant vi (vi < 0: TMA interior config -1 - vi); returns 1 if it
// launched a kernel.
template <typename T>
int launch_part(mittet_handle *h, bool e, int part, int vi, const PhaseArgs<T> &a, cudaStream_t st = nullptr) {
    if (!st) st = h->st;
    if (vi < 0) {
        if (part == 0 && tma_usable<T>(h, a)) return launch_tma<T>(h, e, -1 - vi, a, st);
        vi = h->ldg_int[e ? 0 : 1];  // other buffers (gradient replays): best plain-load body
    }
    const Variant<T> &v = variants<T>()[vi];
    const int slot = 2 * vi + (e ? 0 : 1);
    const TileMap *tm = h->tmaps.as<TileMap>() + slot;
    const int first = h->ptile[slot][part], last = h->ptile[slot][part + 1];
    if (last <= first) return 0;
    const TileMap &th = h->tmaps_host[slot];
    dim3 block(v.bx, v.by, v.bz > 0 ? v.bz : 1), grid(last - first, h->nshot);
    v.k[e ? 0 : 1][part]<<<grid, block, 0, st>>>(a, tm, first, th.pbox[part], th.pbox[part + 1]);
    return 1;
}

// Side streams and events of the concurrent parts, created once per handle.
int ensure_part_streams(mittet_handle *h) {
    if (h->ev_fork) return MITTET_OK;
    for (int p = 1; p < kParts; p++) {
        CK(cudaStreamCreateWithFlags(&h->pst[p], cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&h->ev_join[p], cudaEventDisableTiming));
    }
    CK(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
    return MITTET_OK;
}

// One phase = interior, x/y/z faces and edges, each part with its own variant.
// The parts write disjoint cells (and their own psi and ring entries) and
// only read the other field, so the x/y/z faces and edges run on side streams
// concurrently with the interior, forked from and joined back to the
// handle's stream (inside a capture these become parallel graph branches,
// and each part's tail overlaps the others).  Returns the number of launches.
template <typename T>
int launch_phase(mittet_handle *h, bool e, const int *vi, const PhaseArgs<T> &a) {
    int n = 0;
    const int mb = h->merge_b[e ? 0 : 1];
    if (mb >= 0 && h->ev_fork) {  // interior + one merged boundary launch
        cudaEventRecord(h->ev_fork, h->st);
        cudaStreamWaitEvent(h->pst[1], h->ev_fork, 0);
        n += launch_boundary<T>(h, e, mb, a, h->pst[1]);
        n += launch_part<T>(h, e, 0, vi[0], a, h->st);
        cudaEventRecord(h->ev_join[1], h->pst[1]);
        cudaStreamWaitEvent(h->st, h->ev_join[1], 0);
        return n;
    }
    const int bz = h->band[e ? 0 : 1];
    if (bz > 0 && h->ev_fork && h->has_ibox[e ? 0 : 1] && h->layout[e ? 0 : 1] != kLayoutOneBox) {  // band + rest
        cudaEventRecord(h->ev_fork, h->st);
        for (int p = 2; p < kParts; p++) {
            cudaStreamWaitEvent(h->pst[p], h->ev_fork, 0);
            n += launch_part<T>(h, e, p, vi[p], a, h->pst[p]);
        }
        n += launch_band<T>(h, e, bz, a, h->st);
        for (int p = 2; p < kParts; p++) {
            cudaEventRecord(h->ev_join[p], h->pst[p]);
            cudaStreamWaitEvent(h->st, h->ev_join[p], 0);
        }
        return n;
    }
    if (!h->ev_fork || std::getenv("MITTET_SERIAL_PARTS")) {
        for (int part = 0; part < kParts; part++) n += launch_part<T>(h, e, part, vi[part], a);
        return n;
    }
    cudaEventRecord(h->ev_fork, h->st);
    for (int p = 1; p < kParts; p++) cudaStreamWaitEvent(h->pst[p], h->ev_fork, 0);
    // the small, latency-bound faces and edges are submitted before the
    // interior, whose many CTAs would otherwise occupy every SM first
    const bool faces_first = !std::getenv("MITTET_INTERIOR_FIRST");
    if (!faces_first) n += launch_part<T>(h, e, 0, vi[0], a, h->st);
    for (int p = 1; p < kParts; p++) n += launch_part<T>(h, e, p, vi[p], a, h->pst[p]);
    if (faces_first) n += launch_part<T>(h, e, 0, vi[0], a, h->st);
    for (int p = 1; p < kParts; p++) {
        cudaEventRecord(h->ev_join[p], h->pst[p]);
        cudaStreamWaitEvent(h->st, h->ev_join[p], 0);
    }
    return n;
}

template <typename T>
void launch_step(mittet_handle *h, const PhaseArgs<T> &ea, const PhaseArgs<T> &ha, const InjectArgs<T> &ia_m,
                 const InjectArgs<T> &ia_e, const SampleArgs<T> &sa) {
    if (h->has_mag) { inject_kernel<T><<<1, 128, 0, h->st>>>(ia_m); h->launches++; }
    h->launches += launch_phase<T>(h, true, h->var_e, ea);
    if (h->has_ele) { inject_kernel<T><<<1, 128, 0, h->st>>>(ia_e); h->launches++; }
    h->launches += launch_phase<T>(h, false, h->var_h, ha);
    sample_kernel<T><<<1, 1024, 0, h->st>>>(sa);
    h->launches++;
}

// ------------------------------------------------------- persistent launch
// The kernel instances of persistent.cuh, by thread shape: each serves the
// stencil variants of that shape (their tile maps give the z chunk ZC).
template <typename T>
using PersistKernel = void (*)(PersistArgs<T>);

template <typename T>
PersistKernel<T> persist_kernel_for(int vx, int bx, int by) {
    if (vx == 2 && bx == 32 && by == 4) return persistent_steps_kernel<T, 2, 32, 4>;
    if (vx == 2 && bx == 16 && by == 8) return persistent_steps_kernel<T, 2, 16, 8>;
    if constexpr (sizeof(T) == 4)
        if (vx == 4 && bx == 16 && by == 8) return persistent_steps_kernel<T, 4, 16, 8>;
    return nullptr;
}

// Co-resident grid of the persistent kernel of variant vi: CTAs per SM from
// its occupancy times the SMs, at most one CTA per tile of the larger phase.
template <typename T>
int persist_grid_for(mittet_handle *h, int vi) {
    const Variant<T> &v = variants<T>()[vi];
    PersistKernel<T> k = persist_kernel_for<T>(v.vx, v.bx, v.by);
    if (!k || v.bz > 0) return 0;
    int nb = 0, nsm = 0, coop = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, v.bx * v.by, 0) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->ph.device) != cudaSuccess ||
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, h->ph.device) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (!coop || nb <= 0) return 0;
    const long long tiles = (long long)std::max(h->ptile[2 * vi][kParts], h->ptile[2 * vi + 1][kParts]) * h->nshot;
    return (int)std::min<long long>((long long)nb * nsm, tiles);
}

template <typename T>
PersistArgs<T> persist_args(mittet_handle *h, int vi, int grid, int nsteps, const PhaseArgs<T> &ea,
                            const PhaseArgs<T> &ha, const InjectArgs<T> &ia_m, const InjectArgs<T> &ia_e,
                            const SampleArgs<T> &sa) {
    PersistArgs<T> p;
    memset(&p, 0, sizeof(p));
    p.e = ea;
    p.h = ha;
    p.tme = h->tmaps.as<TileMap>() + 2 * vi;
    p.tmh = h->tmaps.as<TileMap>() + 2 * vi + 1;
    p.ntile_e = h->ptile[2 * vi][kParts];
    p.ntile_h = h->ptile[2 * vi + 1][kParts];
    p.nshot = h->nshot;
    p.im = ia_m;
    p.ie = ia_e;
    p.has_mag = h->has_mag ? 1 : 0;
    p.has_ele = h->has_ele ? 1 : 0;
    p.smp = sa;
    p.nsteps = nsteps;
    p.ctl.bar = h->bar.as<GridBarrier>();
    p.ctl.err = h->d_flag.as<int>();
    // MITTET_PERSIST_STALL=1 makes every barrier wait for one CTA more than
    // the grid has, so that a test can watch the waits give up
    const char *stall = std::getenv("MITTET_PERSIST_STALL");
    p.ctl.expect = (unsigned)grid + ((stall && std::atoi(stall) == 1) ? 1u : 0u);
    const char *wms = std::getenv("MITTET_PERSIST_WAIT_MS");
    const double ms = wms ? std::max(1.0, std::atof(wms)) : 2000.0;
    p.ctl.wait_ns = (unsigned long long)(ms * 1e6);
    return p;
}

// One cooperative launch of nsteps steps (and the reset of its barrier words).
template <typename T>
int launch_persistent(mittet_handle *h, int vi, int grid, const PersistArgs<T> &p, cudaStream_t st) {
    const Variant<T> &v = variants<T>()[vi];
    PersistKernel<T> k = persist_kernel_for<T>(v.vx, v.bx, v.by);
    CK(cudaMemsetAsync(h->bar.p, 0, sizeof(GridBarrier), st));
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)v.bx, (unsigned)v.by);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, k, p));
    return MITTET_OK;
}

// Device time of one replay of a graph (after one untimed replay).
int time_graph(mittet_handle *h, cudaGraphExec_t g, float *ms) {
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaGraphLaunch(g, h->st));
    CK(cudaEventRecord(e0, h->st));
    CK(cudaGraphLaunch(g, h->st));
    CK(cudaEventRecord(e1, h->st));
    CK(cudaEventSynchronize(e1));
    CK(cudaEventElapsedTime(ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return MITTET_OK;
}

// Chooses between the stepped graph of part kernels and the persistent
// launch for this grid and batch by timing one captured block of G steps of
// each (MITTET_PERSIST=0 / 1 forces one).  Leaves zero fields behind.
std::mutex g_persist_mu;
std::map<std::array<long long, 8>, int> g_persist_cache;  // choice per (grid, shots, precision, points, ring)

template <typename T>
int decide_persistent(mittet_handle *h, const PhaseArgs<T> &ea, const PhaseArgs<T> &ha, const InjectArgs<T> &ia_m,
                      const InjectArgs<T> &ia_e, const SampleArgs<T> &sa, int G) {
    h->persist_decided = true;
    h->persist_vi = -1;
    const char *mode = std::getenv("MITTET_PERSIST");
    const int force = mode ? std::atoi(mode) : -1;
    if (force == 0) return MITTET_OK;
    CK(h->bar.ensure(sizeof(GridBarrier)));
    const std::array<long long, 8> key = {h->g.nx, h->g.ny, h->g.nz, h->nshot, (long long)h->fp64 + 2 * (force == 1),
                                          (long long)h->has_mag + 2 * h->has_ele, ea.ring_k, h->nrec};
    if (!std::getenv("MITTET_PERSIST_STALL")) {
        std::lock_guard<std::mutex> lk(g_persist_mu);
        auto it = g_persist_cache.find(key);
        if (it != g_persist_cache.end()) {
            h->persist_vi = it->second;
            if (h->persist_vi >= 0) h->persist_grid = persist_grid_for<T>(h, h->persist_vi);
            return MITTET_OK;
        }
    }
    // The persistent launch only competes where a step holds little work
    // (launch gaps dominate): measured on a B200 it is 1.5x slower than the
    // stepped graph for one 64^3 shot and 4-6x slower for 32 of them, so it
    // is timed only for steps of at most 4 M cells (or when forced), and only
    // in the two-cell shapes with short z chunks that came closest.
    const long long step_cells = (long long)h->nshot * h->fshot;
    if (force != 1 && step_cells > (4LL << 20)) {
        h->persist_vi = -1;
        std::lock_guard<std::mutex> lk(g_persist_mu);
        g_persist_cache[key] = -1;
        return MITTET_OK;
    }
    const bool log = std::getenv("MITTET_TUNE_LOG") != nullptr;
    auto capture = [&](int vi, cudaGraphExec_t *out) -> int {
        cudaGraph_t graph;
        *out = nullptr;
        if (cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            return 1;
        }
        int bad = 0;
        if (vi < 0) {
            for (int s = 0; s < G; s++) launch_step<T>(h, ea, ha, ia_m, ia_e, sa);
        } else {
            const int grid = persist_grid_for<T>(h, vi);
            bad = grid <= 0 || launch_persistent<T>(h, vi, grid, persist_args<T>(h, vi, grid, G, ea, ha, ia_m, ia_e, sa),
                                                     h->st) != MITTET_OK;
        }
        cudaError_t ec = cudaStreamEndCapture(h->st, &graph);
        if (ec != cudaSuccess || bad) {
            cudaGetLastError();
            if (ec == cudaSuccess) cudaGraphDestroy(graph);
            return 1;
        }
        ec = cudaGraphInstantiate(out, graph, 0);
        cudaGraphDestroy(graph);
        if (ec != cudaSuccess) {
            cudaGetLastError();
            *out = nullptr;
            return 1;
        }
        return 0;
    };
    float best = 1e30f;
    int best_vi = -1;
    if (force != 1) {
        cudaGraphExec_t g;
        if (capture(-1, &g) == 0) {
            float ms = 0;
            int rc = time_graph(h, g, &ms);
            cudaGraphExecDestroy(g);
            if (rc) return rc;
            best = ms;
            if (log) fprintf(stderr, "persist? stepped graph: %.4f ms per %d steps\n", ms, G);
        }
    }
    const auto &vs = variants<T>();
    for (int vi = 0; vi < (int)vs.size(); vi++) {
        if (vs[vi].bz != 0 || !persist_kernel_for<T>(vs[vi].vx, vs[vi].bx, vs[vi].by) || vs[vi].zc > 4 ||
            vs[vi].vx != 2)
            continue;
        cudaGraphExec_t g;
        if (capture(vi, &g)) continue;
        CK(cudaMemsetAsync(h->d_flag.p, 0, sizeof(int), h->st));
        float ms = 0;
        int rc = time_graph(h, g, &ms);
        cudaGraphExecDestroy(g);
        if (rc) return rc;
        int flag = 0;
        CK(cudaMemcpy(&flag, h->d_flag.p, sizeof(int), cudaMemcpyDeviceToHost));
        CK(cudaMemsetAsync(h->d_flag.p, 0, sizeof(int), h->st));
        if (log)
            fprintf(stderr, "persist? vx%d %dx%dx%d grid %d: %.4f ms per %d steps%s\n", vs[vi].vx, vs[vi].bx, vs[vi].by,
                    vs[vi].zc, persist_grid_for<T>(h, vi), ms, G, (flag & 4) ? " (barrier gave up)" : "");
        if ((flag & 4) && force != 1) continue;
        if (ms < best || (force == 1 && best_vi < 0)) {
            best = ms;
            best_vi = vi;
        }
    }
    h->persist_vi = best_vi;
    if (best_vi >= 0) h->persist_grid = persist_grid_for<T>(h, best_vi);
    if (!std::getenv("MITTET_PERSIST_STALL")) {
        std::lock_guard<std::mutex> lk(g_persist_mu);
        g_persist_cache[key] = best_vi;
    }
    int rc = ensure_state(h);  // back to zero fields and psi
    if (rc) return rc;
    CK(cudaMemsetAsync(h->d_step.p, 0, sizeof(int), h->st));
    return MITTET_OK;
}

// ------------------------------------------------------------- autotuner
// Picks, per phase, the fastest stencil variant for this grid, shot count and
// precision by timing each candidate on the handle's own buffers (zero
// fields, so the state is untouched apart from the ring slot written by the
// E phase).  Results are cached for the process.
// Sets the forward layout of each phase (partitioned, or the whole grid as
// one general box) and re-uploads the tile maps when it changed.
template <typename T>
int sync_layout(mittet_handle *h, int e_layout, int h_layout) {
    h->layout[0] = e_layout;
    h->layout[1] = h_layout;
    if (h->tm_layout[0] == e_layout && h->tm_layout[1] == h_layout) return MITTET_OK;
    return upload_tilemaps<T>(h);
}

std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int, int, int>, std::array<int, 2 * kParts + 8>> g_tune_cache;

template <typename T>
int autotune(mittet_handle *h, const PhaseArgs<T> &ea, const PhaseArgs<T> &ha) {
    const char *imode = std::getenv("MITTET_INTERIOR");  // "ldg" / "tma": restrict the interior body
    const bool only_ldg = imode && std::string(imode) == "ldg";
    const bool only_tma = imode && std::string(imode) == "tma" && tma_usable<T>(h, ea) && tma_usable<T>(h, ha);
    const bool try_tma = !only_ldg && tma_usable<T>(h, ea) && tma_usable<T>(h, ha);
    // MITTET_TMA_CFG=<c> with MITTET_INTERIOR=tma pins the interior of both
    // phases to TMA configuration c (the other parts are still tuned).
    const char *tcfg = std::getenv("MITTET_TMA_CFG");
    const int pin_tma = (only_tma && tcfg) ? std::atoi(tcfg) : -1;
    const bool pinned = pin_tma >= 0 && pin_tma < (int)tma_cfgs<T>().size();
    // MITTET_VARIANT=<v> forces variant v on every part (neither cached nor
    // looked up), e.g. to check that every body gives the same result.
    const char *fix = std::getenv("MITTET_VARIANT");
    const int nv = (int)variants<T>().size();
    if (fix) {
        const int v = std::atoi(fix);
        if (v >= 0 && v < nv) {
            for (int p = 0; p < kParts; p++) h->var_e[p] = h->var_h[p] = v;
            h->ldg_int[0] = h->ldg_int[1] = v;
            h->merge_b[0] = h->merge_b[1] = -1;
            h->band[0] = h->band[1] = 0;
            if (only_tma) h->var_e[0] = h->var_h[0] = -1;
            return sync_layout<T>(h, kLayoutParts, kLayoutParts);
        }
    }
    const auto key = std::make_tuple(h->g.nx, h->g.ny, h->g.nz, h->nshot, (int)h->fp64, ea.ring_k > 0 ? 1 : 0,
                                     (try_tma ? 1 : 0) + (only_tma ? 2 : 0) + (pinned ? 4 * (pin_tma + 1) : 0));
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            for (int p = 0; p < kParts; p++) {
                h->var_e[p] = it->second[p];
                h->var_h[p] = it->second[kParts + p];
            }
            h->ldg_int[0] = it->second[2 * kParts];
            h->ldg_int[1] = it->second[2 * kParts + 1];
            h->merge_b[0] = it->second[2 * kParts + 2];
            h->merge_b[1] = it->second[2 * kParts + 3];
            h->band[0] = it->second[2 * kParts + 4];
            h->band[1] = it->second[2 * kParts + 5];
            return sync_layout<T>(h, it->second[2 * kParts + 6], it->second[2 * kParts + 7]);
        }
    }
    // A tune file (MITTET_TUNE_CACHE) carries choices across processes, e.g. so
    // that a profiled run launches the kernels a plain run chose.
    const char *tfile = std::getenv("MITTET_TUNE_CACHE");
    auto key_text = [&]() {
        char b[128];
        snprintf(b, sizeof(b), "%d %d %d %d %d %d %d", std::get<0>(key), std::get<1>(key), std::get<2>(key),
                 std::get<3>(key), std::get<4>(key), std::get<5>(key), std::get<6>(key));
        return std::string(b);
    };
    if (tfile) {
        if (FILE *f = fopen(tfile, "r")) {
            char line[512];
            const std::string kt = key_text();
            while (fgets(line, sizeof(line), f)) {
                if (strncmp(line, kt.c_str(), kt.size()) != 0 || line[kt.size()] != ':') continue;
                std::array<int, 2 * kParts + 8> e;
                int n = 0, off = (int)kt.size() + 1, used = 0;
                while (n < (int)e.size() && sscanf(line + off, "%d%n", &e[n], &used) == 1) {
                    off += used;
                    n++;
                }
                if (n == 2 * kParts + 4 || n == 2 * kParts + 6) {  // a line without (some) later fields
                    for (int q = n; q < (int)e.size(); q++) e[q] = 0;
                } else if (n != (int)e.size()) {
                    continue;
                }
                for (int p = 0; p < kParts; p++) {
                    h->var_e[p] = e[p];
                    h->var_h[p] = e[kParts + p];
                }
                h->ldg_int[0] = e[2 * kParts];
                h->ldg_int[1] = e[2 * kParts + 1];
                h->merge_b[0] = e[2 * kParts + 2];
                h->merge_b[1] = e[2 * kParts + 3];
                h->band[0] = e[2 * kParts + 4];
                h->band[1] = e[2 * kParts + 5];
                fclose(f);
                {
                    std::lock_guard<std::mutex> lk(g_tune_mu);
                    g_tune_cache[key] = e;
                }
                return sync_layout<T>(h, e[2 * kParts + 6], e[2 * kParts + 7]);
            }
            fclose(f);
        }
    }
    h->merge_b[0] = h->merge_b[1] = -1;
    h->band[0] = h->band[1] = 0;
    if (int rc = sync_layout<T>(h, kLayoutParts, kLayoutParts)) return rc;  // tune the partitioned layout first
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    const long long cells = (long long)h->nshot * h->g.nx * h->g.ny * h->g.nz;
    const int reps = cells > (1LL << 24) ? 3 : (cells > (1LL << 20) ? 8 : 20);
    static const char *pname[kParts] = {"interior", "xfaces", "yfaces", "zfaces", "edges"};
    for (int ph = 0; ph < 2; ph++) {
        const PhaseArgs<T> &a = ph == 0 ? ea : ha;
        int *var = ph == 0 ? h->var_e : h->var_h;
        for (int part = 0; part < kParts; part++) {
            // candidates: TMA interior configs (v < 0, part 0 only), then the plain-load variants
            float best = 1e30f, best_ldg = 1e30f;
            var[part] = 0;
            if (part == 0) h->ldg_int[ph] = 0;
            const int ntma = (part == 0 && try_tma) ? (int)tma_cfgs<T>().size() : 0;
            for (int v = -ntma; v < nv; v++) {
                if (!launch_part<T>(h, ph == 0, part, v, a)) break;  // warm-up; part is empty
                CK(cudaEventRecord(e0, h->st));
                for (int r = 0; r < reps; r++) launch_part<T>(h, ph == 0, part, v, a);
                CK(cudaEventRecord(e1, h->st));
                CK(cudaEventSynchronize(e1));
                CK(cudaGetLastError());
                float ms = 0;
                CK(cudaEventElapsedTime(&ms, e0, e1));
                if (std::getenv("MITTET_TUNE_LOG")) {
                    if (v < 0)
                        fprintf(stderr, "autotune %s %s tma %dx%dx%d: %.4f ms\n", ph == 0 ? "E" : "H", pname[part],
                                TmaShape<T>::TX, TmaShape<T>::TY, tma_cfgs<T>()[-1 - v].zc, ms / reps);
                    else
                        fprintf(stderr, "autotune %s %s vx%d %dx%dx%d%s: %.4f ms\n", ph == 0 ? "E" : "H", pname[part],
                                variants<T>()[v].vx, variants<T>()[v].bx, variants<T>()[v].by, variants<T>()[v].zc,
                                variants<T>()[v].bz > 0 ? " one-plane" : "", ms / reps);
                }
                const bool eligible = !(only_tma && part == 0 && v >= 0) && !(pinned && part == 0 && v != -1 - pin_tma);
                if (eligible && ms < best) {
                    best = ms;
                    var[part] = v;
                }
                if (part == 0 && v >= 0 && ms < best_ldg) {
                    best_ldg = ms;
                    h->ldg_int[ph] = v;
                }
            }
        }
    }
    // Refinement on the whole phase.  The per-part times above are taken with
    // each part alone on the GPU; in a step the five parts run at once on
    // side streams and share the SMs, so a part's best shape alone need not
    // be its best beside the others.  Coordinate descent over the parts,
    // timing the full phase (fork, five parts, join) for each candidate.
    if (h->ev_fork && !only_tma && !pinned && !std::getenv("MITTET_PART_TUNE_ONLY")) {
        for (int ph = 0; ph < 2; ph++) {
            const PhaseArgs<T> &a = ph == 0 ? ea : ha;
            int *var = ph == 0 ? h->var_e : h->var_h;
            auto phase_ms = [&](float *out) -> int {
                launch_phase<T>(h, ph == 0, var, a);  // warm-up
                CK(cudaEventRecord(e0, h->st));
                for (int r = 0; r < reps; r++) launch_phase<T>(h, ph == 0, var, a);
                CK(cudaEventRecord(e1, h->st));
                CK(cudaEventSynchronize(e1));
                CK(cudaGetLastError());
                CK(cudaEventElapsedTime(out, e0, e1));
                *out /= reps;
                return MITTET_OK;
            };
            float best = 0;
            if (int rc = phase_ms(&best)) return rc;
            for (int pass = 0; pass < 2; pass++) {
                bool changed = false;
                for (int part = 0; part < kParts; part++) {
                    if (h->ptile[2 * 0 + (ph == 0 ? 0 : 1)][part + 1] <= h->ptile[2 * 0 + (ph == 0 ? 0 : 1)][part])
                        continue;  // the part is empty
                    const int cur = var[part];
                    int keep = cur;
                    const int ntma = (part == 0 && try_tma) ? (int)tma_cfgs<T>().size() : 0;
                    for (int v = -ntma; v < nv; v++) {
                        if (v == cur) continue;
                        var[part] = v;
                        float ms = 0;
                        if (int rc = phase_ms(&ms)) return rc;
                        if (ms < best * 0.99f) {
                            best = ms;
                            keep = v;
                        }
                    }
                    var[part] = keep;
                    changed |= keep != cur;
                }
                if (std::getenv("MITTET_TUNE_LOG"))
                    fprintf(stderr, "autotune %s phase pass %d: %.4f ms\n", ph == 0 ? "E" : "H", pass, best);
                if (!changed) break;
            }
            // the four boundary parts merged into one launch, per shape
            int &mb = h->merge_b[ph];
            int keep = -1;
            for (int v = 0; v < nv; v++) {
                const Variant<T> &vv = variants<T>()[v];
                if (vv.bz != 0 || !boundary_kernel_for<T>(vv.vx, vv.bx, vv.by, ph == 0)) continue;
                mb = v;
                float ms = 0;
                if (int rc = phase_ms(&ms)) return rc;
                if (std::getenv("MITTET_TUNE_LOG"))
                    fprintf(stderr, "autotune %s merged boundary vx%d %dx%dx%d: %.4f ms\n", ph == 0 ? "E" : "H", vv.vx,
                            vv.bx, vv.by, vv.zc, ms);
                if (ms < best * 0.99f) {
                    best = ms;
                    keep = v;
                }
            }
            mb = keep;
            // the interior and x faces as one band launch (no merged boundary)
            const int mb_keep = mb;
            int &bz = h->band[ph];
            int bkeep = 0;
            if (h->has_ibox[ph]) {
                mb = -1;
                for (int zc : kBandZc) {
                    bz = zc;
                    float ms = 0;
                    if (int rc = phase_ms(&ms)) return rc;
                    if (std::getenv("MITTET_TUNE_LOG"))
                        fprintf(stderr, "autotune %s band launch 16x8x%d: %.4f ms\n", ph == 0 ? "E" : "H", zc, ms);
                    if (ms < best * 0.99f) {
                        best = ms;
                        bkeep = zc;
                    }
                }
            }
            bz = bkeep;
            mb = bkeep > 0 ? -1 : mb_keep;
            // other layouts: the whole grid as one general box (wins where
            // most cells are CPML slab), and the interior and x faces as
            // before with the y- and z-slab rows whole in general boxes;
            // every variant on the general boxes, kept if the phase is faster
            if (h->has_ibox[ph] && !std::getenv("MITTET_PARTS_ONLY")) {
                const int keep_v = var[4], keep_mb = mb, keep_bz = bz;
                int win_layout = kLayoutParts, win_v = keep_v;
                for (int lay : {kLayoutOneBox, kLayoutCoreRows}) {
                    h->layout[ph] = lay;
                    if (int rc = sync_layout<T>(h, h->layout[0], h->layout[1])) return rc;
                    mb = lay == kLayoutOneBox ? -1 : keep_mb;
                    bz = lay == kLayoutOneBox ? 0 : keep_bz;
                    for (int v = 0; v < nv; v++) {
                        var[4] = v;
                        float ms = 0;
                        if (int rc = phase_ms(&ms)) return rc;
                        if (std::getenv("MITTET_TUNE_LOG"))
                            fprintf(stderr, "autotune %s layout %d vx%d %dx%dx%d%s: %.4f ms\n", ph == 0 ? "E" : "H", lay,
                                    variants<T>()[v].vx, variants<T>()[v].bx, variants<T>()[v].by, variants<T>()[v].zc,
                                    variants<T>()[v].bz > 0 ? " one-plane" : "", ms);
                        if (ms < best * 0.99f) {
                            best = ms;
                            win_layout = lay;
                            win_v = v;
                        }
                    }
                }
                h->layout[ph] = win_layout;
                var[4] = win_v;
                mb = win_layout == kLayoutOneBox ? -1 : keep_mb;
                bz = win_layout == kLayoutOneBox ? 0 : keep_bz;
                if (int rc = sync_layout<T>(h, h->layout[0], h->layout[1])) return rc;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    std::array<int, 2 * kParts + 8> entry;
    for (int p = 0; p < kParts; p++) {
        entry[p] = h->var_e[p];
        entry[kParts + p] = h->var_h[p];
    }
    entry[2 * kParts] = h->ldg_int[0];
    entry[2 * kParts + 1] = h->ldg_int[1];
    entry[2 * kParts + 2] = h->merge_b[0];
    entry[2 * kParts + 3] = h->merge_b[1];
    entry[2 * kParts + 4] = h->band[0];
    entry[2 * kParts + 5] = h->band[1];
    entry[2 * kParts + 6] = h->layout[0];
    entry[2 * kParts + 7] = h->layout[1];
    g_tune_cache[key] = entry;
    if (tfile) {
        if (FILE *f = fopen(tfile, "a")) {
            fprintf(f, "%s:", key_text().c_str());
            for (int v : entry) fprintf(f, " %d", v);
            fprintf(f, "\n");
            fclose(f);
        }
    }
    return MITTET_OK;
}

// Folds the last cnt ring steps (time steps n0 .. n0+cnt-1) into the volume
// accumulators: one launch per group of up to four frequencies.
template <typename T>
void launch_volume_flush(mittet_handle *h, int cnt, int n0) {
    const int nf = (int)h->omega.size();
    int vc[3] = {0, 0, 0}, nvc = 0;
    for (int c = 0; c < 3; c++)
        if (h->vmask >> c & 1) vc[nvc++] = c;
    const dim3 grid((unsigned)((h->fshot + 255) / 256), nvc, h->nshot);
    for (int f0 = 0; f0 < nf; f0 += kFlushFreqs) {
        FlushWeights w;
        memset(&w, 0, sizeof(w));
        for (int s = 0; s < cnt; s++)
            for (int f = 0; f < kFlushFreqs && f0 + f < nf; f++) {
                const size_t q = ((size_t)(n0 + s) * nf + f0 + f) * 2;
                w.wr[s][f] = h->wt_host[q];
                w.wi[s][f] = h->wt_host[q + 1];
            }
        volume_dft_kernel<T><<<grid, 256, 0, h->st>>>(h->ring.as<T>(), ring_comp_of((long long)h->nshot * h->fshot), h->ring_k,
                                                      make_int3(vc[0], vc[1], vc[2]), h->fshot, cnt, f0, nf, w,
                                                      h->acc.as<double2>());
        h->launches++;
    }
}

template <typename T>
int run_forward(mittet_handle *h, int nt) {
    const int ns = h->nshot;
    int rc = ensure_state(h);
    if (rc) return rc;
    rc = ensure_part_streams(h);
    if (rc) return rc;
    CK(h->d_step.ensure(sizeof(int)));
    CK(h->d_flag.ensure(sizeof(int)));
    CK(cudaMemsetAsync(h->d_step.p, 0, sizeof(int), h->st));
    CK(cudaMemsetAsync(h->d_flag.p, 0, sizeof(int), h->st));
    const size_t ntr = (size_t)ns * std::max(h->nrec, 1) * nt;
    CK(h->traces.ensure(ntr * h->esz));
    const int nf = (int)h->omega.size();
    const bool vol = h->vmask && nf > 0;
    if (vol) {
        const size_t ring_b = (size_t)h->ring_k * 3 * ring_comp_of((long long)ns * h->fshot) * h->esz;
        CK(h->ring.ensure(ring_b));
        const size_t acc_b = (size_t)ns * 3 * nf * h->fshot * sizeof(double2);
        CK(h->acc.ensure(acc_b));
        CK(cudaMemsetAsync(h->acc.p, 0, acc_b, h->st));
        // weights wt[n][f] = dt exp((i-1) sqrt(w0 w) n dt)
        std::vector<double> &wt = h->wt_host;
        wt.assign((size_t)nt * nf * 2, 0.0);
        for (int n = 0; n < nt; n++)
            for (int f = 0; f < nf; f++) {
                const double xa = std::sqrt(h->ph.omega0 * h->omega[f]) * (double)n * h->ph.dt;
                const double e = std::exp(-xa) * h->ph.dt;
                wt[((size_t)n * nf + f) * 2] = e * std::cos(xa);
                wt[((size_t)n * nf + f) * 2 + 1] = e * std::sin(xa);
            }
    }

    PhaseArgs<T> ea = phase_args<T>(h, true);
    PhaseArgs<T> ha = phase_args<T>(h, false);
    if (!vol) ea.ring_k = 0;
    InjectArgs<T> ia;
    memset(&ia, 0, sizeof(ia));
    for (int c = 0; c < 6; c++) ia.f[c] = h->fields[c].as<T>();
    ia.pts = h->d_pts.as<SrcPoint>();
    ia.npts = h->npts;
    ia.wave = h->wave.as<double>();
    ia.d_step = h->d_step.as<int>();
    if (vol) {
        ia.ring = h->ring.as<T>();
        ia.ring_k = h->ring_k;
        ia.vmask = (int)h->vmask;
        ia.ring_comp = ring_comp_of((long long)ns * h->fshot);
    }
    InjectArgs<T> ia_m = ia, ia_e = ia;
    ia_m.kind = 0;
    ia_e.kind = 1;
    SampleArgs<T> sa;
    memset(&sa, 0, sizeof(sa));
    for (int c = 0; c < 6; c++) sa.f[c] = h->fields[c].as<T>();
    sa.rec_off = h->rec_off.as<long long>();
    sa.rec_comp = h->rec_comp.as<int>();
    sa.nrec = h->nrec;
    sa.nshot = ns;
    sa.fshot = h->fshot;
    sa.traces = h->traces.as<T>();
    sa.nt = nt;
    sa.d_step = h->d_step.as<int>();

    rc = build_tma_maps<T>(h);
    if (rc) return rc;
    if (!h->tuned) {
        rc = autotune<T>(h, ea, ha);
        if (rc) return rc;
        rc = ensure_state(h);  // back to zero fields and psi
        if (rc) return rc;
        h->tuned = true;
    }
    // MITTET_BOUNDARY=<v> forces the merged boundary launch with variant v on
    // both phases (-1: the four part launches), e.g. to check bit-identity
    if (const char *mbv = std::getenv("MITTET_BOUNDARY")) {
        const int v = std::atoi(mbv);
        const auto &vs = variants<T>();
        const bool ok = v >= 0 && v < (int)vs.size() && vs[v].bz == 0 &&
                        boundary_kernel_for<T>(vs[v].vx, vs[v].bx, vs[v].by, true) != nullptr;
        h->merge_b[0] = h->merge_b[1] = ok ? v : -1;
        if (ok) h->band[0] = h->band[1] = 0;
    }
    // MITTET_BAND=<zc> forces the band launch of the interior and x faces
    // with zc planes per band on both phases (0: the part launches)
    if (const char *bv = std::getenv("MITTET_BAND")) {
        const int zc = std::max(0, std::atoi(bv));
        h->band[0] = h->band[1] = zc;
        if (zc > 0) h->merge_b[0] = h->merge_b[1] = -1;
    }
    // MITTET_LAYOUT=0 / 1 / 2 forces on both phases the partitioned layout /
    // the whole grid as one general box / the interior and x faces as parts
    // with the slab rows whole (the general boxes run the edge part's variant)
    if (const char *ob = std::getenv("MITTET_LAYOUT")) {
        const int lay = std::min(2, std::max(0, std::atoi(ob)));
        if (lay == kLayoutOneBox) {
            h->band[0] = h->band[1] = 0;
            h->merge_b[0] = h->merge_b[1] = -1;
        }
        rc = sync_layout<T>(h, lay, lay);
        if (rc) return rc;
    }
    // One graph holds G = ring_k steps; the volume flush of those steps (when
    // enabled) is launched after each replay.
    const int G = h->ring_k;
    if (!h->persist_decided) {
        rc = decide_persistent<T>(h, ea, ha, ia_m, ia_e, sa, G);
        if (rc) return rc;
    }
    h->launches = 0;
    const long long key = ((long long)nt << 20) ^ ((long long)ns << 4) ^ (vol ? 1 : 0) ^ ((long long)h->nrec << 40) ^
                          ((long long)(h->persist_vi + 1) << 52);
    if (!h->gexec || h->graph_key != key) {
        if (h->gexec) cudaGraphExecDestroy(h->gexec);
        h->gexec = nullptr;
        cudaGraph_t graph;
        CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
        h->launches = 0;
        if (h->persist_vi >= 0) {
            rc = launch_persistent<T>(h, h->persist_vi, h->persist_grid,
                                      persist_args<T>(h, h->persist_vi, h->persist_grid, G, ea, ha, ia_m, ia_e, sa),
                                      h->st);
            if (rc) {
                cudaGraph_t dead;
                cudaStreamEndCapture(h->st, &dead);
                if (dead) cudaGraphDestroy(dead);
                return rc;
            }
            h->launches = 1;
        } else {
            for (int s = 0; s < G; s++) launch_step<T>(h, ea, ha, ia_m, ia_e, sa);
        }
        h->graph_launches = h->launches;
        cudaError_t ec = cudaStreamEndCapture(h->st, &graph);
        if (ec != cudaSuccess) return fail(MITTET_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ec));
        ec = cudaGraphInstantiate(&h->gexec, graph, 0);
        cudaGraphDestroy(graph);
        if (ec != cudaSuccess) return fail(MITTET_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ec));
        h->graph_key = key;
        h->graph_steps = G;
    }
    h->launches = 0;
    int done = 0;
    while (done + G <= nt) {
        CK(cudaGraphLaunch(h->gexec, h->st));
        h->launches += h->graph_launches;
        if (vol) launch_volume_flush<T>(h, G, done);
        done += G;
    }
    const int rem = nt - done;
    if (rem > 0 && h->persist_vi >= 0) {
        rc = launch_persistent<T>(h, h->persist_vi, h->persist_grid,
                                  persist_args<T>(h, h->persist_vi, h->persist_grid, rem, ea, ha, ia_m, ia_e, sa), h->st);
        if (rc) return rc;
        h->launches++;
    } else {
        for (int s = 0; s < rem; s++) launch_step<T>(h, ea, ha, ia_m, ia_e, sa);
    }
    if (rem > 0 && vol) launch_volume_flush<T>(h, rem, done);
    CK(cudaGetLastError());

    if (h->nrec > 0) {
        finite_check_kernel<T><<<64, 256, 0, h->st>>>(h->traces.as<T>(), (long long)ns * h->nrec * nt,
                                                      h->d_flag.as<int>());
        h->launches++;
        if (nf > 0) {
            CK(h->spectra.ensure((size_t)ns * h->nrec * nf * sizeof(double2)));
            trace_dft_kernel<T><<<nf, 256, 0, h->st>>>(h->traces.as<T>(), ns * h->nrec, nt, h->d_omega.as<double>(),
                                                       nf, h->ph.dt, h->ph.omega0, h->rec_is_h.as<unsigned char>(),
                                                       h->nrec, h->hfac, h->spectra.as<double2>());
            h->launches++;
        }
    }
    CK(cudaGetLastError());
    h->last_nt = nt;
    return MITTET_OK;
}

template <typename T>
int time_kernels(mittet_handle *h, int nsteps, double *ms) {
    int rc = ensure_state(h);
    if (rc) return rc;
    rc = ensure_part_streams(h);
    if (rc) return rc;
    rc = build_tma_maps<T>(h);
    if (rc) return rc;
    CK(cudaMemsetAsync(h->d_step.p, 0, sizeof(int), h->st));
    const int nt = h->last_nt;
    const bool vol = h->vmask && !h->omega.empty();
    PhaseArgs<T> ea = phase_args<T>(h, true);
    PhaseArgs<T> ha = phase_args<T>(h, false);
    if (!vol) ea.ring_k = 0;
    InjectArgs<T> ia;
    memset(&ia, 0, sizeof(ia));
    for (int c = 0; c < 6; c++) ia.f[c] = h->fields[c].as<T>();
    ia.pts = h->d_pts.as<SrcPoint>();
    ia.npts = h->npts;
    ia.wave = h->wave.as<double>();
    ia.d_step = h->d_step.as<int>();
    if (vol) {
        ia.ring = h->ring.as<T>();
        ia.ring_k = h->ring_k;
        ia.vmask = (int)h->vmask;
        ia.ring_comp = ring_comp_of((long long)h->nshot * h->fshot);
    }
    InjectArgs<T> ia_m = ia, ia_e = ia;
    ia_m.kind = 0;
    ia_e.kind = 1;
    SampleArgs<T> sa;
    memset(&sa, 0, sizeof(sa));
    for (int c = 0; c < 6; c++) sa.f[c] = h->fields[c].as<T>();
    sa.rec_off = h->rec_off.as<long long>();
    sa.rec_comp = h->rec_comp.as<int>();
    sa.nrec = h->nrec;
    sa.nshot = h->nshot;
    sa.fshot = h->fshot;
    sa.traces = h->traces.as<T>();
    sa.nt = nt;
    sa.d_step = h->d_step.as<int>();
    cudaEvent_t ev[12];
    for (int q = 0; q < 12; q++) CK(cudaEventCreate(&ev[q]));
    double acc[6] = {0, 0, 0, 0, 0, 0};
    int cnt[6] = {0, 0, 0, 0, 0, 0};
    for (int s = 0; s < nsteps; s++) {
        CK(cudaEventRecord(ev[0], h->st));
        if (h->has_mag) inject_kernel<T><<<1, 128, 0, h->st>>>(ia_m);
        CK(cudaEventRecord(ev[1], h->st));
        launch_phase<T>(h, true, h->var_e, ea);
        CK(cudaEventRecord(ev[2], h->st));
        if (h->has_ele) inject_kernel<T><<<1, 128, 0, h->st>>>(ia_e);
        CK(cudaEventRecord(ev[3], h->st));
        launch_phase<T>(h, false, h->var_h, ha);
        CK(cudaEventRecord(ev[4], h->st));
        sample_kernel<T><<<1, 1024, 0, h->st>>>(sa);  // also advances the step counter
        CK(cudaEventRecord(ev[5], h->st));
        const bool flush = vol && ((s + 1) % h->ring_k == 0);
        if (flush) launch_volume_flush<T>(h, h->ring_k, s + 1 - h->ring_k);
        CK(cudaEventRecord(ev[6], h->st));
        CK(cudaGetLastError());
        CK(cudaEventSynchronize(ev[6]));
        float t;
        const bool ran[6] = {h->has_mag, true, h->has_ele, true, true, flush};
        for (int q = 0; q < 6; q++) {
            if (!ran[q]) continue;
            CK(cudaEventElapsedTime(&t, ev[q], ev[q + 1]));
            acc[q] += t;
            cnt[q]++;
        }
    }
    for (int q = 0; q < 12; q++) cudaEventDestroy(ev[q]);
    for (int q = 0; q < 6; q++) ms[q] = cnt[q] ? acc[q] / cnt[q] : 0.0;
    return MITTET_OK;
}


// ------------------------------------------------------------------ gradient
// Forward (receiver spectra, misfit) -> adjoint sources -> per group of shots:
// forward pass keeping a checkpoint every K steps, then segments in reverse:
// recompute the segment's K states from its checkpoint into a history
// buffer and run the adjoint steps over it.  Shot groups are sized so the
// history fits in a share of the free device memory.
template <typename T>
int run_gradient(mittet_handle *h, int nt, const double *obs_host, int K, double *misfit_out, double *grad_out);

int validate_ready(mittet_handle *h, int nt);

int validate_ready(mittet_handle *h, int nt) {
    if (!h->has_model) return fail(MITTET_ERR_STATE, "mittet_set_model has not been called");
    if (h->nshot <= 0) return fail(MITTET_ERR_STATE, "mittet_set_sources has not been called");
    if (h->nt_wave < nt) return fail(MITTET_ERR_STATE, "wavelet has %d steps, forward asked for %d", h->nt_wave, nt);
    if (nt <= 0) return fail(MITTET_ERR_INVALID_ARG, "nt must be positive");
    return MITTET_OK;
}

// Upload the point sources with their per-point gain (depends on the model).
// The captured step graph reads the points from d_pts at run time, so it
// stays valid unless the buffer moves or the number or kinds of points
// change (those are baked into the graph's launches).
double model_value(mittet_handle *h, int which, size_t c0);

int upload_sources(mittet_handle *h) {
    if (!h->has_model || h->pts.empty()) return MITTET_OK;
    std::vector<SrcPoint> dp(h->pts.size());
    const double vol = h->g.dx * h->g.dy * h->g.dz;
    const bool mag0 = h->has_mag, ele0 = h->has_ele;
    const int npts0 = h->npts;
    const void *buf0 = h->d_pts.p;
    h->has_mag = h->has_ele = false;
    for (size_t q = 0; q < h->pts.size(); q++) {
        const mittet_point_source &p = h->pts[q];
        const long long cell = ((long long)(p.iz - 1) * h->g.ny + (p.iy - 1)) * h->px + (p.ix - 1);
        const size_t c0 = ((size_t)(p.iz - 1) * h->g.ny + (p.iy - 1)) * h->g.nx + (p.ix - 1);
        dp[q].off = (long long)p.shot * h->fshot + cell;
        dp[q].comp = p.comp;
        dp[q].kind = p.kind;
        if (p.kind == MITTET_SRC_MAGNETIC) {
            const double mu = h->has_mu ? model_value(h, 1, c0) : h->ph.mu0;
            dp[q].g = p.amp * h->ph.dt / mu / vol;
            h->has_mag = true;
        } else {
            dp[q].g = p.amp * h->ph.dt * 2.0 * h->ph.omega0 / model_value(h, 0, c0) / vol;
            h->has_ele = true;
        }
    }
    CK(h->d_pts.ensure(dp.size() * sizeof(SrcPoint)));
    CK(cudaMemcpyAsync(h->d_pts.p, dp.data(), dp.size() * sizeof(SrcPoint), cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    h->npts = (int)dp.size();
    if (h->d_pts.p != buf0 || h->npts != npts0 || h->has_mag != mag0 || h->has_ele != ele0) drop_graph(h);
    return MITTET_OK;
}

template <typename T>
int run_gradient(mittet_handle *h, int nt, const double *obs_host, int K, double *misfit_out, double *grad_out) {
    const int ns = h->nshot, nrec = h->nrec, nf = (int)h->omega.size();
    // MITTET_GRAD_LOG: device time of each stage (CUDA events on the handle's
    // stream, synchronised per stage) printed to stderr
    const bool glog = std::getenv("MITTET_GRAD_LOG") != nullptr;
    struct EventPair {  // destroyed on every return
        cudaEvent_t e[2] = {nullptr, nullptr};
        ~EventPair() {
            for (cudaEvent_t x : e)
                if (x) cudaEventDestroy(x);
        }
    } gevs;
    cudaEvent_t *gev = gevs.e;
    double gms[3] = {0, 0, 0};  // checkpoint pass, recompute, adjoint
    if (glog) {
        CK(cudaEventCreate(&gev[0]));
        CK(cudaEventCreate(&gev[1]));
    }
    auto gmark = [&](int stage) -> int {
        if (!glog) return MITTET_OK;
        CK(cudaEventRecord(gev[1], h->st));
        CK(cudaEventSynchronize(gev[1]));
        float ms = 0.f;
        if (stage >= 0) {
            CK(cudaEventElapsedTime(&ms, gev[0], gev[1]));
            gms[stage] += ms;
        }
        CK(cudaEventRecord(gev[0], h->st));
        return MITTET_OK;
    };
    int rc = MITTET_OK;
    if (!h->tuned) {
        // one step of a plain forward tunes the stencil variants on this grid
        const uint32_t vmask_saved = h->vmask;
        if (h->vmask) { h->vmask = 0; drop_graph(h); }
        rc = run_forward<T>(h, 1);
        h->vmask = vmask_saved;
        if (vmask_saved) drop_graph(h);
        if (rc) return rc;
    }
    if ((rc = ensure_part_streams(h))) return rc;
    CK(h->d_step.ensure(sizeof(int)));
    CK(h->d_flag.ensure(sizeof(int)));
    CK(cudaMemsetAsync(h->d_flag.p, 0, sizeof(int), h->st));
    // The checkpoint pass of each shot group samples the receivers, so the
    // group's residual and adjoint sources follow from it (no separate
    // forward).
    const size_t nspec = (size_t)ns * nrec * nf;
    auto &B = h->gb;
    DevBuf &d_obs = B.obs, &d_R = B.R, &d_mis = B.mis, &d_asrc = B.asrc;
    CK(d_obs.ensure(std::max<size_t>(nspec, 1) * sizeof(double2)));
    CK(d_R.ensure(std::max<size_t>(nspec, 1) * sizeof(double2)));
    CK(d_mis.ensure(sizeof(double)));
    CK(d_asrc.ensure(std::max<size_t>((size_t)ns * nrec * nt, 1) * sizeof(double)));
    CK(h->traces.ensure((size_t)ns * std::max(nrec, 1) * nt * h->esz));
    CK(h->spectra.ensure(std::max<size_t>(nspec, 1) * sizeof(double2)));
    CK(cudaMemcpyAsync(d_obs.p, obs_host, nspec * sizeof(double2), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemsetAsync(d_mis.p, 0, sizeof(double), h->st));

    // source points, absolute shots
    const double vol = h->g.dx * h->g.dy * h->g.dz;
    std::vector<AdjSrc> asp(h->pts.size());
    for (size_t q = 0; q < h->pts.size(); q++) {
        const mittet_point_source &p = h->pts[q];
        const size_t c0 = ((size_t)(p.iz - 1) * h->g.ny + (p.iy - 1)) * h->g.nx + (p.ix - 1);
        AdjSrc &a = asp[q];
        a.off = ((long long)(p.iz - 1) * h->g.ny + (p.iy - 1)) * h->px + (p.ix - 1);
        a.moff = a.off;
        a.shot = p.shot; a.comp = p.comp; a.kind = p.kind;
        a.i = p.ix - 1; a.j = p.iy - 1; a.k = p.iz - 1;
        a.g = p.kind == MITTET_SRC_MAGNETIC ? p.amp * h->ph.dt / (h->has_mu ? model_value(h, 1, c0) : h->ph.mu0) / vol
                                            : p.amp * h->ph.dt * 2.0 * h->ph.omega0 / model_value(h, 0, c0) / vol;
    }
    DevBuf &d_asp = B.asp;
    CK(d_asp.ensure(std::max<size_t>(asp.size(), 1) * sizeof(AdjSrc)));
    CK(cudaMemcpyAsync(d_asp.p, asp.data(), asp.size() * sizeof(AdjSrc), cudaMemcpyHostToDevice, h->st));

    // group size from memory
    size_t psiE = 0, psiH = 0;
    for (int a = 0; a < 3; a++) { psiE += 2 * psi_elems(h, h->su.se[a], a); psiH += 2 * psi_elems(h, h->su.sh[a], a); }
    const int ncheck = (nt + K - 1) / K;
    const size_t F = (size_t)h->fshot;
    const size_t per_shot = h->esz * ((size_t)(K + 1) * 6 * F + (size_t)ncheck * (6 * F + psiE + psiH) + 6 * F +
                                      psiE + psiH + 6 * F + psiE + psiH + 7 * F) + 8 * F;
    size_t freeb = 0, totb = 0;
    CK(cudaMemGetInfo(&freeb, &totb));
    const size_t budget = (size_t)(0.75 * (double)(freeb + B.held() - d_obs.bytes - d_R.bytes - d_mis.bytes -
                                                   d_asrc.bytes - d_asp.bytes));
    int G = (int)std::min<size_t>((size_t)ns, std::max<size_t>(1, budget / std::max<size_t>(per_shot, 1)));
    if (const char *gcap = std::getenv("MITTET_GRAD_GROUP")) G = std::max(1, std::min(G, std::atoi(gcap)));
    if ((size_t)G * per_shot > budget) return fail(MITTET_ERR_OOM, "one shot of the gradient needs %zu bytes, %zu free", per_shot, freeb);

    DevBuf(&fl)[6] = B.fl, (&lam)[6] = B.lam, (&mu)[7] = B.mu;
    DevBuf(&pe)[3][2] = B.pe, (&pH)[3][2] = B.pH, (&lpe)[3][2] = B.lpe, (&lph)[3][2] = B.lph;
    DevBuf &hist = B.hist, &ck = B.ck, &gacc = B.gacc, &gred = B.gred;
    const size_t gF = (size_t)G * F;
    for (int c = 0; c < 6; c++) { CK(fl[c].ensure(gF * h->esz)); CK(lam[c].ensure(gF * h->esz)); }
    for (int c = 0; c < 7; c++) CK(mu[c].ensure(gF * h->esz));
    for (int a = 0; a < 3; a++)
        for (int w = 0; w < 2; w++) {
            const size_t ne = (size_t)G * psi_elems(h, h->su.se[a], a), nh = (size_t)G * psi_elems(h, h->su.sh[a], a);
            CK(pe[a][w].ensure(ne * h->esz)); CK(pH[a][w].ensure(nh * h->esz));
            CK(lpe[a][w].ensure(ne * h->esz)); CK(lph[a][w].ensure(nh * h->esz));
        }
    CK(hist.ensure((size_t)(K + 1) * 6 * gF * h->esz));
    const size_t ck_stride = (6 * F + psiE + psiH) * (size_t)G * h->esz;
    CK(ck.ensure((size_t)ncheck * ck_stride));
    CK(gacc.ensure(gF * sizeof(double)));
    const size_t ncell = (size_t)h->g.nx * h->g.ny * h->g.nz;
    CK(gred.ensure(ncell * sizeof(double)));
    std::vector<double> gsum(ncell, 0.0), gpart(ncell);
    for (int c = 0; c < 7; c++) CK(cudaMemsetAsync(mu[c].p, 0, gF * h->esz, h->st));

    const int ns_saved = h->nshot;
    const int vmask_keep = (int)h->vmask;
    h->vmask = 0;
    for (int s0 = 0; s0 < ns; s0 += G) {
        const int s1 = std::min(ns, s0 + G), Gg = s1 - s0;
        h->nshot = Gg;
        // group-local source list for the forward injection
        std::vector<SrcPoint> gp;
        for (size_t q = 0; q < h->pts.size(); q++) {
            const mittet_point_source &p = h->pts[q];
            if (p.shot < s0 || p.shot >= s1) continue;
            SrcPoint sp;
            sp.off = (long long)(p.shot - s0) * h->fshot + asp[q].off;
            sp.comp = p.comp;
            sp.kind = p.kind;
            sp.g = asp[q].g;
            gp.push_back(sp);
        }
        DevBuf &d_gp = h->gb.gpts;  // kept: a freed buffer would synchronise the device
        CK(d_gp.ensure(std::max<size_t>(gp.size(), 1) * sizeof(SrcPoint)));
        CK(cudaMemcpyAsync(d_gp.p, gp.data(), gp.size() * sizeof(SrcPoint), cudaMemcpyHostToDevice, h->st));
        PhaseArgs<T> ea = phase_args<T>(h, true), ha = phase_args<T>(h, false);
        for (int c = 0; c < 6; c++) ea.f[c] = ea.fo[c] = ha.f[c] = ha.fo[c] = fl[c].as<T>();
        for (int a = 0; a < 3; a++)
            for (int w = 0; w < 2; w++) { ea.psi[a][w] = pe[a][w].as<T>(); ha.psi[a][w] = pH[a][w].as<T>(); }
        ea.ring_k = 0;
        InjectArgs<T> ia;
        memset(&ia, 0, sizeof(ia));
        for (int c = 0; c < 6; c++) ia.f[c] = fl[c].as<T>();
        ia.pts = d_gp.as<SrcPoint>();
        ia.npts = (int)gp.size();
        ia.wave = h->wave.as<double>();
        ia.d_step = h->d_step.as<int>();
        InjectArgs<T> ia_m = ia, ia_e = ia;
        ia_m.kind = 0;
        ia_e.kind = 1;
        // receivers are sampled in the checkpoint pass only (sa_rec), into
        // the group's rows of the trace buffer
        SampleArgs<T> sa;
        memset(&sa, 0, sizeof(sa));
        for (int c = 0; c < 6; c++) sa.f[c] = fl[c].as<T>();
        sa.nrec = 0;
        sa.nshot = Gg;
        sa.fshot = h->fshot;
        sa.traces = h->traces.as<T>() + (size_t)s0 * nrec * nt;
        sa.nt = nt;
        sa.d_step = h->d_step.as<int>();
        SampleArgs<T> sa_rec = sa;
        sa_rec.rec_off = h->rec_off.as<long long>();
        sa_rec.rec_comp = h->rec_comp.as<int>();
        sa_rec.nrec = nrec;
        bool hm = false, he = false;
        for (const auto &q : gp) { hm |= q.kind == 0; he |= q.kind == 1; }
        const bool mag0 = h->has_mag, ele0 = h->has_ele;
        h->has_mag = hm;
        h->has_ele = he;
        auto save_state = [&](char *dst) -> int {
            size_t o = 0;
            for (int c = 0; c < 6; c++) { CK(cudaMemcpyAsync(dst + o, fl[c].p, (size_t)Gg * F * h->esz, cudaMemcpyDeviceToDevice, h->st)); o += (size_t)G * F * h->esz; }
            for (int a = 0; a < 3; a++)
                for (int w = 0; w < 2; w++) {
                    const size_t ne = (size_t)Gg * psi_elems(h, h->su.se[a], a) * h->esz, nh = (size_t)Gg * psi_elems(h, h->su.sh[a], a) * h->esz;
                    CK(cudaMemcpyAsync(dst + o, pe[a][w].p, ne, cudaMemcpyDeviceToDevice, h->st)); o += (size_t)G * psi_elems(h, h->su.se[a], a) * h->esz;
                    CK(cudaMemcpyAsync(dst + o, pH[a][w].p, nh, cudaMemcpyDeviceToDevice, h->st)); o += (size_t)G * psi_elems(h, h->su.sh[a], a) * h->esz;
                }
            return MITTET_OK;
        };
        // fields to fdst[c] (the working fields when null), psi to the working psi
        auto load_state = [&](const char *src, T *const *fdst) -> int {
            size_t o = 0;
            for (int c = 0; c < 6; c++) {
                void *d = fdst ? (void *)fdst[c] : fl[c].p;
                CK(cudaMemcpyAsync(d, src + o, (size_t)Gg * F * h->esz, cudaMemcpyDeviceToDevice, h->st));
                o += (size_t)G * F * h->esz;
            }
            for (int a = 0; a < 3; a++)
                for (int w = 0; w < 2; w++) {
                    const size_t ne = (size_t)Gg * psi_elems(h, h->su.se[a], a) * h->esz, nh = (size_t)Gg * psi_elems(h, h->su.sh[a], a) * h->esz;
                    CK(cudaMemcpyAsync(pe[a][w].p, src + o, ne, cudaMemcpyDeviceToDevice, h->st)); o += (size_t)G * psi_elems(h, h->su.se[a], a) * h->esz;
                    CK(cudaMemcpyAsync(pH[a][w].p, src + o, nh, cudaMemcpyDeviceToDevice, h->st)); o += (size_t)G * psi_elems(h, h->su.sh[a], a) * h->esz;
                }
            return MITTET_OK;
        };
        auto set_step = [&](int n) -> int {
            CK(cudaMemcpyAsync(h->d_step.p, &n, sizeof(int), cudaMemcpyHostToDevice, h->st));
            CK(cudaStreamSynchronize(h->st));  // n lives on the host stack
            return MITTET_OK;
        };
        auto fwd_step = [&](bool sample) {
            if (h->has_mag) inject_kernel<T><<<1, 128, 0, h->st>>>(ia_m);
            launch_phase<T>(h, true, h->var_e, ea);
            if (h->has_ele) inject_kernel<T><<<1, 128, 0, h->st>>>(ia_e);
            launch_phase<T>(h, false, h->var_h, ha);
            if (sample) sample_kernel<T><<<1, 1024, 0, h->st>>>(sa_rec);
            else sample_kernel<T><<<1, 32, 0, h->st>>>(sa);
        };
        // forward pass with checkpoints
        for (int c = 0; c < 6; c++) CK(cudaMemsetAsync(fl[c].p, 0, gF * h->esz, h->st));
        for (int a = 0; a < 3; a++)
            for (int w = 0; w < 2; w++) {
                CK(cudaMemsetAsync(pe[a][w].p, 0, (size_t)G * psi_elems(h, h->su.se[a], a) * h->esz, h->st));
                CK(cudaMemsetAsync(pH[a][w].p, 0, (size_t)G * psi_elems(h, h->su.sh[a], a) * h->esz, h->st));
            }
        if ((rc = set_step(0))) return rc;
        if ((rc = gmark(-1))) return rc;
        for (int n = 0; n < nt; n++) {
            if (n % K == 0 && (rc = save_state(ck.as<char>() + (size_t)(n / K) * ck_stride))) return rc;
            fwd_step(true);
        }
        CK(cudaGetLastError());
        // receiver spectra, residual, misfit and adjoint sources of the group
        if (nrec > 0 && nf > 0) {
            const size_t g0 = (size_t)s0 * nrec;
            finite_check_kernel<T><<<64, 256, 0, h->st>>>(sa_rec.traces, (long long)Gg * nrec * nt,
                                                          h->d_flag.as<int>());
            trace_dft_kernel<T><<<nf, 256, 0, h->st>>>(sa_rec.traces, Gg * nrec, nt, h->d_omega.as<double>(), nf,
                                                       h->ph.dt, h->ph.omega0, h->rec_is_h.as<unsigned char>(), nrec,
                                                       h->hfac, h->spectra.as<double2>() + g0 * nf);
            residual_kernel<<<64, 256, 0, h->st>>>(h->spectra.as<double2>() + g0 * nf, d_obs.as<double2>() + g0 * nf,
                                                   (long long)Gg * nrec * nf, d_R.as<double2>() + g0 * nf,
                                                   d_mis.as<double>());
            adj_source_kernel<<<256, 256, 0, h->st>>>(d_R.as<double2>() + g0 * nf, Gg * nrec, nrec, nf, nt,
                                                      h->d_omega.as<double>(), h->ph.dt, h->ph.omega0,
                                                      h->rec_is_h.as<unsigned char>(), h->hfac,
                                                      d_asrc.as<double>() + g0 * nt);
        } else if (nrec > 0) {
            CK(cudaMemsetAsync(d_asrc.as<double>() + (size_t)s0 * nrec * nt, 0,
                               (size_t)Gg * nrec * nt * sizeof(double), h->st));
        }
        CK(cudaGetLastError());
        if ((rc = gmark(0))) return rc;
        // adjoint
        for (int c = 0; c < 6; c++) CK(cudaMemsetAsync(lam[c].p, 0, gF * h->esz, h->st));
        for (int a = 0; a < 3; a++)
            for (int w = 0; w < 2; w++) {
                CK(cudaMemsetAsync(lpe[a][w].p, 0, (size_t)G * psi_elems(h, h->su.se[a], a) * h->esz, h->st));
                CK(cudaMemsetAsync(lph[a][w].p, 0, (size_t)G * psi_elems(h, h->su.sh[a], a) * h->esz, h->st));
            }
        CK(cudaMemsetAsync(gacc.p, 0, gF * sizeof(double), h->st));
        AdjArgs<T> aa;
        memset(&aa, 0, sizeof(aa));
        aa.m = h->m.as<T>();
        aa.dtmu = h->has_mu ? h->dtmu.as<T>() : nullptr;
        aa.dtmu0 = (T)(h->ph.dt / h->ph.mu0);
        aa.prof = h->prof.as<T>();
        aa.nmax = h->su.nmax;
        aa.nx = h->g.nx; aa.ny = h->g.ny; aa.nz = h->g.nz; aa.px = h->px;
        aa.plane = h->plane; aa.fshot = h->fshot;
        aa.c1 = (T)h->ph.c1; aa.c2 = (T)h->ph.c2; aa.c2t = (T)(h->ph.psi_hyx_typo ? h->ph.c2 : h->ph.c1);
        aa.inv2w0dt = 1.0 / (2.0 * h->ph.omega0 * h->ph.dt);
        for (int c = 0; c < 6; c++) aa.lam[c] = lam[c].as<T>();
        aa.grad = gacc.as<double>();
        AdjArgs<T> ah = aa, ae = aa;
        for (int ax = 0; ax < 3; ax++) {
            ah.pshot[ax] = (long long)psi_elems(h, h->su.sh[ax], ax);
            ae.pshot[ax] = (long long)psi_elems(h, h->su.se[ax], ax);
            ah.slab[ax] = to_dslab(h->su.sh[ax]);
            ae.slab[ax] = to_dslab(h->su.se[ax]);
            ah.upd[ax] = to_dbox(h->su.upd[3 + ax]);
            ae.upd[ax] = to_dbox(h->su.upd[ax]);
            ah.ik[ax] = ae.ik[ax] = (T)(1.0 / (ax == 0 ? h->g.dx : (ax == 1 ? h->g.dy : h->g.dz)));
            // the forward's interior boxes (empty when the grid has none)
            ae.ibox.lo[ax] = h->has_ibox[0] ? h->ibox[0][ax] : 0;
            ae.ibox.hi[ax] = h->has_ibox[0] ? h->ibox[0][3 + ax] : 0;
            ah.ibox.lo[ax] = h->has_ibox[1] ? h->ibox[1][ax] : 0;
            ah.ibox.hi[ax] = h->has_ibox[1] ? h->ibox[1][3 + ax] : 0;
            for (int w = 0; w < 2; w++) { ah.lpsi[ax][w] = lph[ax][w].as<T>(); ae.lpsi[ax][w] = lpe[ax][w].as<T>(); }
        }
        ah.sgn = (T)h->ph.h_sign;
        ae.sgn = (T)h->ph.e_sign;
        for (int c = 0; c < 7; c++) { ah.mu[c] = mu[c].as<T>(); ae.mu[c] = mu[c].as<T>(); }
        const dim3 ablk(32, 8), agrd((h->g.nx + 31) / 32, (h->g.ny + 7) / 8, h->g.nz * Gg);
        // gathers: AVX x cells per thread (MITTET_ADJ_GATHER=cell: one per
        // thread, bit-identical)
        constexpr int AVX = sizeof(T) == 4 ? 4 : 2;
        const char *gmode = std::getenv("MITTET_ADJ_GATHER");
        const bool gather_cell = gmode && std::string(gmode) == "cell";
        // own kernels per part of the forward's boxes (MITTET_ADJ_OWN=cell:
        // one kernel over every cell with run-time CPML tests, bit-identical)
        const char *omode = std::getenv("MITTET_ADJ_OWN");
        const bool own_cell = omode && std::string(omode) == "cell";
        const dim3 vblk(32, 4), vgrd((h->g.nx + 32 * AVX - 1) / (32 * AVX), (h->g.ny + 3) / 4, h->g.nz * Gg);
        const T *H = hist.as<T>();
        const size_t slot = 6 * gF;
        for (int seg = ncheck - 1; seg >= 0; seg--) {
            const int n0 = seg * K, n1 = std::min(nt, n0 + K);
            if (!hm && !std::getenv("MITTET_GRAD_COPY")) {
                // Each recomputed step reads history slot q and writes slot
                // q + 1 (the phases' outputs go straight to the next slot; the
                // electric injection lands on the new E), so no copies.  With
                // magnetic sources the injection changes the step's input H,
                // which the history keeps as it was before it: copy instead.
                // MITTET_GRAD_COPY forces the copying path (same results).
                T *slot_f[6];
                for (int c = 0; c < 6; c++) slot_f[c] = hist.as<T>() + c * gF;
                if ((rc = load_state(ck.as<char>() + (size_t)seg * ck_stride, slot_f))) return rc;
                if ((rc = set_step(n0))) return rc;
                for (int q = 0; q < n1 - n0; q++) {
                    T *in = hist.as<T>() + (size_t)q * slot, *out = hist.as<T>() + (size_t)(q + 1) * slot;
                    PhaseArgs<T> eq = ea, hq = ha;
                    for (int c = 0; c < 6; c++) {
                        eq.f[c] = eq.fo[c] = in + c * gF;
                        hq.f[c] = hq.fo[c] = (c < 3 ? out : in) + c * gF;
                    }
                    for (int c = 0; c < 3; c++) {
                        eq.fo[c] = out + c * gF;
                        hq.fo[3 + c] = out + (3 + c) * gF;
                    }
                    InjectArgs<T> iq = ia_e;
                    for (int c = 0; c < 6; c++) iq.f[c] = out + c * gF;
                    launch_phase<T>(h, true, h->var_e, eq);
                    if (h->has_ele) inject_kernel<T><<<1, 128, 0, h->st>>>(iq);
                    launch_phase<T>(h, false, h->var_h, hq);
                    sample_kernel<T><<<1, 32, 0, h->st>>>(sa);
                }
            } else {
                if ((rc = load_state(ck.as<char>() + (size_t)seg * ck_stride, nullptr))) return rc;
                if ((rc = set_step(n0))) return rc;
                const dim3 cgrid(148 * 2, 6);
                copy_state_kernel<T><<<cgrid, 256, 0, h->st>>>(fl[0].as<T>(), fl[1].as<T>(), fl[2].as<T>(),
                                                              fl[3].as<T>(), fl[4].as<T>(), fl[5].as<T>(), hist.as<T>(),
                                                              (long long)gF);
                for (int q = 0; q < n1 - n0; q++) {
                    fwd_step(false);
                    copy_state_kernel<T><<<cgrid, 256, 0, h->st>>>(fl[0].as<T>(), fl[1].as<T>(), fl[2].as<T>(),
                                                                  fl[3].as<T>(), fl[4].as<T>(), fl[5].as<T>(),
                                                                  hist.as<T>() + (size_t)(q + 1) * slot, (long long)gF);
                }
            }
            CK(cudaGetLastError());
            if ((rc = gmark(1))) return rc;
            for (int n = n1 - 1; n >= n0; n--) {
                const int q = n - n0;
                for (int c = 0; c < 3; c++) {
                    ah.E0[c] = ae.E0[c] = H + (size_t)q * slot + c * gF;
                    ah.H0[c] = ae.H0[c] = H + (size_t)q * slot + (3 + c) * gF;
                    ah.E1[c] = ae.E1[c] = H + (size_t)(q + 1) * slot + c * gF;
                    ah.H1[c] = ae.H1[c] = H + (size_t)(q + 1) * slot + (3 + c) * gF;
                }
                const double *asrc = d_asrc.as<double>() + (size_t)s0 * nrec * nt;
                adj_inject_kernel<T><<<4, 256, 0, h->st>>>(aa.lam[0], aa.lam[1], aa.lam[2], aa.lam[3], aa.lam[4],
                                                          aa.lam[5], h->rec_off.as<long long>(), h->rec_comp.as<int>(),
                                                          nrec, Gg, h->fshot, asrc, nt, n, 1);
                if (hm) adj_src_kernel<T><<<(int)(asp.size() + 63) / 64, 64, 0, h->st>>>(ah, d_asp.as<AdjSrc>(), (int)asp.size(), h->wave.as<double>(), n, 0, s0, s1);
                if (own_cell) adj_h_own_kernel<T><<<agrd, ablk, 0, h->st>>>(ah);
                else launch_adj_own<T>(h, false, ah, Gg);
                if (gather_cell) adj_h_gather_kernel<T><<<agrd, ablk, 0, h->st>>>(ah);
                else adjv_h_gather_kernel<T, AVX><<<vgrd, vblk, 0, h->st>>>(ah);
                adj_inject_kernel<T><<<4, 256, 0, h->st>>>(aa.lam[0], aa.lam[1], aa.lam[2], aa.lam[3], aa.lam[4],
                                                          aa.lam[5], h->rec_off.as<long long>(), h->rec_comp.as<int>(),
                                                          nrec, Gg, h->fshot, asrc, nt, n, 0);
                if (he) adj_src_kernel<T><<<(int)(asp.size() + 63) / 64, 64, 0, h->st>>>(ae, d_asp.as<AdjSrc>(), (int)asp.size(), h->wave.as<double>(), n, 1, s0, s1);
                if (own_cell) adj_e_own_kernel<T><<<agrd, ablk, 0, h->st>>>(ae);
                else launch_adj_own<T>(h, true, ae, Gg);
                if (gather_cell) adj_e_gather_kernel<T><<<agrd, ablk, 0, h->st>>>(ae);
                else adjv_e_gather_kernel<T, AVX><<<vgrd, vblk, 0, h->st>>>(ae);
            }
            CK(cudaGetLastError());
            if ((rc = gmark(2))) return rc;
        }
        h->has_mag = mag0;
        h->has_ele = ele0;
        grad_reduce_kernel<<<512, 256, 0, h->st>>>(gacc.as<double>(), Gg, h->fshot, h->g.nx, h->g.ny, h->g.nz, h->px,
                                                   h->plane, h->g.ncpml, gred.as<double>());
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(gpart.data(), gred.p, ncell * sizeof(double), cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
        for (size_t e = 0; e < ncell; e++) gsum[e] += gpart[e];
    }
    h->nshot = ns_saved;
    h->vmask = (uint32_t)vmask_keep;
    drop_graph(h);
    int flag = 0;
    double mis = 0.0;
    CK(cudaMemcpyAsync(&flag, h->d_flag.p, sizeof(int), cudaMemcpyDeviceToHost, h->st));
    CK(cudaMemcpyAsync(&mis, d_mis.p, sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    if (glog)
        fprintf(stderr, "gradient stages (ms): checkpoint pass %.1f, recompute %.1f, adjoint %.1f\n", gms[0], gms[1],
                gms[2]);
    if (flag & 2) return fail(MITTET_ERR_DEVICE_TIMEOUT, "a bounded wait for a TMA copy gave up");
    if (flag & 4) return fail(MITTET_ERR_DEVICE_TIMEOUT, "a bounded grid-barrier wait of the persistent launch gave up");
    if (flag) return fail(MITTET_ERR_DIVERGED, "non-finite receiver samples (unstable time step or model)");
    *misfit_out = mis;
    memcpy(grad_out, gsum.data(), ncell * sizeof(double));
    return MITTET_OK;
}

template <typename T>
__global__ void model_kernel(const double *__restrict__ sig, const double *__restrict__ mu, int nx, int ny, int nz,
                             int px, double two_w0_dt, double dt, T *__restrict__ m, T *__restrict__ dtmu) {
    const long long n = (long long)nx * ny * nz;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % nx);
        const long long r = e / nx;
        const long long o = r * px + i;
        m[o] = (T)(two_w0_dt / sig[e]);
        if (mu) dtmu[o] = (T)(dt / mu[e]);
    }
}

template <typename S, typename T>
__global__ void model_kernel_dev(const S *__restrict__ sig, const S *__restrict__ mu, int nx, int ny, int nz, int px,
                                 double two_w0_dt, double dt, T *__restrict__ m, T *__restrict__ dtmu) {
    const long long n = (long long)nx * ny * nz;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % nx);
        const long long r = e / nx;
        const long long o = r * px + i;
        m[o] = (T)(two_w0_dt / (double)sig[e]);
        if (mu) dtmu[o] = (T)(dt / (double)mu[e]);
    }
}

// A device model's check (sig64 == nullptr: bit 0 of *bad when a
// conductivity, bit 1 when a permeability is not positive and finite) or its
// FP64 copy for the source gains.
template <typename T>
__global__ void model_stage_kernel(const T *__restrict__ sig, const T *__restrict__ mu, long long n,
                                   double *__restrict__ sig64, double *__restrict__ mu64, int *bad) {
    int b = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const double s = (double)sig[e];
        const double u = mu ? (double)mu[e] : 1.0;
        if (sig64) {
            sig64[e] = s;
            if (mu) mu64[e] = u;
        } else {
            b |= (!(s > 0.0) || !isfinite(s)) | ((!(u > 0.0) || !isfinite(u)) << 1);
        }
    }
    if (b) atomicOr(bad, b);
}

// sigma (which 0) or mu (which 1) at model cell c0 (x fastest, no padding):
// from the host copy of a host-set model, else from the device stage of a
// device-set one (one 8-byte read, for the few source cells).
double model_value(mittet_handle *h, int which, size_t c0) {
    const std::vector<double> &hv = which ? h->mu_h : h->sigma_h;
    if (!h->model_dev) return hv[c0];
    double v = 0.0;
    const DevBuf &d = which ? h->stage_mu : h->stage_sigma;
    cudaMemcpy(&v, d.as<double>() + c0, 8, cudaMemcpyDeviceToHost);
    return v;
}

}  // namespace

// ======================================================================= API

extern "C" {

int mittet_last_error(char *buf, size_t len) {
    if (buf && len) {
        strncpy(buf, g_err.c_str(), len - 1);
        buf[len - 1] = 0;
    }
    return (int)g_err.size();
}

int mittet_phys_defaults(int32_t flavor, mittet_phys *p) {
    if (!p) return fail(MITTET_ERR_INVALID_ARG, "null phys");
    memset(p, 0, sizeof(*p));
    p->flavor = flavor;
    p->c1 = 1.125;
    p->e_sign = 1;
    p->h_sign = 1;
    p->precision = MITTET_FP32;
    p->check_cfl = 1;
    if (flavor == MITTET_FLAVOR_NCVER0027) {
        // ncver0027/cpu_parameter_wafe.f90:30-32,40,84,123-132
        p->c2 = -0.04167;
        p->omega0 = 2.0 * 3.14159265358979 * 1.0;
        p->mu0 = 1.2566370614e-6;
        p->psi_hyx_typo = 1;
        p->cpml_nn = 3.0; p->cpml_order = 0.0; p->cpml_kappa_max = 1.0; p->cpml_a_max = 0.2;
        p->cpml_ma = 1.0; p->cpml_rcoef = 0.01; p->cpml_opt_to_max_x = 1.0;
    } else if (flavor == MITTET_FLAVOR_SATAN_I) {
        // satan_i/fwi3d_cpu_function_v1.4.c:1187, fwi3d_cpu_alloli1_v1.4.h:3, cpmlabc.c:12-23
        p->c2 = (double)-0.04167f;
        p->omega0 = 2.0 * M_PI;
        p->mu0 = 12.5663706e-7;
        p->psi_hyx_typo = 0;
        p->cpml_nn = 3.0; p->cpml_order = 0.0; p->cpml_kappa_max = 1.0; p->cpml_a_max = (double)0.2f;
        p->cpml_ma = 1.0; p->cpml_rcoef = (double)0.01f; p->cpml_opt_to_max_x = 10.0;
    } else {
        return fail(MITTET_ERR_INVALID_ARG, "unknown flavor %d", flavor);
    }
    return MITTET_OK;
}

double mittet_reference_dt(int32_t flavor, const mittet_grid *g, double cmax) {
    if (!g || cmax <= 0) return 0.0;
    if (flavor == MITTET_FLAVOR_SATAN_I) {
        const double courant = 1.0 / cmax / std::sqrt(1.0 / (g->dx * g->dx) + 1.0 / (g->dy * g->dy) + 1.0 / (g->dz * g->dz));
        return courant * 6.0 / 7.0 * (double)0.999f;
    }
    return 0.999 * g->dx / cmax / std::sqrt(3.0) / 1.16667;
}

int mittet_freq_grid_ref(int32_t nt, double dt, int32_t nf, double *omega) {
    if (nt <= 0 || dt <= 0 || nf < 0 || (!omega && nf)) return fail(MITTET_ERR_INVALID_ARG, "bad freq grid args");
    const double om = 2.0 * 3.14159265358979 / (double)nt / dt;
    for (int k = 0; k < nf; k++) omega[k] = om * k;
    return MITTET_OK;
}

int mittet_create(const mittet_grid *g, const mittet_phys *ph, mittet_handle **out) {
    if (!g || !ph || !out) return fail(MITTET_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    if (g->nx < 8 || g->ny < 8 || g->nz < 8) return fail(MITTET_ERR_INVALID_ARG, "grid must be at least 8 cells per axis");
    if (g->ncpml < 2 || 2 * g->ncpml + 4 > std::min(g->nx, std::min(g->ny, g->nz)))
        return fail(MITTET_ERR_INVALID_ARG, "ncpml %d does not fit the grid", g->ncpml);
    if (!(g->dx > 0 && g->dy > 0 && g->dz > 0)) return fail(MITTET_ERR_INVALID_ARG, "cell sizes must be positive");
    if (!(ph->dt > 0 && ph->omega0 > 0 && ph->cmax > 0 && ph->mu0 > 0))
        return fail(MITTET_ERR_INVALID_ARG, "dt, omega0, cmax and mu0 must be positive");
    if (ph->flavor != MITTET_FLAVOR_NCVER0027 && ph->flavor != MITTET_FLAVOR_SATAN_I)
        return fail(MITTET_ERR_INVALID_ARG, "unknown flavor %d", ph->flavor);
    if (ph->precision != MITTET_FP32 && ph->precision != MITTET_FP64)
        return fail(MITTET_ERR_INVALID_ARG, "precision must be MITTET_FP32 or MITTET_FP64");
    if (ph->check_cfl) {
        // Taylor (2,4) limit, ncver0027/cpu_set_condition.f90:279,285
        const double dmin = std::min(g->dx, std::min(g->dy, g->dz));
        const double taylor_dt = dmin / ph->cmax / std::sqrt(3.0) / 1.16667;
        if (ph->dt > taylor_dt * (1.0 + 1e-12))
            return fail(MITTET_ERR_CFL, "dt %.6e exceeds the (2,4) Taylor limit %.6e", ph->dt, taylor_dt);
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return fail(MITTET_ERR_CUDA, "no CUDA device available");
    }
    if (ph->device < 0 || ph->device >= ndev) return fail(MITTET_ERR_INVALID_ARG, "device %d out of range", ph->device);

    mittet_handle *h = new mittet_handle();
    h->g = *g;
    h->ph = *ph;
    h->fp64 = ph->precision == MITTET_FP64;
    h->esz = h->fp64 ? 8 : 4;
    // MITTET_TMA_SPIN_LIMIT=<polls> shortens the bounded waits of the TMA
    // interior, so that a test can make them give up (MITTET_ERR_DEVICE_TIMEOUT)
    if (const char *sl = std::getenv("MITTET_TMA_SPIN_LIMIT")) h->tma_spin = std::max(0, std::atoi(sl));
    h->px = (g->nx + 31) / 32 * 32;
    h->plane = (long long)h->px * g->ny;
    h->fshot = h->plane * g->nz;
    if (h->fshot >= (1LL << 31) - 64) {
        const long long cells = h->fshot;
        delete h;
        return fail(MITTET_ERR_INVALID_ARG, "grid of %lld padded cells exceeds the 2^31 per-shot limit", cells);
    }
    CpmlConst cc{ph->cpml_nn, ph->cpml_order, ph->cpml_kappa_max, ph->cpml_a_max, ph->cpml_ma, ph->cpml_rcoef,
                 ph->cpml_opt_to_max_x};
    build_setup(ph->flavor, g->nx, g->ny, g->nz, g->dx, g->dy, g->dz, g->ncpml, ph->cmax, ph->dt, cc, h->su);
    if (!ranges_in_bounds(h->su)) {
        delete h;
        return fail(MITTET_ERR_INVALID_ARG, "grid too small for the flavour's index ranges");
    }
    int rc = set_device(h);
    if (rc) { delete h; return rc; }
    if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return fail(MITTET_ERR_CUDA, "stream creation failed");
    }
    // profiles in the field precision
    const size_t np = h->su.prof.size();
    cudaError_t e = h->prof.ensure(np * h->esz);
    if (e == cudaSuccess) {
        if (h->fp64) {
            e = cudaMemcpy(h->prof.p, h->su.prof.data(), np * 8, cudaMemcpyHostToDevice);
        } else {
            std::vector<float> pf(np);
            for (size_t q = 0; q < np; q++) pf[q] = (float)h->su.prof[q];
            e = cudaMemcpy(h->prof.p, pf.data(), np * 4, cudaMemcpyHostToDevice);
        }
    }
    if (e != cudaSuccess) {
        cudaStreamDestroy(h->st);
        delete h;
        return fail(e == cudaErrorMemoryAllocation ? MITTET_ERR_OOM : MITTET_ERR_CUDA, "profile upload: %s",
                    cudaGetErrorString(e));
    }
    int rc2 = h->fp64 ? upload_tilemaps<double>(h) : upload_tilemaps<float>(h);
    if (rc2) {
        cudaStreamDestroy(h->st);
        delete h;
        return rc2;
    }
    *out = h;
    return MITTET_OK;
}

void mittet_destroy(mittet_handle *h) {
    if (!h) return;
    cudaSetDevice(h->ph.device);
    drop_graph(h);
    if (h->st) cudaStreamSynchronize(h->st);
    for (int p = 0; p < kParts; p++) {
        if (h->pst[p]) cudaStreamDestroy(h->pst[p]);
        if (h->ev_join[p]) cudaEventDestroy(h->ev_join[p]);
    }
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
}

int mittet_set_model(mittet_handle *h, const double *sigma, const double *mu) {
    if (!h || !sigma) return fail(MITTET_ERR_INVALID_ARG, "null argument");
    int rc = set_device(h);
    if (rc) return rc;
    const size_t n = (size_t)h->g.nx * h->g.ny * h->g.nz;
    for (size_t q = 0; q < n; q++)
        if (!(sigma[q] > 0) || !std::isfinite(sigma[q]))
            return fail(MITTET_ERR_INVALID_ARG, "sigma[%zu] = %g is not a positive finite conductivity", q, sigma[q]);
    if (mu)
        for (size_t q = 0; q < n; q++)
            if (!(mu[q] > 0) || !std::isfinite(mu[q]))
                return fail(MITTET_ERR_INVALID_ARG, "mu[%zu] = %g is not positive and finite", q, mu[q]);
    h->sigma_h.assign(sigma, sigma + n);
    if (mu) h->mu_h.assign(mu, mu + n); else h->mu_h.clear();
    h->model_dev = false;
    DevBuf &ds = h->stage_sigma, &dm = h->stage_mu;
    CK(ds.ensure(n * 8));
    CK(cudaMemcpyAsync(ds.p, sigma, n * 8, cudaMemcpyHostToDevice, h->st));
    if (mu) {
        CK(dm.ensure(n * 8));
        CK(cudaMemcpyAsync(dm.p, mu, n * 8, cudaMemcpyHostToDevice, h->st));
    }
    const size_t cb = (size_t)h->fshot * h->esz;
    const void *m0 = h->m.p, *dm0 = h->dtmu.p;
    CK(h->m.ensure(cb));
    CK(cudaMemsetAsync(h->m.p, 0, cb, h->st));
    if (mu) {
        CK(h->dtmu.ensure(cb));
        CK(cudaMemsetAsync(h->dtmu.p, 0, cb, h->st));
    }
    // the step graph reads the model words at run time: it stays valid while
    // the buffers stay where they are and the permeability mode is unchanged
    if (h->m.p != m0 || h->dtmu.p != dm0 || h->has_mu != (mu != nullptr) || !h->has_model) drop_graph(h);
    const double k = 2.0 * h->ph.omega0 * h->ph.dt;
    if (h->fp64)
        model_kernel<double><<<1024, 256, 0, h->st>>>(ds.as<double>(), mu ? dm.as<double>() : nullptr, h->g.nx, h->g.ny,
                                                      h->g.nz, h->px, k, h->ph.dt, h->m.as<double>(),
                                                      mu ? h->dtmu.as<double>() : nullptr);
    else
        model_kernel<float><<<1024, 256, 0, h->st>>>(ds.as<double>(), mu ? dm.as<double>() : nullptr, h->g.nx, h->g.ny,
                                                     h->g.nz, h->px, k, h->ph.dt, h->m.as<float>(),
                                                     mu ? h->dtmu.as<float>() : nullptr);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->st));
    h->has_model = true;
    h->has_mu = mu != nullptr;
    return upload_sources(h);
}

int mittet_set_model_device(mittet_handle *h, const void *sigma, const void *mu, int32_t is_fp64) {
    if (!h || !sigma) return fail(MITTET_ERR_INVALID_ARG, "null argument");
    int rc = set_device(h);
    if (rc) return rc;
    const size_t n = (size_t)h->g.nx * h->g.ny * h->g.nz;
    // the model stays on the device: a device-side check (a rejected model
    // leaves the handle's model as it was), then an FP64 stage that the
    // source gains read their few cells from; no host round trip
    CK(h->d_flag.ensure(sizeof(int)));
    CK(cudaMemsetAsync(h->d_flag.p, 0, sizeof(int), h->st));
    auto stage = [&](double *s64, double *m64) {
        if (is_fp64)
            model_stage_kernel<double><<<1024, 256, 0, h->st>>>((const double *)sigma, (const double *)mu, (long long)n,
                                                                s64, m64, h->d_flag.as<int>());
        else
            model_stage_kernel<float><<<1024, 256, 0, h->st>>>((const float *)sigma, (const float *)mu, (long long)n,
                                                               s64, m64, h->d_flag.as<int>());
    };
    stage(nullptr, nullptr);
    CK(cudaGetLastError());
    int bad = 0;
    CK(cudaMemcpyAsync(&bad, h->d_flag.p, sizeof(int), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    if (bad & 1) return fail(MITTET_ERR_INVALID_ARG, "sigma holds a conductivity that is not positive and finite");
    if (bad & 2) return fail(MITTET_ERR_INVALID_ARG, "mu holds a permeability that is not positive and finite");
    CK(h->stage_sigma.ensure(n * 8));
    if (mu) CK(h->stage_mu.ensure(n * 8));
    stage(h->stage_sigma.as<double>(), mu ? h->stage_mu.as<double>() : nullptr);
    CK(cudaGetLastError());
    h->sigma_h.clear();
    h->mu_h.clear();
    h->model_dev = true;
    const size_t cb = (size_t)h->fshot * h->esz;
    const void *m0 = h->m.p, *dm0 = h->dtmu.p;
    CK(h->m.ensure(cb));
    CK(cudaMemsetAsync(h->m.p, 0, cb, h->st));
    if (mu) {
        CK(h->dtmu.ensure(cb));
        CK(cudaMemsetAsync(h->dtmu.p, 0, cb, h->st));
    }
    if (h->m.p != m0 || h->dtmu.p != dm0 || h->has_mu != (mu != nullptr) || !h->has_model) drop_graph(h);
    const double k = 2.0 * h->ph.omega0 * h->ph.dt;
    // m = 2 w0 dt / sigma formed in FP64 from the given values, as set_model does
    auto launch = [&](auto *sg, auto *mg) {
        using S = std::remove_const_t<std::remove_pointer_t<decltype(sg)>>;
        if (h->fp64)
            model_kernel_dev<S, double><<<1024, 256, 0, h->st>>>(sg, mg, h->g.nx, h->g.ny, h->g.nz, h->px, k, h->ph.dt,
                                                                 h->m.as<double>(), mu ? h->dtmu.as<double>() : nullptr);
        else
            model_kernel_dev<S, float><<<1024, 256, 0, h->st>>>(sg, mg, h->g.nx, h->g.ny, h->g.nz, h->px, k, h->ph.dt,
                                                                h->m.as<float>(), mu ? h->dtmu.as<float>() : nullptr);
    };
    if (is_fp64)
        launch((const double *)sigma, (const double *)mu);
    else
        launch((const float *)sigma, (const float *)mu);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->st));
    h->has_model = true;
    h->has_mu = mu != nullptr;
    return upload_sources(h);
}

int mittet_set_sources(mittet_handle *h, int32_t nshot, int32_t npoint, const mittet_point_source *pts) {
    if (!h || nshot <= 0 || npoint <= 0 || !pts) return fail(MITTET_ERR_INVALID_ARG, "need at least one shot and point");
    for (int q = 0; q < npoint; q++) {
        const mittet_point_source &p = pts[q];
        if (p.shot < 0 || p.shot >= nshot) return fail(MITTET_ERR_INVALID_ARG, "point %d: shot %d out of range", q, p.shot);
        if (p.ix < 1 || p.ix > h->g.nx || p.iy < 1 || p.iy > h->g.ny || p.iz < 1 || p.iz > h->g.nz)
            return fail(MITTET_ERR_INVALID_ARG, "point %d: position (%d,%d,%d) outside the grid", q, p.ix, p.iy, p.iz);
        if (p.comp < 0 || p.comp > 5) return fail(MITTET_ERR_INVALID_ARG, "point %d: bad component", q);
        if (p.kind != MITTET_SRC_MAGNETIC && p.kind != MITTET_SRC_ELECTRIC)
            return fail(MITTET_ERR_INVALID_ARG, "point %d: bad kind", q);
        if (!std::isfinite(p.amp)) return fail(MITTET_ERR_INVALID_ARG, "point %d: amplitude not finite", q);
    }
    int rc = set_device(h);
    if (rc) return rc;
    if (h->nshot != nshot) drop_graph(h);  // the batch shape is baked into the graph and the tuning
    h->nshot = nshot;
    h->pts.assign(pts, pts + npoint);
    return upload_sources(h);
}

int mittet_set_wavelet(mittet_handle *h, int32_t nt, const double *w) {
    if (!h || nt <= 0 || !w) return fail(MITTET_ERR_INVALID_ARG, "bad wavelet");
    for (int q = 0; q <= nt; q++)
        if (!std::isfinite(w[q])) return fail(MITTET_ERR_INVALID_ARG, "wavelet sample %d not finite", q);
    int rc = set_device(h);
    if (rc) return rc;
    CK(h->wave.ensure((size_t)(nt + 1) * 8));
    CK(cudaMemcpy(h->wave.p, w, (size_t)(nt + 1) * 8, cudaMemcpyHostToDevice));
    h->nt_wave = nt;
    drop_graph(h);
    return MITTET_OK;
}

int mittet_set_receivers(mittet_handle *h, int32_t nrec, const mittet_receiver *rec) {
    if (!h || nrec < 0 || (nrec > 0 && !rec)) return fail(MITTET_ERR_INVALID_ARG, "bad receivers");
    std::vector<long long> off(std::max(nrec, 1));
    std::vector<int> comp(std::max(nrec, 1));
    std::vector<unsigned char> ish(std::max(nrec, 1));
    for (int r = 0; r < nrec; r++) {
        const mittet_receiver &q = rec[r];
        if (q.ix < 1 || q.ix > h->g.nx || q.iy < 1 || q.iy > h->g.ny || q.iz < 1 || q.iz > h->g.nz)
            return fail(MITTET_ERR_INVALID_ARG, "receiver %d outside the grid", r);
        if (q.comp < 0 || q.comp > 5) return fail(MITTET_ERR_INVALID_ARG, "receiver %d: bad component", r);
        off[r] = ((long long)(q.iz - 1) * h->g.ny + (q.iy - 1)) * h->px + (q.ix - 1);
        comp[r] = q.comp;
        ish[r] = q.comp >= 3;
    }
    if (nrec * (long long)std::max(h->nshot, 1) > (1 << 24)) return fail(MITTET_ERR_INVALID_ARG, "too many receivers");
    int rc = set_device(h);
    if (rc) return rc;
    CK(h->rec_off.ensure(off.size() * 8));
    CK(h->rec_comp.ensure(comp.size() * 4));
    CK(h->rec_is_h.ensure(ish.size()));
    CK(cudaMemcpy(h->rec_off.p, off.data(), off.size() * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->rec_comp.p, comp.data(), comp.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->rec_is_h.p, ish.data(), ish.size(), cudaMemcpyHostToDevice));
    h->nrec = nrec;
    h->recs.assign(rec, rec + nrec);
    drop_graph(h);
    return MITTET_OK;
}

int mittet_set_freqs(mittet_handle *h, int32_t nf, const double *omega, int32_t h_factor) {
    if (!h || nf < 0 || (nf > 0 && !omega)) return fail(MITTET_ERR_INVALID_ARG, "bad frequencies");
    for (int f = 0; f < nf; f++)
        if (!(omega[f] >= 0) || !std::isfinite(omega[f])) return fail(MITTET_ERR_INVALID_ARG, "omega[%d] invalid", f);
    int rc = set_device(h);
    if (rc) return rc;
    h->omega.assign(omega, omega + nf);
    h->hfac = h_factor ? 1 : 0;
    CK(h->d_omega.ensure(std::max(nf, 1) * 8));
    if (nf) CK(cudaMemcpy(h->d_omega.p, omega, nf * 8, cudaMemcpyHostToDevice));
    drop_graph(h);
    return MITTET_OK;
}

int mittet_set_volume_dft(mittet_handle *h, uint32_t comp_mask) {
    if (!h || comp_mask > 7) return fail(MITTET_ERR_INVALID_ARG, "comp_mask must select Ex/Ey/Ez bits only");
    if (comp_mask && h->omega.size() > 64) return fail(MITTET_ERR_INVALID_ARG, "volume DFT supports at most 64 frequencies");
    h->vmask = comp_mask;
    drop_graph(h);
    return MITTET_OK;
}

int mittet_forward(mittet_handle *h, int32_t nt, double *rec_fd, double *rec_td) {
    if (!h) return fail(MITTET_ERR_INVALID_ARG, "null handle");
    int rc = validate_ready(h, nt);
    if (rc) return rc;
    if (h->vmask && h->omega.empty()) return fail(MITTET_ERR_STATE, "volume DFT needs mittet_set_freqs first");
    rc = set_device(h);
    if (rc) return rc;
    rc = h->fp64 ? run_forward<double>(h, nt) : run_forward<float>(h, nt);
    if (rc) return rc;
    const int nf = (int)h->omega.size();
    const size_t ntr = (size_t)h->nshot * h->nrec;
    if (rec_fd && nf > 0 && ntr > 0)
        CK(cudaMemcpyAsync(rec_fd, h->spectra.p, ntr * nf * sizeof(double2), cudaMemcpyDeviceToHost, h->st));
    if (rec_td && ntr > 0) {
        if (h->fp64) {
            CK(cudaMemcpyAsync(rec_td, h->traces.p, ntr * nt * 8, cudaMemcpyDeviceToHost, h->st));
        } else {
            std::vector<float> tmp(ntr * nt);
            CK(cudaMemcpyAsync(tmp.data(), h->traces.p, ntr * nt * 4, cudaMemcpyDeviceToHost, h->st));
            CK(cudaStreamSynchronize(h->st));
            for (size_t q = 0; q < tmp.size(); q++) rec_td[q] = tmp[q];
        }
    }
    int flag = 0;
    CK(cudaMemcpyAsync(&flag, h->d_flag.p, sizeof(int), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    if (flag & 2) return fail(MITTET_ERR_DEVICE_TIMEOUT, "a bounded wait for a TMA copy gave up");
    if (flag & 4) return fail(MITTET_ERR_DEVICE_TIMEOUT, "a bounded grid-barrier wait of the persistent launch gave up");
    if (flag) return fail(MITTET_ERR_DIVERGED, "non-finite receiver samples (unstable time step or model)");
    return MITTET_OK;
}

int mittet_forward_device(mittet_handle *h, int32_t nt, void *rec_fd_dev, void *stream) {
    if (!h) return fail(MITTET_ERR_INVALID_ARG, "null handle");
    int rc = validate_ready(h, nt);
    if (rc) return rc;
    rc = set_device(h);
    if (rc) return rc;
    // the caller's stream; NULL is the legacy default stream, which the
    // handle's non-blocking stream does not synchronise with implicitly
    cudaStream_t user = stream ? (cudaStream_t)stream : cudaStreamLegacy;
    {
        cudaEvent_t ev;
        CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        CK(cudaEventRecord(ev, user));
        CK(cudaStreamWaitEvent(h->st, ev, 0));
        cudaEventDestroy(ev);
    }
    rc = h->fp64 ? run_forward<double>(h, nt) : run_forward<float>(h, nt);
    if (rc) return rc;
    const int nf = (int)h->omega.size();
    const size_t ntr = (size_t)h->nshot * h->nrec;
    if (rec_fd_dev && nf > 0 && ntr > 0)
        CK(cudaMemcpyAsync(rec_fd_dev, h->spectra.p, ntr * nf * sizeof(double2), cudaMemcpyDeviceToDevice, h->st));
    {
        cudaEvent_t ev;
        CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        CK(cudaEventRecord(ev, h->st));
        CK(cudaStreamWaitEvent(user, ev, 0));
        cudaEventDestroy(ev);
    }
    return MITTET_OK;
}

int mittet_get_volume_dft(mittet_handle *h, int32_t shot, int32_t comp, double *out) {
    if (!h || !out || shot < 0 || shot >= h->nshot || comp < 0 || comp > 2)
        return fail(MITTET_ERR_INVALID_ARG, "bad volume DFT request");
    if (!(h->vmask >> comp & 1) || !h->acc.p) return fail(MITTET_ERR_STATE, "component %d was not accumulated", comp);
    int rc = set_device(h);
    if (rc) return rc;
    const int nf = (int)h->omega.size();
    const double2 *base = h->acc.as<double2>() + (((size_t)shot * 3 + comp) * nf) * h->fshot;
    // strip the row padding: [f][nz][ny][px] -> [f][nz][ny][nx]
    CK(cudaMemcpy2DAsync(out, (size_t)h->g.nx * 16, base, (size_t)h->px * 16, (size_t)h->g.nx * 16,
                         (size_t)nf * h->g.nz * h->g.ny, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return MITTET_OK;
}

int mittet_get_fields(mittet_handle *h, int32_t shot, double *out) {
    if (!h || !out || shot < 0 || shot >= h->nshot || h->alloc_shots != h->nshot)
        return fail(MITTET_ERR_INVALID_ARG, "bad field request");
    int rc = set_device(h);
    if (rc) return rc;
    const size_t n = (size_t)h->g.nx * h->g.ny * h->g.nz;
    for (int c = 0; c < 6; c++) {
        const char *base = (const char *)h->fields[c].p + (size_t)shot * h->fshot * h->esz;
        if (h->fp64) {
            CK(cudaMemcpy2D(out + c * n, (size_t)h->g.nx * 8, base, (size_t)h->px * 8, (size_t)h->g.nx * 8,
                            (size_t)h->g.nz * h->g.ny, cudaMemcpyDeviceToHost));
        } else {
            std::vector<float> tmp(n);
            CK(cudaMemcpy2D(tmp.data(), (size_t)h->g.nx * 4, base, (size_t)h->px * 4, (size_t)h->g.nx * 4,
                            (size_t)h->g.nz * h->g.ny, cudaMemcpyDeviceToHost));
            for (size_t q = 0; q < n; q++) out[c * n + q] = tmp[q];
        }
    }
    return MITTET_OK;
}

int mittet_f_to_d(int32_t device, int32_t ntrace, int32_t nt, double dt, double omega0, const double *x, int32_t nf,
                  const double *omega, int32_t h_factor, double *out) {
    if (ntrace <= 0 || nt <= 0 || nf <= 0 || !x || !omega || !out || !(dt > 0) || !(omega0 > 0))
        return fail(MITTET_ERR_INVALID_ARG, "bad f_to_d arguments");
    CK(cudaSetDevice(device));
    DevBuf dx_, dom, dout, dish;
    CK(dx_.ensure((size_t)ntrace * nt * 8));
    CK(dom.ensure((size_t)nf * 8));
    CK(dout.ensure((size_t)ntrace * nf * 16));
    std::vector<unsigned char> ish(ntrace, h_factor ? 1 : 0);
    CK(dish.ensure(ntrace));
    CK(cudaMemcpy(dx_.p, x, (size_t)ntrace * nt * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dom.p, omega, (size_t)nf * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dish.p, ish.data(), ntrace, cudaMemcpyHostToDevice));
    trace_dft_kernel<double><<<nf, 256>>>(dx_.as<double>(), ntrace, nt, dom.as<double>(), nf, dt, omega0,
                                          dish.as<unsigned char>(), ntrace, h_factor ? 1 : 0, dout.as<double2>());
    CK(cudaGetLastError());
    CK(cudaMemcpy(out, dout.p, (size_t)ntrace * nf * 16, cudaMemcpyDeviceToHost));
    return MITTET_OK;
}

int64_t mittet_last_launch_count(mittet_handle *h) { return h ? h->launches : -1; }

int mittet_boundary_variant(mittet_handle *h, int32_t *e_variant, int32_t *h_variant) {
    if (!h || !e_variant || !h_variant) return fail(MITTET_ERR_INVALID_ARG, "null argument");
    *e_variant = h->merge_b[0];
    *h_variant = h->merge_b[1];
    return MITTET_OK;
}

int mittet_layout_variant(mittet_handle *h, int32_t *e_layout, int32_t *h_layout) {
    if (!h || !e_layout || !h_layout) return fail(MITTET_ERR_INVALID_ARG, "null argument");
    *e_layout = h->layout[0];
    *h_layout = h->layout[1];
    return MITTET_OK;
}

int mittet_band_variant(mittet_handle *h, int32_t *e_zc, int32_t *h_zc) {
    if (!h || !e_zc || !h_zc) return fail(MITTET_ERR_INVALID_ARG, "null argument");
    *e_zc = h->has_ibox[0] ? h->band[0] : 0;
    *h_zc = h->has_ibox[1] ? h->band[1] : 0;
    return MITTET_OK;
}

int mittet_persistent_variant(mittet_handle *h, int32_t *variant, int32_t *grid) {
    if (!h || !variant || !grid) return fail(MITTET_ERR_INVALID_ARG, "null argument");
    *variant = h->persist_decided ? h->persist_vi : -1;
    *grid = *variant >= 0 ? h->persist_grid : 0;
    return MITTET_OK;
}

int mittet_tuned_variant(mittet_handle *h, int32_t *e_cfg, int32_t *h_cfg) {
    if (!h || !e_cfg || !h_cfg) return fail(MITTET_ERR_INVALID_ARG, "null argument");
    int32_t all[2 * kParts * 4];
    int rc = mittet_tuned_variants(h, all);
    if (rc) return rc;
    for (int q = 0; q < 4; q++) {
        e_cfg[q] = all[q];
        h_cfg[q] = all[kParts * 4 + q];
    }
    return MITTET_OK;
}

int mittet_tuned_variants(mittet_handle *h, int32_t *cfg) {
    if (!h || !cfg) return fail(MITTET_ERR_INVALID_ARG, "null argument");
    auto fill = [&](auto tag) {
        using T = decltype(tag);
        for (int ph = 0; ph < 2; ph++)
            for (int p = 0; p < kParts; p++) {
                const int vi = (ph == 0 ? h->var_e : h->var_h)[p];
                int32_t *c = cfg + (ph * kParts + p) * 4;
                if (vi < 0) {  // TMA-staged interior: VX = 0, then the tile and z planes per CTA
                    c[0] = 0; c[1] = TmaShape<T>::TX; c[2] = TmaShape<T>::TY; c[3] = tma_cfgs<T>()[-1 - vi].zc;
                } else {
                    const auto &a = variants<T>()[vi];
                    c[0] = a.vx; c[1] = a.bx; c[2] = a.by; c[3] = a.bz > 0 ? -a.bz : (a.bz < 0 ? a.zc - 1000 * a.bz : a.zc);
                }
            }
    };
    if (h->fp64) fill(double());
    else fill(float());
    return MITTET_OK;
}

int mittet_stencil_variants(int32_t fp64, int32_t *count, int32_t *cfg, int32_t max) {
    if (!count || (max > 0 && !cfg)) return fail(MITTET_ERR_INVALID_ARG, "null argument");
    auto fill = [&](const auto &vs) {
        *count = (int32_t)vs.size();
        for (int v = 0; v < (int)vs.size() && v < max; v++) {
            int32_t *c = cfg + 4 * v;
            c[0] = vs[v].vx; c[1] = vs[v].bx; c[2] = vs[v].by;
            c[3] = vs[v].bz > 0 ? -vs[v].bz : (vs[v].bz < 0 ? vs[v].zc - 1000 * vs[v].bz : vs[v].zc);
        }
    };
    if (fp64) fill(variants<double>());
    else fill(variants<float>());
    return MITTET_OK;
}

int mittet_time_kernels(mittet_handle *h, int32_t nsteps, double *ms) {
    if (!h || !ms || nsteps <= 0) return fail(MITTET_ERR_INVALID_ARG, "bad timing request");
    if (h->last_nt < nsteps || h->alloc_shots != h->nshot)
        return fail(MITTET_ERR_STATE, "run a forward of at least %d steps first", nsteps);
    int rc = set_device(h);
    if (rc) return rc;
    rc = h->fp64 ? time_kernels<double>(h, nsteps, ms) : time_kernels<float>(h, nsteps, ms);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->st));
    return MITTET_OK;
}

int mittet_release_gradient_buffers(mittet_handle *h) {
    if (!h) return fail(MITTET_ERR_INVALID_ARG, "null handle");
    int rc = set_device(h);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->st));
    h->gb.release();
    return MITTET_OK;
}

int mittet_gradient(mittet_handle *h, int32_t nt, const double *obs, int32_t checkpoint_every, double *misfit,
                    double *grad) {
    if (!h || !obs || !misfit || !grad) return fail(MITTET_ERR_INVALID_ARG, "null argument");
    int rc = validate_ready(h, nt);
    if (rc) return rc;
    if (h->nrec <= 0 || h->omega.empty()) return fail(MITTET_ERR_STATE, "the gradient needs receivers and frequencies");
    for (double w : h->omega)
        if (!(w > 0)) return fail(MITTET_ERR_INVALID_ARG, "gradient frequencies must be positive");
    for (const auto &p : h->pts)
        if ((p.kind == MITTET_SRC_ELECTRIC) != (p.comp < 3))
            return fail(MITTET_ERR_INVALID_ARG, "gradient supports electric points on E and magnetic points on H");
    const int K = checkpoint_every > 0 ? checkpoint_every : 200;
    rc = set_device(h);
    if (rc) return rc;
    return h->fp64 ? run_gradient<double>(h, nt, obs, K, misfit, grad) : run_gradient<float>(h, nt, obs, K, misfit, grad);
}

int mittet_fwi_update(mittet_handle *h, int32_t nt, const double *obs, const double *ecal, const double *grad,
                      int32_t iseabed, double minval, double maxval, double *sigma, double *step) {
    if (!h || !obs || !ecal || !grad || !sigma || !step) return fail(MITTET_ERR_INVALID_ARG, "null argument");
    int rc = validate_ready(h, nt);
    if (rc) return rc;
    if (h->nrec <= 0 || h->omega.empty()) return fail(MITTET_ERR_STATE, "the update needs receivers and frequencies");
    if (!(minval <= maxval)) return fail(MITTET_ERR_INVALID_ARG, "minval must not exceed maxval");
    const int nx = h->g.nx, ny = h->g.ny, nz = h->g.nz, nc = h->g.ncpml;
    const size_t n = (size_t)nx * ny * nz;
    // calc_phi (satan_i/fwi3d_cpu_function_v1.4.c:2565-2603): maxima of sigma
    // and grad over k <= iseabed, starting from cell 0; trial sigma2.
    double sigmax2 = sigma[0], gradmax = grad[0];
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                const size_t ijk = ((size_t)k * ny + j) * nx + i;
                if (k <= iseabed) {
                    if (sigma[ijk] > sigmax2) sigmax2 = sigma[ijk];
                    if (grad[ijk] > gradmax) gradmax = grad[ijk];
                }
            }
    if (!(gradmax != 0.0) || !std::isfinite(gradmax))
        return fail(MITTET_ERR_INVALID_ARG, "largest gradient above the seabed is %g: no step scale", gradmax);
    const double scaler = (double)0.01f * sigmax2 / gradmax;
    std::vector<double> sig2(n);
    for (size_t q = 0; q < n; q++) sig2[q] = sigma[q] - scaler * grad[q];
    // trial forward of every shot (media_coeff_sig_tmp + fwdpropagation + laplaceToFreq_3)
    std::vector<double> mu_keep = h->mu_h;
    if (h->model_dev && h->has_mu) {  // a device-set permeability: bring it to the host once
        mu_keep.resize(n);
        CK(cudaMemcpy(mu_keep.data(), h->stage_mu.p, n * 8, cudaMemcpyDeviceToHost));
    }
    const double *mu = (h->has_mu && !mu_keep.empty()) ? mu_keep.data() : nullptr;
    rc = mittet_set_model(h, sig2.data(), mu);
    if (rc) return rc;
    const int nf = (int)h->omega.size();
    const size_t nspec = (size_t)h->nshot * h->nrec * nf;
    std::vector<double> e2(2 * nspec);
    const uint32_t vmask_saved = h->vmask;
    if (h->vmask) { h->vmask = 0; drop_graph(h); }
    rc = mittet_forward(h, nt, e2.data(), nullptr);
    h->vmask = vmask_saved;
    if (vmask_saved) drop_graph(h);
    if (rc) return rc;
    // calc_alpha (function.c:2757-2785): k1 = sum dE (E2 - Ecal), k2 = sum (E2 - Ecal)^2
    std::complex<double> k1 = 0.0, k2 = 0.0;
    for (size_t q = 0; q < nspec; q++) {
        const std::complex<double> d(obs[2 * q] - ecal[2 * q], obs[2 * q + 1] - ecal[2 * q + 1]);
        const std::complex<double> c(e2[2 * q] - ecal[2 * q], e2[2 * q + 1] - ecal[2 * q + 1]);
        k1 += d * c;
        k2 += c * c;
    }
    if (!(std::abs(k2) > 0)) return fail(MITTET_ERR_INVALID_ARG, "trial model changes no receiver value (k2 = 0)");
    // update_para2 (function.c:2787-2832)
    const double alpha = 3.0f * std::abs(k1) / std::abs(k2);
    for (int k = nc; k < nz - nc; k++)
        for (int j = nc; j < ny - nc; j++)
            for (int i = nc; i < nx - nc; i++) {
                const size_t ijk = ((size_t)k * ny + j) * nx + i;
                if (k <= iseabed) sigma[ijk] += alpha * scaler * grad[ijk];
                if (sigma[ijk] < minval) sigma[ijk] = minval;
                if (sigma[ijk] > maxval) sigma[ijk] = maxval;
            }
    step[0] = scaler;
    step[1] = alpha;
    return mittet_set_model(h, sigma, mu);
}

}  // extern "C"
