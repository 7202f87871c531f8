// kernels.cuh -- sm_100a kernels of the Mittet fictitious-wave FDTD step.
//
// One time step of one batch of shots runs on one stream:
//   inject_kernel (magnetic points, before E)   ncver0027/cpu_waveform.f90:46-50
//   E phase: e_part_kernel x 5 (interior, x/y/z faces, edges) or
//            interior_tma_kernel for the interior
//                   E update + CPML psi_E        cpu_eh_field_cpml42.f90:114-158, cpu_cpml4.f90:271-361
//   inject_kernel (electric points, after E)    satan_i/fwi3d_cpu_function_v1.4.c:526-527
//   H phase: h_part_kernel x 5 / interior_tma_kernel
//                   H update + CPML psi_H        cpu_eh_field_cpml42.f90:210-253, cpu_cpml4.f90:384-474
//   sample_kernel   receiver gather + step++     cpu_output.f90:20-30
// and every 128 steps volume_dft_kernel folds the E ring into the spectra.
// The step index lives in device memory (d_step) so a block of steps can be
// captured once in a CUDA graph and replayed.
//
// Layout in HBM: every field component is one array [shot][nz][ny][px]
// (px = nx rounded up to 32 elements so rows start 128-byte aligned).  The
// model is one word per cell, m = dt/eps' = 2 w0 dt / sigma (the interior cb),
// plus dt/mu per cell only when a permeability volume is given.  CPML psi
// variables exist only inside their slabs (compact [shot][...] boxes).
//
// The half-step kernels are in stencil.cuh and tma_interior.cuh.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mittet {

struct DBox {
    int lo[3], hi[3];
};
struct DSlab {
    int nlo, nhi, flo, fhi, width, fofs;  // see Slab (setup_host.h)
    DBox other;
};

template <typename T>
struct PhaseArgs {
    T *f[6];                // Ex Ey Ez Hx Hy Hz, shot 0: the phase's inputs
    T *fo[6];               // where the phase writes its own three fields (= f: in place)
    T *psi[3][2];           // psi of this phase's slab groups (axis, which)
    const T *m;             // per-cell 2 w0 dt / sigma
    const T *dtmu;          // per-cell dt/mu or nullptr
    T dtmu0;                // dt/mu0 when dtmu == nullptr
    const T *prof;          // [3][P_COUNT][nmax]
    int nmax;
    int nx, ny, nz, px;
    long long plane;        // px * ny
    long long fshot;        // nz * plane
    long long pshot[3];     // psi elements per shot per slab axis
    DBox upd[3];            // update boxes of the three components of this phase
    DSlab slab[3];          // slab groups of this phase (x, y, z)
    T c1, c2, c2t;          // stencil weights; c2t = c2 (psi_Hyx typo) or c1
    T sgn;                  // +1 / -1 ("bp" updates)
    T ik[3];                // 1/d per axis: the 1/ked (1/khd) value of every interior cell
    // full-volume DFT ring (E phase only), see ring_index
    T *ring;
    int ring_k;             // ring depth K (0 = no ring)
    int vmask;              // E components written to the ring
    long long ring_comp;    // elements per (slot, vcomp): ring_comp_of(nshot * fshot)
    const int *d_step;
};

// Ring layout [vcomp][tile of kRingTile cells][slot][kRingTile]: one step's
// values of a tile are kRingTile * 4 contiguous bytes (E-phase writes), and
// the ring_k steps of a tile are one contiguous block (flush reads).  Tiles
// shorter than about 256 cells cost the E phase DRAM write efficiency (the
// per-step pieces land ring_k * tile apart).  e = shot * fshot + cell
// (padded layout); ring_comp = nshot * fshot rounded up to whole tiles.
#ifndef MITTET_RING_TILE
#define MITTET_RING_TILE 256
#endif
constexpr int kRingTile = MITTET_RING_TILE;
static_assert(kRingTile >= 32 && (kRingTile & (kRingTile - 1)) == 0, "ring tile: a power of two, >= 32 cells");
__host__ __device__ __forceinline__ long long ring_comp_of(long long cells) {
    return (cells + kRingTile - 1) / kRingTile * kRingTile;
}
__device__ __forceinline__ long long ring_index(long long ring_comp, int K, int vc, long long e, int slot) {
    return (long long)vc * ring_comp * K + (e & ~(long long)(kRingTile - 1)) * K + (long long)slot * kRingTile +
           (e & (kRingTile - 1));
}

__device__ __forceinline__ bool in_box(const DBox &b, int i, int j, int k) {
    return i >= b.lo[0] && i < b.hi[0] && j >= b.lo[1] && j < b.hi[1] && k >= b.lo[2] && k < b.hi[2];
}

// Local index along the slab axis, or -1 if v is in neither interval.
__device__ __forceinline__ int slab_local(const DSlab &s, int v) {
    if (v >= s.nlo && v < s.nhi) return v - s.nlo;
    if (v >= s.flo && v < s.fhi) return s.fofs + (v - s.flo);
    return -1;
}

template <typename T>
__device__ __forceinline__ T ldg(const T *p) {
    return __ldg(p);
}

template <typename T>
__device__ __forceinline__ T rcp(T x);
template <>
__device__ __forceinline__ float rcp<float>(float x) {
    return __frcp_rn(x);
}
template <>
__device__ __forceinline__ double rcp<double>(double x) {
    return 1.0 / x;
}

// Profile value of one axis.
template <typename T>
__device__ __forceinline__ T pv(const PhaseArgs<T> &a, int axis, int which, int i) {
    return ldg(a.prof + ((size_t)axis * 8 + which) * a.nmax + i);
}

}  // namespace mittet

#include "stencil.cuh"

namespace mittet {

// ---------------------------------------------------------- point sources
struct SrcPoint {
    long long off;  // shot * fshot + cell offset (padded layout)
    int comp;
    int kind;       // 0 magnetic (uses w[n+1]), 1 electric (uses (w[n]+w[n+1])/2)
    double g;       // amp * dt/mu/(dx dy dz)  or  amp * dt * 2 w0/sigma/(dx dy dz)
};

template <typename T>
struct InjectArgs {
    T *f[6];
    const SrcPoint *pts;
    int npts;
    int kind;
    const double *wave;  // w[0..nt]
    const int *d_step;
    T *ring;             // full-volume ring or nullptr
    int ring_k, vmask;
    long long ring_comp;
};

template <typename T>
__global__ void inject_kernel(InjectArgs<T> a) {
    const int n = *a.d_step;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < a.npts; p += gridDim.x * blockDim.x) {
        const SrcPoint s = a.pts[p];
        if (s.kind != a.kind) continue;
        const double w = s.kind == 0 ? a.wave[n + 1] : (a.wave[n] + a.wave[n + 1]) / 2.0;
        T *cell = a.f[s.comp] + s.off;
        const T v = atomicAdd(cell, (T)(-s.g * w)) + (T)(-s.g * w);
        if (a.ring && s.comp < 3 && (a.vmask >> s.comp & 1)) {
            const int slot = n % a.ring_k;
            a.ring[ring_index(a.ring_comp, a.ring_k, s.comp, s.off, slot)] = v;
        }
    }
}

// ---------------------------------------------------------------- sampling
template <typename T>
struct SampleArgs {
    const T *f[6];
    const long long *rec_off;  // cell offsets (padded layout, shot 0)
    const int *rec_comp;
    int nrec, nshot;
    long long fshot;
    T *traces;                 // [shot][rec][nt]
    int nt;
    int *d_step;
};

// One block: every thread reads d_step, gathers, then thread 0 advances it.
template <typename T>
__global__ void sample_kernel(SampleArgs<T> a) {
    const int n = *a.d_step;
    const int tot = a.nrec * a.nshot;
    for (int q = threadIdx.x; q < tot; q += blockDim.x) {
        const int s = q / a.nrec, r = q % a.nrec;
        a.traces[(long long)q * a.nt + n] = a.f[a.rec_comp[r]][(long long)s * a.fshot + a.rec_off[r]];
    }
    __syncthreads();
    if (threadIdx.x == 0) *a.d_step = n + 1;
}

// ---------------------------------------------------------- f_to_d (traces)
//
// X(w_f) = sum_n x[n] dt exp((i-1) sqrt(w0 w_f) n dt), times sqrt(-2 w0/(i w_f))
// for H traces when hfac is set (cpu_f_to_d_e.f90:140-148, cpu_f_to_d_h.f90:146-148).
// Trace t is receiver t % nrec_h of its shot (is_h has nrec_h entries).
// Block = one frequency; threads stride over traces; the weights of a chunk
// of time samples are computed once per block into shared memory in FP64.
template <typename T>
__global__ void trace_dft_kernel(const T *__restrict__ x, int ntrace, int nt, const double *__restrict__ omega,
                                 int nf, double dt, double omega0, const unsigned char *__restrict__ is_h, int nrec_h,
                                 int hfac, double2 *__restrict__ out) {
    constexpr int CH = 256;
    __shared__ double2 w[CH];
    const int f = blockIdx.x;
    if (f >= nf) return;
    const double sw = sqrt(omega0 * omega[f]);
    double2 hf = make_double2(1.0, 0.0);
    if (hfac) {
        // sqrt(-2 w0/(i w)) = sqrt(2 w0/w) * exp(i pi/4)  (principal branch)
        const double r = sqrt(2.0 * omega0 / omega[f]);
        hf = make_double2(r * 0.70710678118654752440, r * 0.70710678118654752440);
    }
    for (int t0 = 0; t0 < ntrace; t0 += blockDim.x) {
        const int t = t0 + threadIdx.x;
        double re = 0.0, im = 0.0;
        for (int n0 = 0; n0 < nt; n0 += CH) {
            __syncthreads();
            for (int q = threadIdx.x; q < CH && n0 + q < nt; q += blockDim.x) {
                const double xa = sw * (double)(n0 + q) * dt;
                double s, c;
                sincos(xa, &s, &c);
                const double e = exp(-xa) * dt;
                w[q] = make_double2(e * c, e * s);
            }
            __syncthreads();
            if (t < ntrace) {
                const T *xt = x + (long long)t * nt + n0;
                const int cnt = min(CH, nt - n0);
                for (int q = 0; q < cnt; q++) {
                    const double v = (double)xt[q];
                    re += v * w[q].x;
                    im += v * w[q].y;
                }
            }
        }
        if (t < ntrace) {
            if (hfac && is_h && is_h[t % nrec_h]) {
                const double r2 = re * hf.x - im * hf.y, i2 = re * hf.y + im * hf.x;
                re = r2;
                im = i2;
            }
            out[(long long)t * nf + f] = make_double2(re, im);
        }
    }
}

// ---------------------------------------------------- full-volume f_to_d
//
// Every ring_k (= 128) steps the E phase has left the last values of each
// selected E component in the ring; this kernel folds them into the FP64
// accumulators:
//   acc[shot][vc][f][cell] += sum_{s<cnt} wt[n0+s][f] * ring(vc, shot*fshot + cell, s),
//   wt[n][f] = dt exp((i-1) sqrt(w0 w_f) n dt)  (cpu_f_to_d_e.f90:140-142).
// Grid (cells, component, shot), one thread per cell.  A thread issues the
// ring loads of a chunk of 64 (FP32) or 32 (FP64) steps (one 128-byte line
// per warp each) before that chunk's arithmetic and forms every product and
// partial sum in FP64 (the ring samples are exact in FP64, the weights are
// FP64), so the whole
// transform is accumulated in FP64 whatever the field precision: the FP32
// path's only DFT error is the rounding of the field samples themselves.  The
// weights of one group of up to four frequencies are a by-value kernel
// parameter (8 KB; zero for s >= cnt), so every multiply reads its weight
// from the constant bank.  A ring of 128 steps reads and writes the
// accumulators half as often as one of 64, for twice the ring memory.
constexpr int kFlushRing = 128;
constexpr int kFlushFreqs = 4;
struct FlushWeights {
    double wr[kFlushRing][kFlushFreqs];
    double wi[kFlushRing][kFlushFreqs];
};

template <typename T>
__global__ void __launch_bounds__(256) volume_dft_kernel(const T *__restrict__ ring, long long ring_comp, int ring_k,
                                                         int3 vcs, long long fshot, int cnt, int f0, int nf,
                                                         const __grid_constant__ FlushWeights w,
                                                         double2 *__restrict__ acc) {
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= fshot) return;
    const int vi = blockIdx.y, shot = blockIdx.z;
    const int vc = vi == 0 ? vcs.x : (vi == 1 ? vcs.y : vcs.z);
    const long long e = (long long)shot * fshot + cell;
    const T *__restrict__ rp = ring + ring_index(ring_comp, ring_k, vc, e, 0);
    constexpr int kFlushChunk = sizeof(T) == 4 ? 64 : 32;  // ring loads in flight per thread
    double pr[kFlushFreqs], pi[kFlushFreqs];
#pragma unroll
    for (int f = 0; f < kFlushFreqs; f++) { pr[f] = 0.0; pi[f] = 0.0; }
#pragma unroll
    for (int s0 = 0; s0 < kFlushRing; s0 += kFlushChunk) {
        if (s0 >= cnt) break;
        T xs[kFlushChunk];
#pragma unroll
        for (int s = 0; s < kFlushChunk; s++) xs[s] = s0 + s < cnt ? __ldcs(rp + (s0 + s) * kRingTile) : T(0);
#pragma unroll
        for (int s = 0; s < kFlushChunk; s++) {
            const double x = (double)xs[s];
#pragma unroll
            for (int f = 0; f < kFlushFreqs; f++) {
                pr[f] = fma(w.wr[s0 + s][f], x, pr[f]);
                pi[f] = fma(w.wi[s0 + s][f], x, pi[f]);
            }
        }
    }
    double2 *__restrict__ ap = acc + (((long long)shot * 3 + vc) * nf + f0) * fshot + cell;
#pragma unroll
    for (int f = 0; f < kFlushFreqs; f++)
        if (f0 + f < nf) {
            double2 v = ap[(long long)f * fshot];
            v.x += pr[f];
            v.y += pi[f];
            ap[(long long)f * fshot] = v;
        }
}

// Non-finite check of the receiver traces: sets *flag if any sample is NaN/Inf.
template <typename T>
__global__ void finite_check_kernel(const T *__restrict__ x, long long n, int *flag) {
    int bad = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        bad |= !isfinite((double)x[e]);
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

}  // namespace mittet
