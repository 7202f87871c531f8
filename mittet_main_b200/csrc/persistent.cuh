// persistent.cuh -- one persistent launch for a block of G time steps of
// every shot.
//
// The stepped path launches, per step, the five part kernels of each phase
// plus the point kernels (inject, sample), about a dozen launches replayed
// from a CUDA graph.  On small grids each launch holds too little work to
// fill the GPU and the step is bound by launch gaps and tails.  This kernel
// instead keeps one cooperative grid resident (every CTA co-resident,
// persistent_grid() sizes it from the occupancy of this body) and walks all
// G steps itself:
//
//   [magnetic points]  barrier  E tiles of every part and shot  barrier
//   [electric points]  barrier  H tiles of every part and shot  barrier
//   receiver samples + next step's magnetic points (block 0)    barrier
//
// Tiles of all five parts (interior, x/y/z faces, edges) of all shots are
// spread over the CTAs round-robin; each tile runs the same e_cells/h_cells
// body as the part kernels (same fma forms: bit-identical results), with
// L2-coherent loads for every array the launch writes (fields, psi), since a
// tile's neighbours were written by other CTAs earlier in the same launch.
// The point work (sources, receivers) is a handful of cells done by block 0.
//
// The grid barrier is a counter and a generation word in global memory
// (arrive with an atomic, the last arrival releases the next generation).
// Every wait is bounded by %globaltimer: a wait that runs past wait_ns, or
// sees another CTA's failure, sets bit 2 of the error word and the CTA
// returns; the host reports MITTET_ERR_DEVICE_TIMEOUT.  The step counter is
// read from device memory at entry and advanced at exit, so the launch can
// sit in a CUDA graph replayed nt / G times.
#pragma once

namespace mittet {

struct GridBarrier {
    unsigned int count;
    unsigned int gen;
};

struct PersistCtl {
    GridBarrier *bar;
    int *err;                 // bit 2: a barrier wait gave up
    unsigned int expect;      // arrivals that complete a barrier (= gridDim.x)
    unsigned long long wait_ns;
};

template <typename T>
struct PersistArgs {
    PhaseArgs<T> e, h;
    const TileMap *tme, *tmh;  // tile maps (every part) of the E and H phases
    int ntile_e, ntile_h;      // tiles per shot
    int nshot;
    InjectArgs<T> im, ie;      // magnetic / electric points
    int has_mag, has_ele;
    SampleArgs<T> smp;
    int nsteps;
    PersistCtl ctl;
};

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid-wide barrier; false when this CTA must leave (a wait gave up here or
// in another CTA).  Writes before it are visible to loads after it in every
// CTA (fence, release on the generation word, acquire on the wait).
__device__ __forceinline__ bool grid_barrier(const PersistCtl &c) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
        int ok = 1;
        const unsigned g = ld_acquire_gpu(&c.bar->gen);
        __threadfence();
        const unsigned arrived = atomicAdd(&c.bar->count, 1u) + 1u;
        if (arrived == c.expect) {
            atomicExch(&c.bar->count, 0u);
            __threadfence();
            st_release_gpu(&c.bar->gen, g + 1u);
        } else {
            const unsigned long long t0 = global_ns();
            while (ld_acquire_gpu(&c.bar->gen) == g) {
                if (*(volatile int *)c.err & 4) {
                    ok = 0;
                    break;
                }
                if (global_ns() - t0 > c.wait_ns) {
                    atomicOr(c.err, 4);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Point sources of one kind at step n, by the threads of one CTA (the body
// of inject_kernel with the step given).
template <typename T>
__device__ __forceinline__ void persist_inject(const InjectArgs<T> &a, int n) {
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nth = blockDim.x * blockDim.y;
    for (int p = tid; p < a.npts; p += nth) {
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

// Receiver samples after step n (the body of sample_kernel with the step given).
template <typename T>
__device__ __forceinline__ void persist_sample(const SampleArgs<T> &a, int n) {
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nth = blockDim.x * blockDim.y;
    const int tot = a.nrec * a.nshot;
    for (int q = tid; q < tot; q += nth) {
        const int s = q / a.nrec, r = q % a.nrec;
        a.traces[(long long)q * a.nt + n] = __ldcg(a.f[a.rec_comp[r]] + (long long)s * a.fshot + a.rec_off[r]);
    }
}

// The tile b of a phase's map: box by kind, then the part body.
template <typename T, int VX, int BX, int BY, bool EPH>
__device__ __forceinline__ void persist_tile(const PhaseArgs<T> &a, const TileMap *__restrict__ tm, int b,
                                             int shot, int n) {
    const int nbox = __ldg(&tm->nbox);
    int q = 0;
    for (int t = 1; t < nbox; t++)
        if (b >= __ldg(&tm->start[t])) q = t;
    int i0, j, kb, ke;
    bool inside;
    locate<VX, BX, BY>(tm, q, q + 1, b, i0, j, kb, ke, inside);
    if (!inside) return;
    const int kind = __ldg(&tm->kind[q]);
    if constexpr (EPH) {
        switch (kind) {
            case 0: e_cells<T, VX, 0, false, true>(a, shot, i0, j, kb, ke, n); break;
            case 1: e_cells<T, VX, 1, false, true>(a, shot, i0, j, kb, ke, n); break;
            case 2: e_cells<T, VX, 2, false, true>(a, shot, i0, j, kb, ke, n); break;
            case 4: e_cells<T, VX, 4, false, true>(a, shot, i0, j, kb, ke, n); break;
            default: e_cells<T, VX, 7, false, true>(a, shot, i0, j, kb, ke, n); break;
        }
    } else {
        switch (kind) {
            case 0: h_cells<T, VX, 0, false, true>(a, shot, i0, j, kb, ke); break;
            case 1: h_cells<T, VX, 1, false, true>(a, shot, i0, j, kb, ke); break;
            case 2: h_cells<T, VX, 2, false, true>(a, shot, i0, j, kb, ke); break;
            case 4: h_cells<T, VX, 4, false, true>(a, shot, i0, j, kb, ke); break;
            default: h_cells<T, VX, 7, false, true>(a, shot, i0, j, kb, ke); break;
        }
    }
}

// Resident CTAs per SM asked of the kernel: it carries every part's body, so
// it needs the registers of the edge body; 3 x 128 threads fit FP32 two-cell
// threads without spilling, the wider ones get 2.
template <typename T, int VX>
constexpr int persist_min_blocks() {
    return (sizeof(T) == 4 && VX == 2) ? 3 : 2;
}

template <typename T, int VX, int BX, int BY>
__global__ void __launch_bounds__(BX *BY, (persist_min_blocks<T, VX>())) persistent_steps_kernel(
    const __grid_constant__ PersistArgs<T> p) {
    const int n0 = __ldcg(p.e.d_step);
    const long long te = (long long)p.ntile_e * p.nshot, th = (long long)p.ntile_h * p.nshot;
    if (p.has_mag) {
        if (blockIdx.x == 0) persist_inject<T>(p.im, n0);
        if (!grid_barrier(p.ctl)) return;
    }
    for (int s = 0; s < p.nsteps; s++) {
        const int n = n0 + s;
        for (long long t = blockIdx.x; t < te; t += gridDim.x)
            persist_tile<T, VX, BX, BY, true>(p.e, p.tme, (int)(t % p.ntile_e), (int)(t / p.ntile_e), n);
        if (!grid_barrier(p.ctl)) return;
        if (p.has_ele) {
            if (blockIdx.x == 0) persist_inject<T>(p.ie, n);
            if (!grid_barrier(p.ctl)) return;
        }
        for (long long t = blockIdx.x; t < th; t += gridDim.x)
            persist_tile<T, VX, BX, BY, false>(p.h, p.tmh, (int)(t % p.ntile_h), (int)(t / p.ntile_h), n);
        if (!grid_barrier(p.ctl)) return;
        if (blockIdx.x == 0) {
            persist_sample<T>(p.smp, n);
            // the next step's magnetic points go in after the samples of this one
            if (p.has_mag && s + 1 < p.nsteps) {
                __syncthreads();
                persist_inject<T>(p.im, n + 1);
            }
        }
        if (!grid_barrier(p.ctl)) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0) *p.smp.d_step = n0 + p.nsteps;
}

}  // namespace mittet
