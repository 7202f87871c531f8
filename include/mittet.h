/*
 * mittet.h -- C ABI of the B200 Mittet fictitious-wave FDTD solver.
 *
 * One call of mittet_forward() replaces the reference's whole per-shot time
 * loop and its f_to_d transform:
 *
 *   ncver0027/cpu_main.f90:99-143   do istep: read_source_3d, e_field_cpml4,
 *                                    CPML_E4, h_field_cpml4, CPML_H4, output_EH_J
 *   ncver0027/cpu_main.f90:182-185  f_to_d_e, f_to_d_h
 *   satan_i/fwi3d_cpu_rec2rec_v1.4.c:48-59 (fwdpropagation loop + laplaceToFreq)
 *
 * and mittet_gradient() replaces the FWI gradient of
 * satan_i/fwi3d_cpu_inv_fwi_v1.4.c:27-81 (residualE, sensitivity, conv_GdelE,
 * calc_gamma), returning the gradient in the satan_i layout
 * (double grad[nz][ny][nx], x fastest, zero in the CPML frame).
 *
 * Conventions
 *   - Arrays are x fastest: index c = (k*ny + j)*nx + i with 0-based i,j,k;
 *     this is Fortran sig(nx,ny,nz) column-major order and the satan_i
 *     ijk = k*ix*iy + j*ix + i order.
 *   - Source and receiver positions are 1-based (ix, iy, iz), exactly as the
 *     Fortran driver and satan_i's model_env.dat give them.
 *   - Complex outputs are interleaved (re, im) doubles (C99 double _Complex
 *     layout, Fortran complex(kind(0d0))).
 *   - Every call returns MITTET_OK (0) or a negative MITTET_ERR_* code;
 *     mittet_last_error() gives the message of the calling thread's last error.
 *   - The caller owns all host arrays; nothing is retained past a call.  A
 *     handle owns its device memory (model, fields, accumulators), so the
 *     model stays resident across calls.  A handle is not thread-safe; use one
 *     handle per host thread.
 */
#ifndef MITTET_H
#define MITTET_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define MITTET_OK 0
#define MITTET_ERR_INVALID_ARG (-1)
#define MITTET_ERR_CFL (-2)            /* dt above the (2,4) Taylor limit, cpu_set_condition.f90:279-286 */
#define MITTET_ERR_OOM (-3)
#define MITTET_ERR_DIVERGED (-4)       /* non-finite receiver samples */
#define MITTET_ERR_DEVICE_TIMEOUT (-5) /* a bounded device wait gave up */
#define MITTET_ERR_CUDA (-6)
#define MITTET_ERR_STATE (-7)          /* call made before its inputs were set */

/* ---- enums ---- */
#define MITTET_FLAVOR_NCVER0027 0 /* Fortran ncver0027 ranges, profiles, c2 = -0.04167d0 */
#define MITTET_FLAVOR_SATAN_I 1   /* C satan_i ranges, profiles (x * optToMax), c2 = -0.04167f */

#define MITTET_FP32 0 /* FP32 fields, FP64 DFT accumulators */
#define MITTET_FP64 1 /* FP64 everything */

#define MITTET_EX 0
#define MITTET_EY 1
#define MITTET_EZ 2
#define MITTET_HX 3
#define MITTET_HY 4
#define MITTET_HZ 5

/* Magnetic source: F -= amp * s((n+1) dt) * dt / mu / (dx dy dz), added
 * before the E half step (ncver0027/cpu_waveform.f90:46-50). */
#define MITTET_SRC_MAGNETIC 0
/* Electric source: F -= amp * (s(n dt) + s((n+1) dt))/2 * dt * 2 w0 / sigma / (dx dy dz),
 * added after the E half step (satan_i/fwi3d_cpu_function_v1.4.c:526-527). */
#define MITTET_SRC_ELECTRIC 1

/* ---- configuration ---- */

/* Grid: replaces the nx/ny/nz, dx/dy/dz and ncpml parameters of
 * ncver0027/cpu_parameter_wafe.f90:25-28 (satan_i: model_env.dat fields 1-6, 14). */
typedef struct {
    int32_t nx, ny, nz;
    double dx, dy, dz;
    int32_t ncpml;
} mittet_grid;

/* Physics and scheme constants: replaces cpu_parameter_wafe.f90:30-40,117,123-132. */
typedef struct {
    double dt;        /* fictitious time step [s] */
    double omega0;    /* 2 pi f0 [rad/s] */
    double cmax;      /* fastest fictitious velocity sqrt(2 w0/(mu sigma_min)); sets the CPML sig_max */
    double mu0;       /* permeability used where no mu volume is given */
    double c1, c2;    /* (2,4) stencil weights (reference: 1.125, -0.04167) */
    int32_t flavor;   /* MITTET_FLAVOR_* : index ranges and CPML profile formulae */
    int32_t psi_hyx_typo; /* 1: psi_Hyx uses c1*Ez(i+1)-c2*Ez(i) as in cpu_cpml4.f90:400,413 */
    int32_t e_sign, h_sign; /* +1; -1 gives the sign-flipped "bp" updates (cpu_eh_field_cpml42.f90:161-300) */
    double cpml_nn, cpml_order, cpml_kappa_max, cpml_a_max, cpml_ma, cpml_rcoef, cpml_opt_to_max_x;
    int32_t precision; /* MITTET_FP32 or MITTET_FP64 */
    int32_t device;    /* CUDA device ordinal */
    int32_t check_cfl; /* 1: reject dt above dx/cmax/sqrt(3)/1.16667 */
} mittet_phys;

/* One point source of one shot (a shot is one source position: the Fortran
 * driver puts two Hz points in each shot, cpu_waveform.f90:46-50). */
typedef struct {
    int32_t shot;        /* 0-based shot index */
    int32_t ix, iy, iz;  /* 1-based cell */
    int32_t comp;        /* MITTET_EX .. MITTET_HZ */
    int32_t kind;        /* MITTET_SRC_MAGNETIC or MITTET_SRC_ELECTRIC */
    double amp;          /* multiplies the wavelet (1.0 in the reference) */
} mittet_point_source;

/* One receiver: point sample of one component after every step
 * (ncver0027/cpu_output.f90:20-30; satan_i output() :772-777). */
typedef struct {
    int32_t ix, iy, iz; /* 1-based cell */
    int32_t comp;       /* MITTET_EX .. MITTET_HZ */
} mittet_receiver;

typedef struct mittet_handle_s mittet_handle;

/* Fill *phys with the reference constants of a flavour (dt, omega0 and cmax
 * must still be set by the caller; dt can come from mittet_reference_dt). */
int mittet_phys_defaults(int32_t flavor, mittet_phys *phys);

/* dt by the reference rule of a flavour:
 *   NCVER0027: 0.999 dx / cmax / sqrt(3) / 1.16667  (cpu_parameter_wafe.f90:117)
 *   SATAN_I  : 1/cmax/sqrt(1/dx^2+1/dy^2+1/dz^2) * 6/7 * 0.999f (fwi3d_cpu_lattice_v1.4.c:38-39) */
double mittet_reference_dt(int32_t flavor, const mittet_grid *grid, double cmax);

/* Reference f_to_d frequency grid w_k = k * 2 pi / (nt dt), k = 0..nf-1
 * (ncver0027/cpu_f_to_d_e.f90:134). */
int mittet_freq_grid_ref(int32_t nt, double dt, int32_t nf, double *omega);

/* Create a solver on phys->device.  Computes the CPML profiles
 * (init_cpml, cpu_cpml4.f90:8-248 / cpmlabc.c:7-175) on the host. */
int mittet_create(const mittet_grid *grid, const mittet_phys *phys, mittet_handle **out);
void mittet_destroy(mittet_handle *h);

/* Conductivity (and optionally permeability) volumes, nx*ny*nz doubles each,
 * x fastest (Fortran sig/myu, cpu_parameter_wafe.f90:100-101).  mu may be NULL
 * (phys->mu0 everywhere).  The model stays on the device until replaced. */
int mittet_set_model(mittet_handle *h, const double *sigma, const double *mu);

/* Shots and their point sources.  Shots share the model and receivers and
 * run together in one batched launch per half step. */
int mittet_set_sources(mittet_handle *h, int32_t nshot, int32_t npoint, const mittet_point_source *pts);

/* Wavelet samples w[n] = s(n dt), n = 0..nt (nt+1 values). */
int mittet_set_wavelet(mittet_handle *h, int32_t nt, const double *w);

/* Receivers, the same for every shot. */
int mittet_set_receivers(mittet_handle *h, int32_t nrec, const mittet_receiver *rec);

/* Angular frequencies of the f_to_d transform.  h_factor = 1 multiplies the
 * spectra of H receivers by sqrt(-2 w0/(i w)) (cpu_f_to_d_h.f90:146-148). */
int mittet_set_freqs(mittet_handle *h, int32_t nf, const double *omega, int32_t h_factor);

/* Full-volume f_to_d of the E components in comp_mask (bit c = MITTET_E*)
 * at the handle's frequencies, accumulated on the fly (0 disables). */
int mittet_set_volume_dft(mittet_handle *h, uint32_t comp_mask);

/* Run nt steps for every shot.
 *   rec_fd: [nshot][nrec][nf] complex (may be NULL)
 *   rec_td: [nshot][nrec][nt] receiver traces (may be NULL)
 * Trace sample n is taken after step n (t = (n+1) dt), as output_EH_J does. */
int mittet_forward(mittet_handle *h, int32_t nt, double *rec_fd, double *rec_td);

/* Full-volume spectra of the last forward: [nf][nz][ny][nx] complex. */
int mittet_get_volume_dft(mittet_handle *h, int32_t shot, int32_t comp, double *out);

/* Fields after the last forward: [6][nz][ny][nx] doubles (Ex Ey Ez Hx Hy Hz). */
int mittet_get_fields(mittet_handle *h, int32_t shot, double *out);

/* The reference's standalone f_to_d on host traces (cpu_f_to_d_e.f90:134-160,
 * cpu_f_to_d_h.f90:141-167) evaluated on the GPU: x [ntrace][nt] real
 * samples, out [ntrace][nf] complex.  h_factor as in mittet_set_freqs. */
int mittet_f_to_d(int32_t device, int32_t ntrace, int32_t nt, double dt, double omega0,
                  const double *x, int32_t nf, const double *omega, int32_t h_factor, double *out);

/* FWI gradient d(misfit)/d(sigma) for every shot of the handle.
 *   obs: [nshot][nrec][nf] complex observed spectra (receivers and freqs of the handle)
 *   misfit: 0.5 * sum |rec_fd - obs|^2 over shots, receivers, frequencies
 *   grad: [nz][ny][nx] doubles, summed over shots, zero outside
 *         [ncpml, n-ncpml) on every axis (satan_i calc_gamma,
 *         fwi3d_cpu_function_v1.4.c:2351-2384).
 * checkpoint_every: forward snapshots kept every that many steps (0 = 200). */
int mittet_gradient(mittet_handle *h, int32_t nt, const double *obs, int32_t checkpoint_every,
                    double *misfit, double *grad);

/* mittet_gradient keeps its work buffers (checkpoints, the segment history,
 * adjoint state: about (K + 1) * 6 + 25 field volumes per shot of a group)
 * in the handle for the next call, since an FWI loop calls it once per
 * iteration and allocating them anew costs up to a second.  This frees them,
 * e.g. before the handle serves other work.  No counterpart in the reference
 * (whose arrays are static). */
int mittet_release_gradient_buffers(mittet_handle *h);

/* One satan_i model update after a gradient (fwi3d_cpu_inv_fwi_v1.4.c:85-107):
 *   calc_phi (fwi3d_cpu_function_v1.4.c:2565-2603): scaler = 0.01f * max sigma /
 *     max grad over the cells with 0-based k <= iseabed (both maxima start at
 *     cell 0); trial model sigma2 = sigma - scaler * grad everywhere;
 *   one forward of every shot on sigma2 (receivers and frequencies of the
 *     handle, volume DFT off);
 *   calc_alpha (:2757-2785): k1 = sum dE (E2 - Ecal), k2 = sum (E2 - Ecal)^2
 *     (complex products, no conjugate) over shots, receivers and frequencies,
 *     dE = obs - Ecal;
 *   update_para2 (:2787-2832): alpha = 3 |k1| / |k2|; inside [ncpml, n-ncpml)
 *     sigma += alpha * scaler * grad where k <= iseabed, then every inside
 *     cell is clamped to [minval, maxval].
 * obs, ecal: [nshot][nrec][nf] complex (ecal = the current model's rec_fd);
 * grad: mittet_gradient's output; sigma: in/out [nz][ny][nx] (x fastest).
 * step[0] = scaler, step[1] = alpha.  The handle's model is left at the new
 * sigma.  A trial model with a non-positive conductivity, a zero largest
 * gradient or k2 = 0 is rejected with MITTET_ERR_INVALID_ARG. */
int mittet_fwi_update(mittet_handle *h, int32_t nt, const double *obs, const double *ecal, const double *grad,
                      int32_t iseabed, double minval, double maxval, double *sigma, double *step);

/* satan_i's frequency-domain gradient formula, evaluated on GPU `device`
 * in one pass over the cells (replaces residualE, sensitivity, conv_GdelE
 * and calc_gamma, satan_i/fwi3d_cpu_function_v1.4.c:2202-2384).  All
 * complex arrays are interleaved (re, im) doubles, cells x fastest
 * (n = nx*ny*nz), frequency index w = 0 .. nf-1 (satan_i's upperF = nf):
 *   rec_pos: [nrec][3] 1-based receiver cells (model_env.dat positions)
 *   obs:     [3 comp][nrec][nf]        Exobs, Eyobs, Ezobs
 *   e_ff:    [3 comp][nf][n]           EcalX_ff, EcalY_ff, EcalZ_ff
 *   e_bb:    [3 comp][nrec][3 dir][nf][n]  EcalX_bb, EcalY_bb, EcalZ_bb
 * Outputs (each may be NULL except grad):
 *   err_sum: sum |dE| over receivers, frequencies and x, y, z (residualE)
 *   de:      [3 dir][nrec][nf]  delEx_f, delEy_f, delEz_f = obs - e_ff at the
 *            receiver; with obs = NULL it is an input instead: the residual
 *            itself (residualE skipped)
 *   sense:   [n]  sum over rec, dir, w, comp of |e_ff e_bb|
 *   e_back:  [3 comp][nf][n]  sum over rec, dir of e_bb conj(de)
 *   grad:    [n]  in/out: += Re sum_w sum_c e_ff e_back (divided by sense
 *            when normalize = 1, as calc_gamma does) on [ncpml, n - ncpml)
 *            per axis; untouched elsewhere. */
int mittet_satan_gamma(int32_t device, const mittet_grid *grid, int32_t nrec, const int32_t *rec_pos, int32_t nf,
                       const double *obs, const double *e_ff, const double *e_bb, int32_t normalize,
                       double *err_sum, double *de, double *sense, double *e_back, double *grad);

/* Device-resident variants for callers that keep data on the GPU (the
 * PyTorch front end).  Pointers are device pointers of the handle's device;
 * stream is the caller's cudaStream_t (NULL = the legacy default stream): the
 * solve starts after the work already queued there and the stream waits for
 * the solve, so events recorded on it bracket the whole solve.
 * mittet_set_model_device: sigma (and mu, or NULL) are [nz][ny][nx] arrays of
 * double (is_fp64 = 1) or float (0), whatever the handle's precision; the
 * model stays on the device (checked there: MITTET_ERR_INVALID_ARG for a
 * value that is not positive and finite), and m = 2 w0 dt / sigma is formed
 * in FP64 from the given values as mittet_set_model does. */
int mittet_set_model_device(mittet_handle *h, const void *sigma, const void *mu, int32_t is_fp64);
int mittet_forward_device(mittet_handle *h, int32_t nt, void *rec_fd_dev, void *stream);

/* Per-kernel timing (CUDA events on the handle's stream): restarts the last
 * forward's shots from zero fields and runs nsteps steps (nsteps <= the last
 * forward's nt) launching each kernel separately.  ms[0..5] receive the mean
 * device time per launch of: magnetic inject, E phase, electric inject,
 * H phase, sampling, volume-DFT flush (0 where a kernel did not run). */
int mittet_time_kernels(mittet_handle *h, int32_t nsteps, double *ms);

/* Stencil variant the autotuner chose for the interior launch of the E and
 * H phases at the last forward: {VX, BX, BY, ZC} = x cells per thread,
 * thread block in x and y, z planes each thread marches through (ZC < 0:
 * single-plane body, see mittet_tuned_variants). */
int mittet_tuned_variant(mittet_handle *h, int32_t *e_cfg, int32_t *h_cfg);

/* All chosen variants: cfg[40] = [phase E, H][launch interior, x faces,
 * y faces, z faces, edges][VX, BX, BY, ZC].  VX = 0 marks the TMA-staged
 * interior kernel, whose BX x BY is then its tile in cells.  ZC < 0 marks a
 * single-plane body: a BX x BY x (-ZC) thread block, one z plane per thread.
 * ZC = 1000 + z marks a marching body of z planes whose interior part
 * prefetches the next plane, ZC = 2000 + z one whose interior body is held
 * to 85 registers (more resident warps). */
int mittet_tuned_variants(mittet_handle *h, int32_t *cfg);

/* The stencil variants the autotuner chooses from for FP32 (fp64 = 0) or
 * FP64 fields: *count receives their number, cfg[4 v .. 4 v + 3] the first
 * min(count, max) as {VX, BX, BY, ZC} (ZC < 0: single-plane body, as above).
 * Variant v is the one the environment variable MITTET_VARIANT=v forces on
 * every launch.  No counterpart in the reference (a tuning introspection). */
int mittet_stencil_variants(int32_t fp64, int32_t *count, int32_t *cfg, int32_t max);

/* Which launch the last forward's time loop used: *variant = -1 for the
 * stepped graph of part kernels, else the stencil variant (index as in
 * mittet_stencil_variants) whose tiles and thread shape the persistent
 * multi-shot launch ran, with *grid its CTAs.  The autotuner picks it by
 * timing a block of steps of each (MITTET_PERSIST=0/1 forces one).  No
 * counterpart in the reference (a tuning introspection). */
int mittet_persistent_variant(mittet_handle *h, int32_t *variant, int32_t *grid);

/* Whether each phase launches its four boundary parts (x, y, z faces and
 * the edges) as one merged launch: the stencil variant it uses (index as in
 * mittet_stencil_variants) for the E and H phase, -1 for four launches.
 * Chosen by the autotuner on the whole phase.  No counterpart in the
 * reference (a tuning introspection). */
int mittet_boundary_variant(mittet_handle *h, int32_t *e_variant, int32_t *h_variant);

/* Whether each phase launches its interior and its two x faces as one band
 * launch (tiles ordered by rows, so the CTAs in flight read whole rows): the
 * z planes per band for the E and H phase, 0 for separate launches.  Chosen
 * by the autotuner on the whole phase.  No counterpart in the reference (a
 * tuning introspection). */
int mittet_band_variant(mittet_handle *h, int32_t *e_zc, int32_t *h_zc);

/* How the forward tiles of the E / H phase cover the grid: 0 split into
 * interior, faces and edges; 1 the whole grid as one box with the general
 * (CPML on every axis) body; 2 the interior and x faces as in 0 and the y-
 * and z-slab rows whole, in general boxes.  Chosen by the autotuner per grid
 * and batch (1 wins on grids that are mostly CPML slab).  No counterpart in
 * the reference (a tuning introspection). */
int mittet_layout_variant(mittet_handle *h, int32_t *e_layout, int32_t *h_layout);

/* Number of kernels the last forward launched (for launch accounting). */
int64_t mittet_last_launch_count(mittet_handle *h);

/* Forward solve that allocates no device memory.  No counterpart in the
 * reference (whose Fortran/C drivers own static arrays); it exists for hosts
 * that cannot call cudaMalloc/cudaFree: cudaFree synchronises the whole
 * device and stalls the other streams of a serving process, and some hosts'
 * device memory belongs to another allocator.  Every intermediate buffer
 * lives in one file-scope __device__ array of 32 MiB that each GPU loading
 * the library keeps until exit; a solve whose padded layout does not fit
 * (about 96^3 cells with a few hundred receivers for a few thousand steps),
 * or with more than 256 cells on an axis, 64 points, 2048 receivers or 256
 * frequencies, is rejected with MITTET_ERR_INVALID_ARG.  FP32 fields with an
 * FP64 f_to_d, one shot (every point has shot 0), uniform permeability
 * phys->mu0.
 *   sigma_dev:   device, nx*ny*nz doubles, x fastest; every value must be
 *                positive and finite: unlike mittet_set_model this call does
 *                not read the model back to check it, and it runs no
 *                finite check on the result (a bad model or an unstable dt
 *                gives Inf/NaN spectra, not MITTET_ERR_DIVERGED)
 *   wavelet_dev: device, nt+1 doubles, w[n] = s(n dt)
 *   pts, rec, omega: host arrays (copied into the device array)
 *   rec_fd_dev:  device output, [nrec][nf] complex (interleaved doubles)
 *   stream:      cudaStream_t (NULL = legacy default stream); the call only
 *                enqueues work, results are ready when the stream reaches it.
 * The first call on a device looks up the array's address with that device
 * current; make it before any stream capture.  Calls share the array and it
 * keeps the last call's contents (what must start at zero is cleared by each
 * call); calls that overlap on the GPU race on it. */
int mittet_forward_noalloc(const mittet_grid *grid, const mittet_phys *phys, const double *sigma_dev,
                           int32_t npoint, const mittet_point_source *pts, int32_t nt, const double *wavelet_dev,
                           int32_t nrec, const mittet_receiver *rec, int32_t nf, const double *omega,
                           int32_t h_factor, double *rec_fd_dev, void *stream);

/* Message of the calling thread's last error; returns its length. */
int mittet_last_error(char *buf, size_t len);

#ifdef __cplusplus
}
#endif
#endif /* MITTET_H */
