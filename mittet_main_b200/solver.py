"""Host-side mirror of the reference's forward-solve surface.

The reference drives the path from Fortran module globals
(ncver0027/cpu_parameter_wafe.f90 ``module const_para``) and argument-light
subroutines called from ``program main`` (ncver0027/cpu_main.f90:35-187):

  source_posi / model / init_cpml / media_coeff      -> MittetSolver set-up
  do istep: read_source_3d, e_field_cpml4, CPML_E4,
            h_field_cpml4, CPML_H4, output_EH_J      -> MittetSolver.forward
  f_to_d_e / f_to_d_h                                -> f_to_d_e / f_to_d_h

Every numerical step runs in ``libmittet_b200.so`` through the C ABI; this
module only shapes arguments.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Iterable, Sequence

import numpy as np

from . import capi
from .capi import (COMP, FLAVOR_NCVER0027, FLAVOR_SATAN_I, FP32, FP64, SRC_ELECTRIC, SRC_MAGNETIC,
                   MittetError, check)

PI_REF = 3.14159265358979  # ncver0027/cpu_parameter_wafe.f90:30
MU0_REF = 1.2566370614e-6  # ncver0027/cpu_parameter_wafe.f90:84


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@dataclass
class ConstPara:
    """The solve's constants; the fields of ``module const_para`` that the hot
    path reads (ncver0027/cpu_parameter_wafe.f90:24-132), made run-time values."""
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    ncpml: int
    dt: float
    cmax: float
    omega0: float = 2.0 * PI_REF * 1.0
    mu0: float = MU0_REF
    flavor: int = FLAVOR_NCVER0027
    precision: int = FP32
    c1: float = 1.125
    c2: float | None = None
    psi_hyx_typo: int | None = None
    e_sign: int = 1
    h_sign: int = 1
    device: int = 0
    check_cfl: bool = True

    def grid(self) -> capi.Grid:
        return capi.Grid(self.nx, self.ny, self.nz, self.dx, self.dy, self.dz, self.ncpml)

    def phys(self) -> capi.Phys:
        lib = capi.load()
        p = capi.Phys()
        check(lib.mittet_phys_defaults(self.flavor, ctypes.byref(p)))
        p.dt = self.dt
        p.omega0 = self.omega0
        p.cmax = self.cmax
        p.mu0 = self.mu0
        p.c1 = self.c1
        if self.c2 is not None:
            p.c2 = self.c2
        if self.psi_hyx_typo is not None:
            p.psi_hyx_typo = self.psi_hyx_typo
        p.e_sign = self.e_sign
        p.h_sign = self.h_sign
        p.precision = self.precision
        p.device = self.device
        p.check_cfl = 1 if self.check_cfl else 0
        return p


def cmax_of(sigma_min: float, omega0: float = 2.0 * PI_REF, mu: float = MU0_REF) -> float:
    """Fastest fictitious velocity c' = sqrt(2 w0/(mu sigma)) (cpu_parameter_wafe.f90:106-110)."""
    return float(np.sqrt(2.0 * omega0 / mu / sigma_min))


def dt_rule(d: float, cmax: float, safety: float = 0.95) -> float:
    """safety x the (2,4) Taylor limit d/(c' sqrt(3) (|c1|+|c2|)), |c1|+|c2| = 1.16667."""
    return safety * d / (cmax * np.sqrt(3.0) * 1.16667)


def firstderiv_gauss(nt: int, dt: float, fmax: float) -> np.ndarray:
    """Wavelet samples w[n] = s(n dt), n = 0..nt, of the Gaussian derivative
    s(t) = -2 beta (t-t0) sqrt(beta/pi) exp(-beta (t-t0)^2), beta = pi fmax^2,
    t0 = pi/fmax (ncver0027/cpu_waveform.f90:20-26;
    satan_i/fwi3d_cpu_waveform_v1.4.c:132-142)."""
    pi = PI_REF
    t0 = pi / fmax
    beta = pi * fmax ** 2
    t = np.arange(nt + 1, dtype=np.float64) * dt
    return -(2.0 * beta * (t - t0) * np.sqrt(beta / pi)) * np.exp(-beta * (t - t0) ** 2.0)


def freq_grid_ref(nt: int, dt: float, nf: int | None = None) -> np.ndarray:
    """w_k = k 2 pi/(nt dt) (ncver0027/cpu_f_to_d_e.f90:134)."""
    nf = nt if nf is None else nf
    out = np.zeros(nf, dtype=np.float64)
    check(capi.load().mittet_freq_grid_ref(nt, dt, nf, _dptr(out)))
    return out


@dataclass
class Shot:
    """One source position: point sources sharing one wavelet."""
    points: list  # (ix, iy, iz, comp, kind, amp), 1-based positions


class MittetSolver:
    """Batched forward solver of one model; all shots run together."""

    def __init__(self, cp: ConstPara):
        self.cp = cp
        lib = capi.load()
        self._lib = lib
        self._h = ctypes.c_void_p()
        g = cp.grid()
        p = cp.phys()
        check(lib.mittet_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(self._h)))
        self.nshot = 0
        self.nrec = 0
        self.nf = 0
        self.nt_wave = 0

    # -------------------------------------------------------------- set-up
    def close(self):
        if self._h:
            self._lib.mittet_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_model(self, sigma: np.ndarray, mu: np.ndarray | None = None):
        """sigma, mu: [nz, ny, nx] (x fastest), Fortran sig/myu."""
        s = np.ascontiguousarray(sigma, dtype=np.float64)
        if s.size != self.cp.nx * self.cp.ny * self.cp.nz:
            raise ValueError("sigma has the wrong number of cells")
        m = None if mu is None else np.ascontiguousarray(mu, dtype=np.float64)
        if m is not None and m.size != s.size:
            raise ValueError("mu has the wrong number of cells")
        check(self._lib.mittet_set_model(self._h, _dptr(s), _dptr(m) if m is not None else None))

    def set_model_device(self, sigma, mu=None):
        """sigma/mu as contiguous [nz, ny, nx] CUDA torch tensors (float64 or
        float32, both the same) on the handle's device; the model stays on the
        device."""
        import torch

        if sigma.dtype not in (torch.float64, torch.float32) or not sigma.is_cuda or not sigma.is_contiguous():
            raise ValueError("sigma must be a contiguous float64 or float32 CUDA tensor")
        if sigma.numel() != self.cp.nx * self.cp.ny * self.cp.nz:
            raise ValueError("sigma has the wrong number of cells")
        if mu is not None and (mu.dtype != sigma.dtype or mu.shape != sigma.shape or not mu.is_cuda
                               or not mu.is_contiguous()):
            raise ValueError("mu must be a contiguous CUDA tensor of sigma's dtype and shape")
        check(self._lib.mittet_set_model_device(self._h, ctypes.c_void_p(sigma.data_ptr()),
                                                ctypes.c_void_p(mu.data_ptr()) if mu is not None else None,
                                                1 if sigma.dtype == torch.float64 else 0))

    def set_shots(self, shots: Sequence[Shot]):
        pts = []
        for s, shot in enumerate(shots):
            for (ix, iy, iz, comp, kind, amp) in shot.points:
                c = COMP[comp] if isinstance(comp, str) else int(comp)
                pts.append(capi.PointSource(s, ix, iy, iz, c, kind, amp))
        arr = (capi.PointSource * len(pts))(*pts)
        check(self._lib.mittet_set_sources(self._h, len(shots), len(pts), arr))
        self.nshot = len(shots)

    def set_wavelet(self, w: np.ndarray):
        w = np.ascontiguousarray(w, dtype=np.float64)
        check(self._lib.mittet_set_wavelet(self._h, w.size - 1, _dptr(w)))
        self.nt_wave = w.size - 1

    def set_receivers(self, receivers: Iterable):
        rs = [capi.Receiver(ix, iy, iz, COMP[c] if isinstance(c, str) else int(c)) for (ix, iy, iz, c) in receivers]
        arr = (capi.Receiver * max(len(rs), 1))(*rs)
        check(self._lib.mittet_set_receivers(self._h, len(rs), arr))
        self.nrec = len(rs)

    def set_freqs(self, omega: np.ndarray, h_factor: bool = True):
        om = np.ascontiguousarray(omega, dtype=np.float64)
        check(self._lib.mittet_set_freqs(self._h, om.size, _dptr(om), 1 if h_factor else 0))
        self.nf = om.size

    def set_volume_dft(self, comps: str = "xyz"):
        mask = sum(1 << "xyz".index(c) for c in comps)
        check(self._lib.mittet_set_volume_dft(self._h, mask))

    # -------------------------------------------------------------- solve
    def forward(self, nt: int, want_traces: bool = False):
        """Returns (spectra [nshot, nrec, nf] complex, traces [nshot, nrec, nt] or None)."""
        fd = np.zeros((self.nshot, self.nrec, max(self.nf, 1), 2), dtype=np.float64)
        td = np.zeros((self.nshot, self.nrec, nt), dtype=np.float64) if want_traces else None
        check(self._lib.mittet_forward(self._h, nt, _dptr(fd) if self.nf else None,
                                       _dptr(td) if td is not None else None))
        spec = (fd[..., 0] + 1j * fd[..., 1])[:, :, : self.nf]
        return spec, td

    def forward_device(self, nt: int, out=None, stream=None):
        """Keep everything on the device; out: CUDA tensor [nshot, nrec, nf, 2] float64."""
        ptr = ctypes.c_void_p(out.data_ptr()) if out is not None else None
        st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        check(self._lib.mittet_forward_device(self._h, nt, ptr, st))
        return out

    def volume_dft(self, shot: int, comp: str, out: np.ndarray | None = None) -> np.ndarray:
        """[nf, nz, ny, nx] complex spectra of one E component.  ``out``: an
        optional C-contiguous complex128 array of that shape (for example a
        view of pinned host memory), filled in place and returned."""
        shape = (self.nf, self.cp.nz, self.cp.ny, self.cp.nx)
        if out is None:
            out = np.empty(shape, dtype=np.complex128)
        elif out.shape != shape or out.dtype != np.complex128 or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous complex128 array of shape {shape}")
        check(self._lib.mittet_get_volume_dft(self._h, shot, "xyz".index(comp[-1]),
                                              out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def fields(self, shot: int = 0) -> np.ndarray:
        out = np.zeros((6, self.cp.nz, self.cp.ny, self.cp.nx), dtype=np.float64)
        check(self._lib.mittet_get_fields(self._h, shot, _dptr(out)))
        return out

    def gradient(self, nt: int, obs: np.ndarray, checkpoint_every: int = 200):
        o = np.zeros((self.nshot, self.nrec, self.nf, 2), dtype=np.float64)
        o[..., 0] = obs.real
        o[..., 1] = obs.imag
        misfit = np.zeros(1, dtype=np.float64)
        grad = np.zeros((self.cp.nz, self.cp.ny, self.cp.nx), dtype=np.float64)
        check(self._lib.mittet_gradient(self._h, nt, _dptr(o), checkpoint_every, _dptr(misfit), _dptr(grad)))
        return float(misfit[0]), grad

    def release_gradient_buffers(self):
        """Free the work buffers ``gradient`` keeps on the device for its next call."""
        check(self._lib.mittet_release_gradient_buffers(self._h))

    def fwi_update(self, nt: int, obs: np.ndarray, ecal: np.ndarray, grad: np.ndarray, sigma: np.ndarray,
                   iseabed: int, minval: float, maxval: float):
        """satan_i's model update (calc_phi, trial forward, calc_alpha,
        update_para2; fwi3d_cpu_inv_fwi_v1.4.c:85-107).  Returns
        (new sigma [nz, ny, nx], scaler, alpha); the solver's model becomes
        the new sigma."""
        def cplx(a):
            o = np.zeros(a.shape + (2,), dtype=np.float64)
            o[..., 0] = a.real
            o[..., 1] = a.imag
            return np.ascontiguousarray(o)
        o, e = cplx(np.asarray(obs)), cplx(np.asarray(ecal))
        g = np.ascontiguousarray(grad, dtype=np.float64)
        sig = np.array(sigma, dtype=np.float64, order="C", copy=True)
        step = np.zeros(2, dtype=np.float64)
        check(self._lib.mittet_fwi_update(self._h, nt, _dptr(o), _dptr(e), _dptr(g), int(iseabed), float(minval),
                                          float(maxval), _dptr(sig), _dptr(step)))
        return sig, float(step[0]), float(step[1])

    def time_kernels(self, nsteps: int) -> dict:
        """Mean device ms per launch of each kernel over nsteps separately launched steps."""
        ms = np.zeros(6, dtype=np.float64)
        check(self._lib.mittet_time_kernels(self._h, nsteps, _dptr(ms)))
        return dict(zip(["inject_magnetic", "e_phase", "inject_electric", "h_phase", "sample", "volume_dft"], ms.tolist()))

    def tuned_variant(self) -> dict:
        """[VX, BX, BY, ZC] the autotuner chose per phase and launch (VX = 0:
        the TMA-staged interior; ZC = 1000 + z: z marching planes with a
        prefetching interior, 2000 + z: with the interior held to 85
        registers; ZC < 0: a single-plane body with -ZC threads
        along z)."""
        parts = ("interior", "xfaces", "yfaces", "zfaces", "edges")
        c = (ctypes.c_int32 * (2 * len(parts) * 4))()
        check(self._lib.mittet_tuned_variants(self._h, c))
        v = list(c)
        return {f"{ph}_{part}": v[(i * len(parts) + p) * 4:(i * len(parts) + p + 1) * 4]
                for i, ph in enumerate(("e", "h")) for p, part in enumerate(parts)}

    def launch_count(self) -> int:
        return int(self._lib.mittet_last_launch_count(self._h))

    def launch_path(self) -> dict:
        """The time loop of the last forward: {"persistent": False, ...} for
        the stepped graph of part kernels (with, per phase, the stencil
        variant [VX, BX, BY, ZC] of its merged boundary launch, or None for
        four boundary launches, the z planes per band of its interior +
        x-face band launch, 0 for separate launches, and its layout: 0
        parts, 1 the grid as one general box, 2 parts with the slab rows
        whole), else the variant of the persistent multi-shot launch and its
        CTAs."""
        v, g = ctypes.c_int32(), ctypes.c_int32()
        check(self._lib.mittet_persistent_variant(self._h, ctypes.byref(v), ctypes.byref(g)))
        vs = stencil_variants(self.cp.precision == FP64)
        if v.value >= 0:
            return {"persistent": True, "variant": vs[v.value], "ctas": g.value}
        be, bh = ctypes.c_int32(), ctypes.c_int32()
        check(self._lib.mittet_boundary_variant(self._h, ctypes.byref(be), ctypes.byref(bh)))
        ze, zh = ctypes.c_int32(), ctypes.c_int32()
        check(self._lib.mittet_band_variant(self._h, ctypes.byref(ze), ctypes.byref(zh)))
        oe, oh = ctypes.c_int32(), ctypes.c_int32()
        check(self._lib.mittet_layout_variant(self._h, ctypes.byref(oe), ctypes.byref(oh)))
        return {"persistent": False, "e_boundary": vs[be.value] if be.value >= 0 else None,
                "h_boundary": vs[bh.value] if bh.value >= 0 else None, "e_band": ze.value, "h_band": zh.value,
                "e_layout": oe.value, "h_layout": oh.value}


def stencil_variants(fp64: bool = False) -> list:
    """The stencil variants the autotuner chooses from, as [VX, BX, BY, ZC]
    (ZC < 0: single-plane body; ZC >= 1000: marching variants of the
    interior, see tuned_variant); index v is what MITTET_VARIANT=v forces."""
    lib = capi.load()
    n = ctypes.c_int32()
    check(lib.mittet_stencil_variants(1 if fp64 else 0, ctypes.byref(n), None, 0))
    c = (ctypes.c_int32 * (4 * n.value))()
    check(lib.mittet_stencil_variants(1 if fp64 else 0, ctypes.byref(n), c, n.value))
    v = list(c)
    return [v[4 * i:4 * i + 4] for i in range(n.value)]


def f_to_d(traces: np.ndarray, dt: float, omega0: float, omega: np.ndarray, h_factor: bool = False,
           device: int = 0) -> np.ndarray:
    """GPU evaluation of the reference's damped DFT of time traces
    (cpu_f_to_d_e.f90:140-148; with h_factor, cpu_f_to_d_h.f90:146-148).
    traces [..., nt] -> spectra [..., nf]."""
    x = np.ascontiguousarray(traces, dtype=np.float64)
    lead = x.shape[:-1]
    nt = x.shape[-1]
    x2 = x.reshape(-1, nt)
    om = np.ascontiguousarray(omega, dtype=np.float64)
    out = np.zeros((x2.shape[0], om.size, 2), dtype=np.float64)
    check(capi.load().mittet_f_to_d(device, x2.shape[0], nt, dt, omega0, _dptr(x2), om.size, _dptr(om),
                                    1 if h_factor else 0, _dptr(out)))
    return (out[..., 0] + 1j * out[..., 1]).reshape(*lead, om.size)


def f_to_d_e(ex_trace: np.ndarray, signal: np.ndarray, dt: float, omega0: float, omega: np.ndarray, device: int = 0):
    """EX_w, JZ_w, GXe_w = EX_w/JZ_w of ncver0027/cpu_f_to_d_e.f90:134-160.
    signal: the unscaled wavelet trace s(istep dt), istep = 1..nt (signal.d)."""
    ex_w = f_to_d(ex_trace, dt, omega0, omega, False, device)
    jz_w = f_to_d(signal, dt, omega0, omega, False, device)
    return ex_w, jz_w, ex_w / jz_w


def f_to_d_h(hz_trace: np.ndarray, signal: np.ndarray, dt: float, omega0: float, omega: np.ndarray, device: int = 0):
    """HZ_w (with sqrt(-2 w0/(i w))), JZ_w, GXh_w of ncver0027/cpu_f_to_d_h.f90:141-167."""
    with np.errstate(divide="ignore", invalid="ignore"):
        hz_w = f_to_d(hz_trace, dt, omega0, omega, True, device)
        jz_w = f_to_d(signal, dt, omega0, omega, False, device)
        return hz_w, jz_w, hz_w / jz_w


def to_time_domain(spec_w: np.ndarray, dt: float) -> np.ndarray:
    """The time series f_to_d_e / f_to_d_h write after their spectra
    (ncver0027/cpu_f_to_d_e.f90:241-320): an unnormalised inverse DFT with
    FFTW's BACKWARD sign over the nd = len(spec_w) samples of the reference
    frequency grid w_k = 2 pi k / (nd dt) (mittet_freq_grid_ref), scaled by
    2 / (nd dt):  x[n] = 2 / (nd dt) sum_k X[k] exp(+2 pi i k n / nd).
    Post-processing of a few thousand samples per trace; not on the GPU."""
    x = np.asarray(spec_w, dtype=complex)
    nd = x.shape[-1]
    return np.fft.ifft(x, axis=-1) * nd * (2.0 / (nd * dt))
