"""Seeded synthetic workloads of the forward solve, gradient and serving path.

The reference runs on compile-time models (ncver0027/cpu_model.f90:5-146,
a seawater half-space over a steel plate) and text-file models (satan_i
conductivity.dat).  No public dataset exists for this path, so the workloads
below are seeded synthetic stand-ins with the sizes the benchmarks use:

  plain_cpu   64^3, dx 50 m, 10-cell CPML, two-layer 0.01 / 1.0 S/m, Ex dipole,
              Nt 3000, 32 receivers x 6 components, f_to_d at 0.25/0.5/1/2 Hz
  plain_gpu   256x256x192, dx 25 m, 16-cell CPML, log-normal 8^3 blocks
              (median 0.3 S/m, log10 sd 0.3, seed 2026) + 40x40x10 body of
              0.01 S/m at k 100..109, Nt 6000, one Ex dipole, 256 receivers,
              full-volume f_to_d of Ex Ey Ez at 4 frequencies
  batched     192x192x128, dx 25 m, 64 shots on an 8x8 grid (x/y dipoles
              alternating), Nt 5000, 128 receivers, 4 frequencies
  gradient    128x128x96, dx 50 m, 16 shots, true 0.3 S/m + 0.01 S/m body,
              start 0.3 S/m, Ex/Ey at 3 frequencies, Nt 4000
Time step: 0.95 of the (2,4) Taylor limit for the fastest fictitious velocity;
wavelet fmax = 0.9 c'_min/(Glim dx), Glim = 10.4 (cpu_set_condition.f90:354).
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace

import numpy as np

from .capi import FLAVOR_NCVER0027, FP32, SRC_ELECTRIC
from .solver import MU0_REF, PI_REF, ConstPara, Shot, cmax_of, dt_rule, firstderiv_gauss

GLIM = 10.4  # ncver0027/cpu_parameter_wafe.f90:39
OMEGA0 = 2.0 * PI_REF * 1.0


@dataclass
class Workload:
    name: str
    cp: ConstPara
    sigma: np.ndarray                 # [nz, ny, nx]
    shots: list                       # list[Shot]
    receivers: list                   # (ix, iy, iz, comp), 1-based
    nt: int
    wavelet: np.ndarray               # w[n] = s(n dt), n = 0..nt
    omega: np.ndarray                 # angular frequencies
    volume_dft: str = ""              # E components with full-volume f_to_d
    mu: np.ndarray | None = None
    fmax: float = 0.0

    @property
    def ncell(self) -> int:
        return self.cp.nx * self.cp.ny * self.cp.nz

    def cell_updates(self) -> int:
        return self.ncell * self.nt * len(self.shots)


def lognormal_blocks(nx, ny, nz, block=8, median=0.3, log10_sd=0.3, seed=2026) -> np.ndarray:
    """Log-normal conductivity constant over block^3 cells, x fastest."""
    rng = np.random.default_rng(seed)
    bx, by, bz = -(-nx // block), -(-ny // block), -(-nz // block)
    lg = rng.normal(np.log10(median), log10_sd, size=(bz, by, bx))
    s = 10.0 ** lg
    s = np.repeat(np.repeat(np.repeat(s, block, 0), block, 1), block, 2)
    return np.ascontiguousarray(s[:nz, :ny, :nx])


def add_body(sig, x0, x1, y0, y1, z0, z1, value) -> np.ndarray:
    s = sig.copy()
    s[z0:z1, y0:y1, x0:x1] = value
    return s


def _time_base(sig, d, flavor=FLAVOR_NCVER0027, precision=FP32, nx=None, ny=None, nz=None, ncpml=10):
    cmax = cmax_of(float(sig.min()), OMEGA0, MU0_REF)
    cmin = cmax_of(float(sig.max()), OMEGA0, MU0_REF)
    dt = dt_rule(d, cmax)
    fmax = 0.9 * cmin / (GLIM * d)
    cp = ConstPara(nx=nx, ny=ny, nz=nz, dx=d, dy=d, dz=d, ncpml=ncpml, dt=dt, cmax=cmax, omega0=OMEGA0,
                   flavor=flavor, precision=precision)
    return cp, fmax


FREQS4 = np.array([0.25, 0.5, 1.0, 2.0])


def plain_cpu(nt: int = 3000, n: int = 64, precision=FP32, flavor=FLAVOR_NCVER0027) -> Workload:
    d = 50.0
    sig = np.full((n, n, n), 1.0)
    sig[: n // 2] = 0.01  # sigma = 0.01 for k < 32 (0-based), 1.0 below
    cp, fmax = _time_base(sig, d, flavor=flavor, precision=precision, nx=n, ny=n, nz=n, ncpml=10)
    c = n // 2
    shots = [Shot(points=[(c, c, c - 2, "ex", SRC_ELECTRIC, 1.0)])]
    rec = [(x, c, c - 1, comp) for x in range(n // 4, n // 4 + 32) for comp in ("ex", "ey", "ez", "hx", "hy", "hz")]
    w = firstderiv_gauss(nt + 1, cp.dt, fmax)
    return Workload("plain_cpu_64", cp, sig, shots, rec, nt, w, 2 * np.pi * FREQS4, fmax=fmax)


def c2_model(nx=256, ny=256, nz=192, seed=2026) -> np.ndarray:
    sig = lognormal_blocks(nx, ny, nz, 8, 0.3, 0.3, seed)
    return add_body(sig, nx // 2 - 20, nx // 2 + 20, ny // 2 - 20, ny // 2 + 20, 100 * nz // 192,
                    100 * nz // 192 + 10, 0.01)


def surface_grid(nx, ny, ncpml, m):
    """m x m positions (1-based) spread over the interior in x and y."""
    xs = np.linspace(ncpml + 4, nx - ncpml - 3, m).round().astype(int)
    ys = np.linspace(ncpml + 4, ny - ncpml - 3, m).round().astype(int)
    return [(int(x), int(y)) for y in ys for x in xs]


def plain_gpu(nt: int = 6000, nx=256, ny=256, nz=192, precision=FP32, volume=True, seed=2026,
              flavor=FLAVOR_NCVER0027) -> Workload:
    d = 25.0 * 256 / nx if nx != 256 else 25.0
    sig = c2_model(nx, ny, nz, seed)
    cp, fmax = _time_base(sig, d, flavor=flavor, precision=precision, nx=nx, ny=ny, nz=nz, ncpml=16)
    kz = cp.ncpml + 3  # receivers at 0-based k = ncpml + 2
    shots = [Shot(points=[(nx // 2, ny // 2, kz, "ex", SRC_ELECTRIC, 1.0)])]
    rec = [(x, y, kz, "ex") for (x, y) in surface_grid(nx, ny, cp.ncpml, 16)]
    w = firstderiv_gauss(nt + 1, cp.dt, fmax)
    return Workload(f"plain_gpu_{nx}x{ny}x{nz}", cp, sig, shots, rec, nt, w, 2 * np.pi * FREQS4,
                    volume_dft="xyz" if volume else "", fmax=fmax)


def batched(nt: int = 5000, nx=192, ny=192, nz=128, nshot=64, precision=FP32, seed=2026) -> Workload:
    d = 25.0
    sig = c2_model(nx, ny, nz, seed)
    cp, fmax = _time_base(sig, d, precision=precision, nx=nx, ny=ny, nz=nz, ncpml=16)
    kz = cp.ncpml + 3
    m = int(round(np.sqrt(nshot)))
    pos = surface_grid(nx, ny, cp.ncpml, m)[:nshot]
    shots = [Shot(points=[(x, y, kz, "ex" if s % 2 == 0 else "ey", SRC_ELECTRIC, 1.0)]) for s, (x, y) in enumerate(pos)]
    rec = [(x, y, kz, comp) for (x, y) in surface_grid(nx, ny, cp.ncpml, 8) for comp in ("ex", "ey")]
    w = firstderiv_gauss(nt + 1, cp.dt, fmax)
    return Workload(f"batched_{nx}x{ny}x{nz}x{nshot}", cp, sig, shots, rec, nt, w, 2 * np.pi * FREQS4, fmax=fmax)


def gradient_case(nt: int = 4000, nx=128, ny=128, nz=96, nshot=16, precision=FP32, true_model=True) -> Workload:
    d = 50.0
    sig = np.full((nz, ny, nx), 0.3)
    if true_model:
        sig = add_body(sig, nx // 2 - 10, nx // 2 + 10, ny // 2 - 10, ny // 2 + 10, nz // 2, nz // 2 + 6, 0.01)
    # both models share the time base of the true model
    tb = add_body(np.full((nz, ny, nx), 0.3), 0, 1, 0, 1, 0, 1, 0.01)
    cp, fmax = _time_base(tb, d, precision=precision, nx=nx, ny=ny, nz=nz, ncpml=16)
    kz = cp.ncpml + 3
    m = int(round(np.sqrt(nshot)))
    pos = surface_grid(nx, ny, cp.ncpml, m)[:nshot]
    shots = [Shot(points=[(x, y, kz, "ex", SRC_ELECTRIC, 1.0)]) for (x, y) in pos]
    rec = [(x, y, kz, comp) for (x, y) in surface_grid(nx, ny, cp.ncpml, 6) for comp in ("ex", "ey")]
    w = firstderiv_gauss(nt + 1, cp.dt, fmax)
    return Workload(f"gradient_{nx}x{ny}x{nz}x{nshot}", cp, sig, shots, rec, nt, w,
                    2 * np.pi * np.array([0.25, 0.5, 1.0]), fmax=fmax)


def serving_case(nx, ny, nz, nshot, nt, seed=2026, precision=FP32) -> Workload:
    """One serving request: its own seeded log-normal model on a grid whose
    domain is 6.4 km wide (dx = 6400/nx), nshot surface dipoles, Nt steps."""
    d = 6400.0 / nx
    sig = c2_model(nx, ny, nz, seed)
    cp, fmax = _time_base(sig, d, precision=precision, nx=nx, ny=ny, nz=nz, ncpml=min(16, nx // 6))
    kz = cp.ncpml + 3
    m = max(1, int(np.ceil(np.sqrt(nshot))))
    pos = surface_grid(nx, ny, cp.ncpml, m)[:nshot]
    shots = [Shot(points=[(x, y, kz, "ex" if s % 2 == 0 else "ey", SRC_ELECTRIC, 1.0)]) for s, (x, y) in enumerate(pos)]
    rec = [(x, y, kz, comp) for (x, y) in surface_grid(nx, ny, cp.ncpml, 6) for comp in ("ex", "ey")]
    w = firstderiv_gauss(nt + 1, cp.dt, fmax)
    return Workload(f"serve_{nx}x{ny}x{nz}x{nshot}", cp, sig, shots, rec, nt, w, 2 * np.pi * FREQS4, fmax=fmax)


def small_case(n=(40, 36, 32), ncpml=8, nt=200, precision=FP32, flavor=FLAVOR_NCVER0027, seed=7,
               magnetic=False) -> Workload:
    """A random small case for parity tests (every slab and corner populated)."""
    nx, ny, nz = n
    d = 50.0
    rng = np.random.default_rng(seed)
    sig = 10.0 ** rng.normal(np.log10(0.3), 0.3, size=(nz, ny, nx))
    cp, fmax = _time_base(sig, d, flavor=flavor, precision=precision, nx=nx, ny=ny, nz=nz, ncpml=ncpml)
    from .capi import SRC_MAGNETIC
    if magnetic:
        pts = [(nx // 2, ny // 2, nz // 2, "hz", SRC_MAGNETIC, 1.0), (nx // 2 + 4, ny // 2, nz // 2, "hz", SRC_MAGNETIC, 1.0)]
    else:
        pts = [(nx // 2, ny // 2, nz // 2, "ex", SRC_ELECTRIC, 1.0)]
    rec = []
    for (x, y, z) in [(3, 3, 3), (nx // 2, ny // 2, nz // 2 + 3), (nx - 2, ny // 2, nz // 2), (nx // 3, ny - 3, 4),
                      (ncpml, ncpml + 1, nz - ncpml), (nx - 1, ny - 1, nz - 1), (1, 1, 1)]:
        for comp in ("ex", "ey", "ez", "hx", "hy", "hz"):
            rec.append((x, y, z, comp))
    w = firstderiv_gauss(nt + 1, cp.dt, fmax)
    return Workload(f"small_{nx}x{ny}x{nz}", cp, sig, [Shot(points=pts)], rec, nt, w, 2 * np.pi * FREQS4, fmax=fmax)


def make_solver(wl: Workload, precision=None):
    """Create a MittetSolver loaded with a workload."""
    from .solver import MittetSolver
    cp = wl.cp if precision is None else replace(wl.cp, precision=precision)
    s = MittetSolver(cp)
    s.set_model(wl.sigma, wl.mu)
    s.set_shots(wl.shots)
    s.set_wavelet(wl.wavelet)
    s.set_receivers(wl.receivers)
    s.set_freqs(wl.omega)
    if wl.volume_dft:
        s.set_volume_dft(wl.volume_dft)
    return s
