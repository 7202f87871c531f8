"""The reference's text files for the forward / gradient path, read and written
so that its drivers, scripts and plots consume this library's results
unchanged.

satan_i (fwi3d_cpu_function_v1.4.c), all under its ./data directory:
  model_env.dat       read_shotrec (:14-78): ix iy iz dx dy dz dt_ratio it mstep
                      trstep omega_0 fmax_w Glim ncpml, five unused numbers,
                      startF upperF shot_num, shot_num (px py pz) triples,
                      rec_num, rec_num (px py pz) triples (whitespace-separated,
                      1-based positions)
  minmax.dat          minval maxval;  iseabed.dat: iseabed
  conductivity.dat    true_model (:268-292): one "x y z sigma" line per cell,
                      k outermost, i innermost
  waveform[XYZ].dat   read_trawave (:80-101): "t value" per time sample
  spectrum_e[xyz]_SSS_RRR.dat
                      read_Eobs (:904-932) / writer (:2011-2077): upperF lines
                      "f re im abs arg" per shot SSS and receiver RRR
  gradient_III.dat, sig_III.dat
                      update_para2 (:2819-2828): "%10.2lf %10.2lf %10.2lf %e"
                      per cell (x y z value), k outermost
ncver0027 (cpu_f_to_d_e.f90:168-216, cpu_f_to_d_h.f90):
  EX_w<name>.d, JZ_w<name>.d, GXe_w<name>.d: "f re im" per frequency;
  absEX_w<name>.d ...: "f abs".

Arrays are [nz, ny, nx] numpy volumes (x fastest), positions 1-based.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np


def _c_double(v: float) -> str:
    """C printf("%lf") / ("%f"): six decimals."""
    return "%f" % v


def _c_exp(v: float) -> str:
    """C printf("%e")."""
    return "%e" % v


@dataclass
class ModelEnv:
    """satan_i model_env.dat (read_shotrec, fwi3d_cpu_function_v1.4.c:14-78)."""
    ix: int
    iy: int
    iz: int
    dx: float
    dy: float
    dz: float
    dt_ratio: float
    it: int
    mstep: int
    trstep: int
    omega_0: float
    fmax_w: float
    glim: float
    ncpml: int
    unused: list = field(default_factory=lambda: [0.0] * 5)
    start_f: int = 0
    upper_f: int = 0
    shots: list = field(default_factory=list)      # [(px, py, pz)], 1-based
    receivers: list = field(default_factory=list)  # [(px, py, pz)], 1-based


def read_model_env(path: str) -> ModelEnv:
    tok = open(path).read().split()
    pos = [0]

    def nxt(conv):
        v = conv(tok[pos[0]])
        pos[0] += 1
        return v

    ix, iy, iz = nxt(int), nxt(int), nxt(int)
    dx, dy, dz, dt_ratio = nxt(float), nxt(float), nxt(float), nxt(float)
    it, mstep, trstep = nxt(int), nxt(int), nxt(int)
    omega_0, fmax_w, glim = nxt(float), nxt(float), nxt(float)
    ncpml = nxt(int)
    unused = [nxt(float) for _ in range(5)]
    start_f, upper_f, nshot = nxt(int), nxt(int), nxt(int)
    shots = [(nxt(int), nxt(int), nxt(int)) for _ in range(nshot)]
    nrec = nxt(int)
    recs = [(nxt(int), nxt(int), nxt(int)) for _ in range(nrec)]
    return ModelEnv(ix, iy, iz, dx, dy, dz, dt_ratio, it, mstep, trstep, omega_0, fmax_w, glim, ncpml, unused,
                    start_f, upper_f, shots, recs)


def write_model_env(path: str, e: ModelEnv) -> None:
    lines = [f"{e.ix}", f"{e.iy}", f"{e.iz}", repr(e.dx), repr(e.dy), repr(e.dz), repr(e.dt_ratio), f"{e.it}",
             f"{e.mstep}", f"{e.trstep}", repr(e.omega_0), repr(e.fmax_w), repr(e.glim), f"{e.ncpml}"]
    lines += [repr(float(v)) for v in e.unused]
    lines += [f"{e.start_f}", f"{e.upper_f}", f"{len(e.shots)}"]
    lines += [f"{p[0]}  {p[1]}  {p[2]}" for p in e.shots]
    lines += [f"{len(e.receivers)}"]
    lines += [f"{p[0]}  {p[1]}  {p[2]}" for p in e.receivers]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def read_minmax(path: str) -> tuple[float, float]:
    a, b = open(path).read().split()[:2]
    return float(a), float(b)


def read_iseabed(path: str) -> int:
    return int(open(path).read().split()[0])


def read_conductivity(path: str, ix: int, iy: int, iz: int) -> np.ndarray:
    """conductivity.dat -> sigma [iz, iy, ix] (true_model, :268-292)."""
    a = np.loadtxt(path, dtype=np.float64, ndmin=2)
    if a.shape[0] < ix * iy * iz:
        raise ValueError(f"{path}: {a.shape[0]} cells, expected {ix * iy * iz}")
    return np.ascontiguousarray(a[:ix * iy * iz, 3].reshape(iz, iy, ix))


def write_conductivity(path: str, sigma: np.ndarray, dx: float, dy: float, dz: float) -> None:
    """"x y z sigma" per cell, k outermost (the layout true_model reads)."""
    iz, iy, ix = sigma.shape
    with open(path, "w") as f:
        for k in range(iz):
            for j in range(iy):
                for i in range(ix):
                    f.write(f"{_c_double(i * dx)}   {_c_double(j * dy)}   {_c_double(k * dz)}   "
                            f"{_c_double(sigma[k, j, i])}\n")


def read_waveform(path: str, it: int) -> np.ndarray:
    """waveform[XYZ].dat -> samples s[0..it-1] (read_trawave, :80-101)."""
    a = np.loadtxt(path, dtype=np.float64, ndmin=2)
    return np.ascontiguousarray(a[:it, 1])


def write_waveform(path: str, dt: float, s: np.ndarray) -> None:
    with open(path, "w") as f:
        for n, v in enumerate(np.asarray(s, dtype=np.float64)):
            f.write(f"{_c_exp(n * dt)} {_c_exp(v)}\n")


def read_signal(path: str) -> tuple[np.ndarray, np.ndarray]:
    """A "t value" trace file (Fortran list-directed or numpy savetxt), e.g.
    residual_wave_abso_rev.d read by corona/ver0030r_a/cpu_main.f90:41-46."""
    a = np.loadtxt(path, dtype=np.float64, ndmin=2)
    return a[:, 0], np.ascontiguousarray(a[:, 1])


def spectrum_name(comp: str, shot: int, rec: int) -> str:
    """spectrum_e[xyz]_SSS_RRR.dat (read_Eobs, :913-915)."""
    return f"spectrum_{comp}_{shot:03d}_{rec:03d}.dat"


def write_spectrum(path: str, freqs_hz: np.ndarray, spec: np.ndarray) -> None:
    """One "f re im abs arg" line per frequency (the writer at :2060-2077)."""
    with open(path, "w") as f:
        for fr, z in zip(np.asarray(freqs_hz), np.asarray(spec)):
            f.write(f"{fr:10e} {z.real:10e}  {z.imag:10e}  {abs(z):10e}   {np.angle(z):10e}\n")


def read_spectrum(path: str, upper_f: int) -> np.ndarray:
    """First upper_f lines of a spectrum file -> complex [upper_f] (read_Eobs)."""
    a = np.loadtxt(path, dtype=np.float64, ndmin=2)[:upper_f]
    return a[:, 1] + 1j * a[:, 2]


def write_observed(dirname: str, spectra: np.ndarray, receivers, freqs_hz) -> None:
    """spectra [nshot, nrec, nf] for receivers (ix, iy, iz, comp): one
    spectrum_e?_SSS_RRR.dat per shot, receiver position and E component, with
    receiver positions numbered in order of first appearance."""
    positions = []
    for r in receivers:
        if tuple(r[:3]) not in positions:
            positions.append(tuple(r[:3]))
    for s in range(spectra.shape[0]):
        for q, r in enumerate(receivers):
            if r[3] not in ("ex", "ey", "ez"):
                continue
            write_spectrum(os.path.join(dirname, spectrum_name(r[3], s, positions.index(tuple(r[:3])))),
                           freqs_hz, spectra[s, q])


def read_observed(dirname: str, nshot: int, positions, upper_f: int, comps=("ex", "ey", "ez")) -> np.ndarray:
    """Inverse of write_observed: [nshot, len(positions) * len(comps), upper_f],
    receivers ordered position-major (ex, ey, ez of position 0, then 1, ...)."""
    out = np.zeros((nshot, len(positions) * len(comps), upper_f), dtype=complex)
    for s in range(nshot):
        for p in range(len(positions)):
            for c, comp in enumerate(comps):
                out[s, p * len(comps) + c] = read_spectrum(os.path.join(dirname, spectrum_name(comp, s, p)), upper_f)
    return out


def write_volume(path: str, vol: np.ndarray, dx: float, dy: float, dz: float) -> None:
    """gradient_III.dat / sig_III.dat: "%10.2lf %10.2lf %10.2lf %e" per cell,
    k outermost (update_para2, :2819-2828)."""
    iz, iy, ix = vol.shape
    with open(path, "w") as f:
        for k in range(iz):
            for j in range(iy):
                for i in range(ix):
                    f.write("%10.2f    %10.2f    %10.2f    %e\n" % (i * dx, j * dy, k * dz, vol[k, j, i]))


def read_volume(path: str, ix: int, iy: int, iz: int) -> np.ndarray:
    a = np.loadtxt(path, dtype=np.float64, ndmin=2)
    return np.ascontiguousarray(a[:ix * iy * iz, 3].reshape(iz, iy, ix))


def write_f_to_d(dirname: str, name: str, freqs_hz: np.ndarray, ex_w: np.ndarray, jz_w: np.ndarray) -> None:
    """ncver0027 f_to_d_e outputs for one trace (cpu_f_to_d_e.f90:168-216):
    EX_w<name>.d, JZ_w<name>.d, GXe_w<name>.d ("f re im") and the abs* files
    ("f abs"), GXe_w = EX_w / JZ_w."""
    gx = np.asarray(ex_w) / np.asarray(jz_w)
    for stem, z in (("EX_w", ex_w), ("JZ_w", jz_w), ("GXe_w", gx)):
        with open(os.path.join(dirname, f"{stem}{name}.d"), "w") as f:
            for fr, v in zip(freqs_hz, z):
                f.write(f"  {float(fr):.17g}  {float(v.real):.17g}  {float(v.imag):.17g}\n")
        with open(os.path.join(dirname, f"abs{stem}{name}.d"), "w") as f:
            for fr, v in zip(freqs_hz, z):
                f.write(f"  {float(fr):.17g}  {float(abs(v)):.17g}\n")


def write_f_to_d_time(dirname: str, name: str, dt: float, ex_t: np.ndarray, jz_t: np.ndarray,
                      gx_t: np.ndarray) -> None:
    """EX_t<name>.d, JZ_t<name>.d, GXe_t<name>.d ("t re im") and the absEX_t
    ... files ("t abs") of cpu_f_to_d_e.f90:303-320, t = n dt."""
    for stem, z in (("EX_t", ex_t), ("JZ_t", jz_t), ("GXe_t", gx_t)):
        with open(os.path.join(dirname, f"{stem}{name}.d"), "w") as f:
            for n, v in enumerate(z):
                f.write(f"  {n * dt:.17g}  {float(v.real):.17g}  {float(v.imag):.17g}\n")
        with open(os.path.join(dirname, f"abs{stem}{name}.d"), "w") as f:
            for n, v in enumerate(z):
                f.write(f"  {n * dt:.17g}  {float(abs(v)):.17g}\n")


def read_f_to_d(path: str) -> tuple[np.ndarray, np.ndarray]:
    """A "f re im" file -> (freqs, complex values)."""
    a = np.loadtxt(path, dtype=np.float64, ndmin=2)
    return a[:, 0], a[:, 1] + 1j * a[:, 2]


def workload_from_satan(dirname: str, precision=None, nt: int | None = None):
    """Builds a forward workload from a satan_i ./data directory: grid,
    conductivity, x-directed electric sources at the transmitter positions,
    Ex/Ey/Ez receivers, the waveformX.dat wavelet and the frequencies
    startF..upperF-1 of its grid om = 2 pi / (it dt) (read_shotrec,
    true_model, read_trawave, laplaceToFreq)."""
    import ctypes

    from . import capi
    from .capi import FLAVOR_SATAN_I, FP64, SRC_ELECTRIC
    from .solver import ConstPara, Shot
    from .workloads import Workload

    e = read_model_env(os.path.join(dirname, "model_env.dat"))
    sig = read_conductivity(os.path.join(dirname, "conductivity.dat"), e.ix, e.iy, e.iz)
    minval, _ = read_minmax(os.path.join(dirname, "minmax.dat"))
    mu0 = 12.5663706e-7  # satan_i/fwi3d_cpu_alloli1_v1.4.h:3
    # lattice (fwi3d_cpu_lattice_v1.4.c:35-39): cmax from minval, dt by the C rule
    cmax = float(np.sqrt(2.0 * e.omega_0 / mu0 / minval))
    grid = capi.Grid(e.ix, e.iy, e.iz, e.dx, e.dy, e.dz, e.ncpml)
    dt = float(capi.load().mittet_reference_dt(FLAVOR_SATAN_I, ctypes.byref(grid), cmax))
    cp = ConstPara(nx=e.ix, ny=e.iy, nz=e.iz, dx=e.dx, dy=e.dy, dz=e.dz, ncpml=e.ncpml, dt=dt, cmax=cmax,
                   omega0=e.omega_0, flavor=FLAVOR_SATAN_I, precision=precision if precision is not None else FP64,
                   mu0=mu0)
    steps = (e.it - 1) if nt is None else nt
    w = read_waveform(os.path.join(dirname, "waveformX.dat"), e.it)
    if w.size < steps + 1:
        w = np.concatenate([w, np.zeros(steps + 1 - w.size)])
    shots = [Shot(points=[(p[0], p[1], p[2], "ex", SRC_ELECTRIC, 1.0)]) for p in e.shots]
    recs = [(p[0], p[1], p[2], c) for p in e.receivers for c in ("ex", "ey", "ez")]
    om = 2 * np.pi / (e.it * dt)
    omega = om * np.arange(max(e.start_f, 1), e.upper_f)
    return Workload("satan_data", cp, sig, shots, recs, steps, w[:steps + 1], omega, fmax=e.fmax_w)
