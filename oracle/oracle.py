"""TEST INFRASTRUCTURE ONLY -- ctypes front end of the FP64 CPU oracle.

The oracle (``oracle/mittet_oracle.c``) restates the reference's forward path
and f_to_d transform on the CPU; ``oracle/_ref/satan_ref`` is the reference's
own satan_i C kernels compiled from their sources.  Only the tests, the smoke
check and bench.py's CPU-baseline leg import this module; the product never
does.

Flavour constants follow:
  * ncver0027/cpu_parameter_wafe.f90:30-40,84,117,123-132 (Fortran)
  * satan_i/fwi3d_cpu_cpmlabc_v1.4.c:10-23, fwi3d_cpu_function_v1.4.c:1187,
    fwi3d_cpu_alloli1_v1.4.h:3, fwi3d_cpu_lattice_v1.4.c:35-39 (C)
"""
from __future__ import annotations

import ctypes
import os
import struct
import subprocess
import tempfile
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "satan_ref")
# the same sources built with the reference's own flags (gcc -fopenmp -O3):
# the timed CPU reference arm; REF_PATH is the bit-parity build
REF_O3_PATH = os.path.join(HERE, "_ref", "satan_ref_o3")

FLAVOR_NCVER0027 = 0
FLAVOR_SATAN_I = 1
SRC_MAGNETIC = 0
SRC_ELECTRIC = 1
COMPS = {"ex": 0, "ey": 1, "ez": 2, "hx": 3, "hy": 4, "hz": 5}

# ncver0027/cpu_parameter_wafe.f90:30,84
PI_F = 3.14159265358979
MU0_F = 1.2566370614e-6
# satan_i/fwi3d_cpu_alloli1_v1.4.h:3 and the float literal of c2 (function.c:1187)
MU0_C = 12.5663706e-7
C2_C = float(np.float32(-0.04167))


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("ncpml", ctypes.c_int32),
        ("flavor", ctypes.c_int32), ("psi_hyx_typo", ctypes.c_int32),
        ("e_sign", ctypes.c_int32), ("h_sign", ctypes.c_int32),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
        ("dt", ctypes.c_double), ("omega0", ctypes.c_double), ("c1", ctypes.c_double), ("c2", ctypes.c_double),
        ("cmax", ctypes.c_double),
        ("nn", ctypes.c_double), ("order", ctypes.c_double), ("kappa_max", ctypes.c_double),
        ("a_max", ctypes.c_double), ("ma", ctypes.c_double), ("rcoef", ctypes.c_double),
        ("opt_to_max_x", ctypes.c_double),
    ]


@dataclass
class Params:
    """Grid + physics + CPML constants of one solve (both flavours)."""
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    dt: float
    ncpml: int
    cmax: float
    omega0: float = 2.0 * PI_F * 1.0
    flavor: int = FLAVOR_NCVER0027
    psi_hyx_typo: int = 1
    e_sign: int = 1
    h_sign: int = 1
    c1: float = 1.125
    c2: float = -0.04167
    nn: float = 3.0
    order: float = 0.0
    kappa_max: float = 1.0
    a_max: float = 0.2
    ma: float = 1.0
    rcoef: float = 0.01

    def to_c(self) -> OrcParams:
        p = OrcParams()
        for name, _ in OrcParams._fields_:
            if name == "opt_to_max_x":
                p.opt_to_max_x = 10.0 if self.flavor == FLAVOR_SATAN_I else 1.0
            else:
                setattr(p, name, getattr(self, name))
        return p


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.check_call(["make", "-s", "-C", HERE, os.path.join(HERE, "liboracle.so")])
        _lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        _lib.orc_forward.argtypes = [
            P(OrcParams), P(ctypes.c_double), P(ctypes.c_double),
            ctypes.c_int, P(ctypes.c_int64), P(ctypes.c_int32), P(ctypes.c_int32), P(ctypes.c_double),
            ctypes.c_int, P(ctypes.c_double),
            ctypes.c_int, P(ctypes.c_int64), P(ctypes.c_int32),
            P(ctypes.c_double), P(ctypes.c_double)]
        _lib.orc_forward.restype = ctypes.c_int
        _lib.orc_dft.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, P(ctypes.c_double),
                                 ctypes.c_int, P(ctypes.c_double), ctypes.c_int, P(ctypes.c_double)]
        _lib.orc_dft.restype = None
        _lib.orc_profiles.argtypes = [P(OrcParams), P(ctypes.c_double), ctypes.c_int]
        _lib.orc_ranges.argtypes = [P(OrcParams), P(ctypes.c_int32)]
    return _lib


def _ptr(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


def cell_index(p: Params, ix1: int, iy1: int, iz1: int) -> int:
    """0-based linear index of a 1-based (ix, iy, iz) position, x fastest."""
    return ((iz1 - 1) * p.ny + (iy1 - 1)) * p.nx + (ix1 - 1)


def forward(p: Params, sigma: np.ndarray, mu: np.ndarray, sources, wavelet: np.ndarray,
            receivers, nt: int, want_fields: bool = False):
    """Run one shot.

    sources:   list of (ix, iy, iz, comp_name, kind, amp) with 1-based positions
    receivers: list of (ix, iy, iz, comp_name)
    Returns traces [nrec, nt] (and the final 6 fields [6, nz, ny, nx]).
    """
    L = lib()
    sigma = np.ascontiguousarray(sigma, dtype=np.float64).reshape(-1)
    mu = np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    wavelet = np.ascontiguousarray(wavelet, dtype=np.float64)
    assert wavelet.size >= nt + 1
    sc = np.array([cell_index(p, *s[:3]) for s in sources], dtype=np.int64)
    sk = np.array([COMPS[s[3]] for s in sources], dtype=np.int32)
    sd = np.array([s[4] for s in sources], dtype=np.int32)
    sa = np.array([s[5] for s in sources], dtype=np.float64)
    rc = np.array([cell_index(p, *r[:3]) for r in receivers], dtype=np.int64)
    rk = np.array([COMPS[r[3]] for r in receivers], dtype=np.int32)
    traces = np.zeros((max(len(receivers), 1), nt), dtype=np.float64)
    fields = np.zeros((6, p.nz, p.ny, p.nx), dtype=np.float64) if want_fields else None
    cp = p.to_c()
    rc_ = L.orc_forward(ctypes.byref(cp), _ptr(sigma, ctypes.c_double), _ptr(mu, ctypes.c_double),
                        len(sources), _ptr(sc, ctypes.c_int64), _ptr(sk, ctypes.c_int32),
                        _ptr(sd, ctypes.c_int32), _ptr(sa, ctypes.c_double),
                        nt, _ptr(wavelet, ctypes.c_double),
                        len(receivers), _ptr(rc, ctypes.c_int64), _ptr(rk, ctypes.c_int32),
                        _ptr(traces, ctypes.c_double),
                        _ptr(fields, ctypes.c_double) if want_fields else None)
    if rc_ != 0:
        raise MemoryError("oracle allocation failed")
    traces = traces[: len(receivers)]
    return (traces, fields) if want_fields else traces


def dft(trace: np.ndarray, dt: float, omega0: float, omegas, h_factor: bool = False) -> np.ndarray:
    """f_to_d damped DFT of one trace at angular frequencies ``omegas``."""
    L = lib()
    x = np.ascontiguousarray(trace, dtype=np.float64)
    om = np.ascontiguousarray(omegas, dtype=np.float64)
    out = np.zeros(2 * om.size, dtype=np.float64)
    L.orc_dft(x.size, dt, omega0, _ptr(x, ctypes.c_double), om.size, _ptr(om, ctypes.c_double),
              1 if h_factor else 0, _ptr(out, ctypes.c_double))
    return out[0::2] + 1j * out[1::2]


def profiles(p: Params) -> np.ndarray:
    """[3 axes, 8 (esig msig be ce bh ch ked khd), nmax] restated CPML profiles."""
    nmax = max(p.nx, p.ny, p.nz)
    out = np.zeros((3, 8, nmax), dtype=np.float64)
    cp = p.to_c()
    lib().orc_profiles(ctypes.byref(cp), _ptr(out, ctypes.c_double), nmax)
    return out


def ranges(p: Params) -> np.ndarray:
    out = np.zeros(36 + 60, dtype=np.int32)
    cp = p.to_c()
    lib().orc_ranges(ctypes.byref(cp), _ptr(out, ctypes.c_int32))
    return out


# ----------------------------------------------------------- satan_i reference

def satan_params(ix, iy, iz, dx, dy, dz, ncpml, omega0, minval):
    """dt and cmax exactly as satan_i/fwi3d_cpu_lattice_v1.4.c:35-39 computes them."""
    f32 = lambda v: float(np.float32(v))
    cmax = np.sqrt(2.0 * omega0 / MU0_C / minval)
    courant = 1.0 / cmax / np.sqrt(1.0 / dx ** 2 + 1.0 / dy ** 2 + 1.0 / dz ** 2)
    dt = courant * 6.0 / 7.0 * f32(0.999)
    return Params(nx=ix, ny=iy, nz=iz, dx=dx, dy=dy, dz=dz, dt=dt, ncpml=ncpml, cmax=cmax,
                  omega0=omega0, flavor=FLAVOR_SATAN_I, psi_hyx_typo=0, c2=C2_C)


def run_satan_reference(ix, iy, iz, dx, dy, dz, ncpml, omega0, sigma, wavelet, nt, src, src_comp, receivers,
                        nvol=0):
    """Run the reference's own satan_i kernels (oracle/_ref/satan_ref).

    src: 1-based (px, py, pz); src_comp in 0..2; receivers: list of (px, py, pz, comp 0..5).
    Returns (dt, cmax, traces[nrec, nt], fields[6, iz, iy, ix]).  With nvol > 0
    a fifth item: the reference's full-volume transform laplaceToFreq_2 of the
    E history, [3, nvol - 1, iz, iy, ix] complex at w = 1 .. nvol-1 of the grid
    w 2 pi / ((nt + 1) dt), divided by sqrt(-2 w0 / (i w)) (its G = E / J with
    a unit current impulse and out_True = 1).
    """
    if not os.path.exists(REF_PATH):
        raise FileNotFoundError(REF_PATH)
    sigma = np.ascontiguousarray(sigma, dtype=np.float64).reshape(-1)
    n = ix * iy * iz
    with tempfile.TemporaryDirectory() as d:
        os.mkdir(os.path.join(d, "data"))
        hdr = [ix, iy, iz, ncpml, nt, src_comp, src[0], src[1], src[2], len(receivers)]
        buf = struct.pack("<10i", *hdr)
        for r in receivers:
            buf += struct.pack("<4i", *r)
        if nvol:
            buf += struct.pack("<i", nvol)
        buf += struct.pack("<6d", dx, dy, dz, omega0, float(sigma.min()), float(sigma.max()))
        buf += sigma.tobytes() + np.ascontiguousarray(wavelet[: nt + 1], dtype=np.float64).tobytes()
        with open(os.path.join(d, "in.bin"), "wb") as f:
            f.write(buf)
        env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "4"))
        args = [REF_PATH, "fwd", "in.bin", "out.bin"] if nvol else [REF_PATH, "in.bin", "out.bin"]
        subprocess.check_call(args, cwd=d, env=env, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        raw = np.fromfile(os.path.join(d, "out.bin"), dtype=np.float64)
    dt, cmax = raw[0], raw[1]
    nrec = len(receivers)
    traces = raw[2: 2 + nrec * nt].reshape(nrec, nt)
    o = 2 + nrec * nt
    fields = raw[o:o + 6 * n].reshape(6, iz, iy, ix)
    if not nvol:
        assert raw.size == o + 6 * n
        return float(dt), float(cmax), traces, fields
    v = raw[o + 6 * n:]
    vol = (v[0::2] + 1j * v[1::2]).reshape(3, nvol - 1, iz, iy, ix)
    return float(dt), float(cmax), traces, fields, vol


def time_satan_reference(ix, iy, iz, dx, dy, dz, ncpml, omega0, sigma, steps_per_seg, nseg, src, src_comp=0,
                         threads=None, binary=None):
    """Wall time of nseg segments of steps_per_seg steps of the reference's own
    satan_i kernels (timing mode of oracle/_ref/satan_ref_o3, the build with
    the reference's own -O3 flags, unless ``binary`` names another).  The
    reference's coefficient dumps (./data/coef*.dat, ./data/pml_conductivity_*)
    go to /dev/null so set-up does not write gigabytes of text."""
    exe = binary or REF_O3_PATH
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    sigma = np.ascontiguousarray(sigma, dtype=np.float64).reshape(-1)
    nt_total = steps_per_seg * nseg
    with tempfile.TemporaryDirectory() as d:
        os.mkdir(os.path.join(d, "data"))
        for f in ("coef1.dat", "coef2.dat", "coef3.dat", "pml_conductivity_x", "pml_conductivity_y",
                  "pml_conductivity_z"):
            os.symlink("/dev/null", os.path.join(d, "data", f))
        hdr = [ix, iy, iz, ncpml, steps_per_seg, src_comp, src[0], src[1], src[2], 0]
        buf = struct.pack("<10i", *hdr)
        buf += struct.pack("<6d", dx, dy, dz, omega0, float(sigma.min()), float(sigma.max()))
        buf += sigma.tobytes() + np.zeros(nt_total + 1, dtype=np.float64).tobytes()
        with open(os.path.join(d, "in.bin"), "wb") as f:
            f.write(buf)
        env = dict(os.environ)
        if threads:
            env["OMP_NUM_THREADS"] = str(threads)
        subprocess.check_call([exe, "in.bin", "out.bin", str(nseg)], cwd=d, env=env,
                              stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        return np.fromfile(os.path.join(d, "out.bin"), dtype=np.float64)


def time_oracle_steps(p: Params, sigma, mu, sources, wavelet, n_short=2, n_long=8):
    """Seconds per time step of the oracle: difference of two runs so set-up cancels."""
    import time as _time
    t = []
    for n in (n_short, n_long):
        t0 = _time.perf_counter()
        forward(p, sigma, mu, sources, wavelet, [], n)
        t.append(_time.perf_counter() - t0)
    return max(t[1] - t[0], 1e-9) / (n_long - n_short)


def gradient(p: Params, sigma, mu, sources, wavelet, receivers, nt, omega, obs, h_factor=True):
    """Discrete-adjoint gradient of one shot (oracle/mittet_oracle.c orc_gradient).
    obs: [nrec, nf] complex.  Returns (misfit, grad [nz, ny, nx], spectra [nrec, nf])."""
    L = lib()
    if not hasattr(L, "_grad_sig"):
        P = ctypes.POINTER
        L.orc_gradient.argtypes = [
            P(OrcParams), P(ctypes.c_double), P(ctypes.c_double),
            ctypes.c_int, P(ctypes.c_int64), P(ctypes.c_int32), P(ctypes.c_int32), P(ctypes.c_double),
            ctypes.c_int, P(ctypes.c_double),
            ctypes.c_int, P(ctypes.c_int64), P(ctypes.c_int32),
            ctypes.c_int, P(ctypes.c_double), ctypes.c_int, P(ctypes.c_double),
            P(ctypes.c_double), P(ctypes.c_double), P(ctypes.c_double)]
        L.orc_gradient.restype = ctypes.c_int
        L._grad_sig = True
    sigma = np.ascontiguousarray(sigma, dtype=np.float64).reshape(-1)
    mu = np.ascontiguousarray(mu, dtype=np.float64).reshape(-1)
    wavelet = np.ascontiguousarray(wavelet, dtype=np.float64)
    sc = np.array([cell_index(p, *s[:3]) for s in sources], dtype=np.int64)
    sk = np.array([COMPS[s[3]] for s in sources], dtype=np.int32)
    sd = np.array([s[4] for s in sources], dtype=np.int32)
    sa = np.array([s[5] for s in sources], dtype=np.float64)
    rc = np.array([cell_index(p, *r[:3]) for r in receivers], dtype=np.int64)
    rk = np.array([COMPS[r[3]] for r in receivers], dtype=np.int32)
    om = np.ascontiguousarray(omega, dtype=np.float64)
    ob = np.zeros((len(receivers), om.size, 2))
    ob[..., 0] = np.real(obs)
    ob[..., 1] = np.imag(obs)
    mis = np.zeros(1)
    g = np.zeros(sigma.size)
    spec = np.zeros((len(receivers), om.size, 2))
    cp = p.to_c()
    r = L.orc_gradient(ctypes.byref(cp), _ptr(sigma, ctypes.c_double), _ptr(mu, ctypes.c_double),
                       len(sources), _ptr(sc, ctypes.c_int64), _ptr(sk, ctypes.c_int32), _ptr(sd, ctypes.c_int32),
                       _ptr(sa, ctypes.c_double), nt, _ptr(wavelet, ctypes.c_double),
                       len(receivers), _ptr(rc, ctypes.c_int64), _ptr(rk, ctypes.c_int32),
                       om.size, _ptr(om, ctypes.c_double), 1 if h_factor else 0, _ptr(ob, ctypes.c_double),
                       _ptr(mis, ctypes.c_double), _ptr(g, ctypes.c_double), _ptr(spec, ctypes.c_double))
    if r != 0:
        raise MemoryError("oracle allocation failed")
    return float(mis[0]), g.reshape(p.nz, p.ny, p.nx), spec[..., 0] + 1j * spec[..., 1]


def misfit(p: Params, sigma, mu, sources, wavelet, receivers, nt, omega, obs, h_factor=True):
    """0.5 sum |S - obs|^2 from a plain forward (for finite differences)."""
    tr = forward(p, sigma, mu, sources, wavelet, receivers, nt)
    J = 0.0
    for r, rec in enumerate(receivers):
        S = dft(tr[r], p.dt, p.omega0, omega, h_factor=h_factor and rec[3].startswith("h"))
        J += 0.5 * float(np.sum(np.abs(S - obs[r]) ** 2))
    return J


def calc_phi(sigma, grad, iseabed):
    """satan_i calc_phi (fwi3d_cpu_function_v1.4.c:2565-2603): maxima of sigma
    and grad over 0-based k <= iseabed, both starting from cell 0;
    scaler = 0.01f * sigmax / gradmax; trial sigma2 = sigma - scaler * grad.
    Arrays are [nz, ny, nx].  Returns (scaler, sigma2)."""
    sigma = np.asarray(sigma, dtype=np.float64)
    grad = np.asarray(grad, dtype=np.float64)
    sigmax, gradmax = float(sigma.flat[0]), float(grad.flat[0])
    top = slice(0, iseabed + 1)
    if sigma[top].size:
        sigmax = max(sigmax, float(sigma[top].max()))
        gradmax = max(gradmax, float(grad[top].max()))
    scaler = float(np.float32(0.01)) * sigmax / gradmax
    return scaler, sigma - scaler * grad


def update_para2(sigma, grad, obs, ecal, e2, scaler, iseabed, minval, maxval, ncpml):
    """satan_i calc_alpha + update_para2 (fwi3d_cpu_function_v1.4.c:2757-2832):
    k1 = sum dE (E2 - Ecal), k2 = sum (E2 - Ecal)^2 with dE = obs - Ecal, in
    the order shot, receiver, frequency; alpha = 3 |k1| / |k2|; inside
    [ncpml, n - ncpml) sigma += alpha * scaler * grad where k <= iseabed, then
    clamp to [minval, maxval].  Returns (new sigma, alpha)."""
    d = (np.asarray(obs) - np.asarray(ecal)).ravel()
    c = (np.asarray(e2) - np.asarray(ecal)).ravel()
    k1 = 0j
    k2 = 0j
    for q in range(d.size):
        k1 += d[q] * c[q]
        k2 += c[q] * c[q]
    alpha = 3.0 * abs(k1) / abs(k2)
    out = np.array(sigma, dtype=np.float64, copy=True)
    nz, ny, nx = out.shape
    inner = out[ncpml:nz - ncpml, ncpml:ny - ncpml, ncpml:nx - ncpml]
    g = np.asarray(grad, dtype=np.float64)[ncpml:nz - ncpml, ncpml:ny - ncpml, ncpml:nx - ncpml]
    ks = np.arange(ncpml, nz - ncpml)[:, None, None]
    inner += np.where(ks <= iseabed, (alpha * scaler) * g, 0.0)
    np.clip(inner, minval, maxval, out=inner)
    return out, alpha


# ------------------------------------ satan_i post-processing, reference runs

def _run_ref_mode(mode: str, payload: bytes, files=()):
    """Run oracle/_ref/satan_ref in one of its array modes; returns (raw output
    bytes, {name: text of each requested ./data file the reference wrote})."""
    if not os.path.exists(REF_PATH):
        raise FileNotFoundError(REF_PATH)
    with tempfile.TemporaryDirectory() as d:
        os.mkdir(os.path.join(d, "data"))
        with open(os.path.join(d, "in.bin"), "wb") as f:
            f.write(payload)
        env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "4"))
        subprocess.check_call([REF_PATH, mode, "in.bin", "out.bin"], cwd=d, env=env,
                              stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        with open(os.path.join(d, "out.bin"), "rb") as f:
            raw = f.read()
        texts = {}
        for name in files:
            with open(os.path.join(d, "data", name)) as f:
                texts[name] = f.read()
    return raw, texts


def _c(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.complex128)).tobytes()


def run_satan_ftod(traces, jx, dt, omega0, upper_f, files=()):
    """satan_i laplaceToFreq (fwi3d_cpu_function_v1.4.c:1976-2089) on given
    traces [nrec, 3, it] (Ex, Ey, Ez) and source trace jx [it].  Returns
    ([nrec, 4, it] complex: EX_w, EY_w, EZ_w, JX_w on w_n = n 2 pi/(it dt),
    texts of the requested spectrum files)."""
    tr = np.ascontiguousarray(traces, dtype=np.float64)
    nrec, _, it = tr.shape
    buf = struct.pack("<3i", it, nrec, upper_f) + struct.pack("<2d", dt, omega0)
    buf += tr.tobytes() + np.ascontiguousarray(jx, dtype=np.float64).tobytes()
    raw, texts = _run_ref_mode("ftod", buf, files)
    out = np.frombuffer(raw, dtype=np.complex128).reshape(nrec, 4, it)
    return out, texts


def run_satan_gamma(shape, ncpml, rec_pos, d, obs, e_ff, e_bb, files=()):
    """satan_i residualE, sensitivity, conv_GdelE and calc_gamma
    (fwi3d_cpu_function_v1.4.c:2202-2384).  shape (ix, iy, iz); rec_pos
    [nrec, 3] 1-based; obs [3, nrec, nf]; e_ff [3, nf, n]; e_bb
    [3, nrec, 3, nf, n].  Returns dict(err_sum, de [3, nrec, nf], sense [n],
    e_back [3, nf, n], grad [n]) and the requested file texts."""
    ix, iy, iz = shape
    n = ix * iy * iz
    nrec, nf = len(rec_pos), np.asarray(e_ff).shape[1]
    buf = struct.pack("<6i", ix, iy, iz, ncpml, nrec, nf)
    buf += np.ascontiguousarray(rec_pos, dtype=np.int32).tobytes() + struct.pack("<3d", *d)
    buf += b"".join(_c(np.asarray(a)[c]) for a in (obs, e_ff, e_bb) for c in range(3))
    raw, texts = _run_ref_mode("gamma", buf, files)
    v = np.frombuffer(raw, dtype=np.float64)
    o = 1
    err = float(v[0])
    cv = lambda a: a[0::2] + 1j * a[1::2]  # noqa: E731
    de = cv(v[o:o + 2 * 3 * nrec * nf]).reshape(3, nrec, nf)
    o += 2 * 3 * nrec * nf
    sense = v[o:o + n].copy()
    o += n
    back = cv(v[o:o + 2 * 3 * nf * n]).reshape(3, nf, n)
    o += 2 * 3 * nf * n
    grad = v[o:o + n].copy()
    return {"err_sum": err, "de": de, "sense": sense, "e_back": back, "grad": grad}, texts


def run_satan_update(shape, ncpml, iseabed, rec_pos, d, minval, maxval, sig, grad, de, e_ffl, e_ff2, files=()):
    """satan_i calc_phi, calc_alpha(0), update_para2(0)
    (fwi3d_cpu_function_v1.4.c:2565-2603, 2757-2832).  de [3, nrec, nf];
    e_ffl, e_ff2 [3, nf, n].  Returns dict(scaler, k1, k2, alpha, sig2 [n],
    sig [n]) and the requested file texts (sig_tmp.dat, gradient_000.dat,
    sig_000.dat)."""
    ix, iy, iz = shape
    n = ix * iy * iz
    nrec, nf = len(rec_pos), np.asarray(e_ffl).shape[1]
    buf = struct.pack("<7i", ix, iy, iz, ncpml, iseabed, nrec, nf)
    buf += np.ascontiguousarray(rec_pos, dtype=np.int32).tobytes() + struct.pack("<5d", *d, minval, maxval)
    buf += np.ascontiguousarray(sig, dtype=np.float64).tobytes() + np.ascontiguousarray(grad, dtype=np.float64).tobytes()
    buf += b"".join(_c(np.asarray(a)[c]) for a in (de, e_ffl, e_ff2) for c in range(3))
    raw, texts = _run_ref_mode("update", buf, files)
    v = np.frombuffer(raw, dtype=np.float64)
    return {"scaler": float(v[0]), "k1": complex(v[1], v[2]), "k2": complex(v[3], v[4]), "alpha": float(v[5]),
            "sig2": v[6:6 + n].copy(), "sig": v[6 + n:6 + 2 * n].copy()}, texts


def satan_gamma(shape, ncpml, rec_pos, obs, e_ff, e_bb):
    """numpy restatement of satan_i residualE, sensitivity, conv_GdelE and
    calc_gamma (fwi3d_cpu_function_v1.4.c:2202-2384), same layouts as
    run_satan_gamma (one shot, grad starting at zero)."""
    ix, iy, iz = shape
    obs, e_ff, e_bb = (np.asarray(a, dtype=np.complex128) for a in (obs, e_ff, e_bb))
    cells = np.array([((z - 1) * iy + (y - 1)) * ix + (x - 1) for (x, y, z) in rec_pos], dtype=np.int64)
    de = obs - e_ff[:, :, cells].transpose(0, 2, 1)                         # residualE :2222-2228
    err = float(np.sum(np.abs(de).transpose(1, 2, 0)))                       # :2236-2238
    sense = np.abs(e_ff[:, None, None] * e_bb).sum(axis=(0, 1, 2, 3))        # sensitivity :2276-2278
    back = np.einsum("crdwn,drw->cwn", e_bb, np.conj(de))                    # conv_GdelE :2329-2342
    g = np.real((e_ff * back).sum(axis=0)).sum(axis=0) / sense               # calc_gamma :2372-2374
    m = np.zeros((iz, iy, ix), dtype=bool)
    m[ncpml:iz - ncpml, ncpml:iy - ncpml, ncpml:ix - ncpml] = True
    return {"err_sum": err, "de": de, "sense": sense, "e_back": back, "grad": np.where(m.ravel(), g, 0.0)}
