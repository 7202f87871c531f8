"""satan_i's frequency-domain FWI gradient, evaluated with the GPU forward.

satan_i does not differentiate its time stepping.  It forms a Born
cross-correlation of frequency-domain fields (fwi3d_cpu_function_v1.4.c):

  residualE   (:2202-2244)  dE[rec, w] = Eobs - Ecal_ff at the receiver
  laplaceToFreq_back        G_bb[rec][dir] = field of a unit electric
                            dipole at receiver rec along dir (reciprocity)
  conv_GdelE  (:2292-2349)  E_back_c = sum_rec sum_dir G_bb,c[rec][dir] conj(dE_dir[rec])
  sensitivity (:2246-2290)  sense = sum_rec,dir,w,c |E_ff,c G_bb,c[rec][dir]|
  calc_gamma  (:2351-2384)  grad += Re sum_w sum_c E_ff,c E_back,c / sense,
                            inside [ncpml, n - ncpml) on every axis.

Here every field is a full-volume f_to_d spectrum of the GPU solver, the
receiver dipoles are solved as one batch of shots, and the source spectrum
normalisation of satan_i (E / J times the FFT of its "true" wavelet) is
replaced by the plain Green's-function form that makes the formula the
first-order derivative of this library's misfit 0.5 sum |Ecal - Eobs|^2:

  gamma_w(x) = Re [ (1/J_w) sum_c E_ff,c(x) E_back,c(x) ] * dx dy dz,

which, like satan_i's gamma, is the descent direction -dJ/dsigma: the
scattering current of a conductivity perturbation, (dsigma / 2 w0) dE'/dt' in
the fictitious domain, enters Ampere's law as the source current does, and
its transform is -i w' (dsigma / 2 w0) E = E dsigma / sqrt(-2 w0 / (i w)),

J_w = the diffusive-domain spectrum of the injected source current: the
f_to_d transform of the wavelet times sqrt(-2 w0 / (i w)), as satan_i's
ctmp_j (fwi3d_cpu_function_v1.4.c laplaceToFreq_2).  With ``normalize=True`` the sum is divided by satan_i's
``sense`` as well.  The formula is a continuous-limit Born gradient: it
matches the discrete adjoint of ``mittet_gradient`` only up to
discretisation and transform-truncation errors, and is used to cross-check
it (cosine similarity), not as a bit-level reference.
"""
from __future__ import annotations

from dataclasses import replace

import numpy as np

from .capi import SRC_ELECTRIC
from .solver import Shot, f_to_d

_DIRS = ("ex", "ey", "ez")


def satan_gamma(nx: int, ny: int, nz: int, ncpml: int, rec_pos, obs, e_ff, e_bb, normalize: bool = True,
                grad=None, residual=None, device: int = 0) -> dict:
    """satan_i's residualE + sensitivity + conv_GdelE + calc_gamma
    (fwi3d_cpu_function_v1.4.c:2202-2384) in one GPU pass
    (``mittet_satan_gamma``).  Arrays in satan_i's layouts, cells [nz, ny, nx]:

      rec_pos [nrec, 3] 1-based;  obs [3, nrec, nf];  e_ff [3, nf, nz, ny, nx];
      e_bb [3 comp, nrec, 3 dir, nf, nz, ny, nx]

    Returns dict(err_sum, de [3, nrec, nf], sense [nz, ny, nx],
    e_back [3, nf, nz, ny, nx], grad [nz, ny, nx]); grad is ``grad`` (or
    zeros) plus this call's gamma, inside [ncpml, n - ncpml) only.  With
    ``obs=None`` the residual [3, nrec, nf] is given as ``residual`` instead
    of being formed from obs (residualE skipped)."""
    import ctypes

    from . import capi

    def cbuf(a, shape):
        a = np.asarray(a, dtype=np.complex128).reshape(shape)
        return np.ascontiguousarray(a).view(np.float64)

    nrec = int(np.asarray(rec_pos).reshape(-1, 3).shape[0]) if len(rec_pos) else 0
    e_ff = np.asarray(e_ff)
    nf = e_ff.shape[1]
    n = nx * ny * nz
    pos = np.ascontiguousarray(np.asarray(rec_pos, dtype=np.int32).reshape(-1, 3))
    o = cbuf(obs, (3, nrec, nf)) if (nrec and obs is not None) else None
    ff = cbuf(e_ff, (3, nf, n))
    bb = cbuf(e_bb, (3, nrec, 3, nf, n)) if nrec else np.zeros(2)
    g = np.zeros(n) if grad is None else np.array(grad, dtype=np.float64).reshape(n)
    err = np.zeros(1)
    de = np.zeros(3 * max(nrec, 1) * nf * 2)
    if o is None and nrec:  # the residual itself is given
        de[: 3 * nrec * nf * 2] = cbuf(residual, (3, nrec, nf)).ravel()
    sense = np.zeros(n)
    back = np.zeros(3 * nf * n * 2)
    D = ctypes.POINTER(ctypes.c_double)
    dp = lambda a: a.ctypes.data_as(D)  # noqa: E731
    grid = capi.Grid(nx, ny, nz, 1.0, 1.0, 1.0, ncpml)
    capi.check(capi.load().mittet_satan_gamma(device, ctypes.byref(grid), nrec,
                                              pos.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), nf, dp(o) if o is not None else None, dp(ff),
                                              dp(bb), 1 if normalize else 0, dp(err), dp(de), dp(sense), dp(back),
                                              dp(g)))
    cplx = lambda a: a[0::2] + 1j * a[1::2]  # noqa: E731
    return {"err_sum": float(err[0]), "de": cplx(de)[: 3 * nrec * nf].reshape(3, nrec, nf),
            "sense": sense.reshape(nz, ny, nx), "e_back": cplx(back).reshape(3, nf, nz, ny, nx),
            "grad": g.reshape(nz, ny, nx)}


def satan_formula_gradient(wl, obs: np.ndarray, normalize: bool = False, shot: int = 0, current_factor: bool = True):
    """Born gradient of one shot of workload ``wl`` (satan_i calc_gamma form).

    obs: [nshot, nrec, nf] observed spectra at wl.receivers / wl.omega.
    Returns (grad [nz, ny, nx], ecal [nrec, nf]).  Only electric receivers
    contribute, as in satan_i.  The reduction over receivers, directions and
    frequencies is ``satan_gamma`` (the GPU kernel pinned to satan_i's own
    functions) with E_ff = E / J_w, E_bb = the dipole spectra and
    dE = the residual of each receiver's component."""
    from . import workloads as W

    cp = wl.cp
    src = replace(wl, shots=[wl.shots[shot]], volume_dft="xyz")
    with W.make_solver(src) as s:
        ecal, _ = s.forward(wl.nt)
        eff = np.stack([s.volume_dft(0, c) for c in _DIRS])  # [3, nf, nz, ny, nx]
    ecal = ecal[0]
    dE = np.asarray(obs)[shot] - ecal
    # one shot per (receiver position, direction); residual of that component
    positions = []
    for (x, y, z, comp) in wl.receivers:
        if comp in _DIRS and (x, y, z) not in positions:
            positions.append((x, y, z))
    index = {(r[0], r[1], r[2], r[3]): q for q, r in enumerate(wl.receivers)}
    nf = len(wl.omega)
    shots, slots = [], []
    for p, (x, y, z) in enumerate(positions):
        for d, name in enumerate(_DIRS):
            if index.get((x, y, z, name)) is not None:
                shots.append(Shot(points=[(x, y, z, name, SRC_ELECTRIC, 1.0)]))
                slots.append((p, d))
    jw = f_to_d(np.asarray(wl.wavelet[:wl.nt], dtype=np.float64)[None], cp.dt, cp.omega0, wl.omega,
                h_factor=current_factor)[0]
    nx, ny, nz = cp.nx, cp.ny, cp.nz
    e_bb = np.zeros((3, len(positions), 3, nf, nz, ny, nx), dtype=np.complex128)
    # the residual of each (position, direction); zero where no receiver
    res = np.zeros((3, len(positions), nf), dtype=np.complex128)
    if shots:
        back = replace(wl, shots=shots, volume_dft="xyz")
        with W.make_solver(back) as s:
            s.forward(wl.nt)
            for k, (p, d) in enumerate(slots):
                for c, name in enumerate(_DIRS):
                    e_bb[c, p, d] = s.volume_dft(k, name)
                res[d, p] = dE[index[(*positions[p], _DIRS[d])]]
    e_ff = eff / jw[None, :, None, None, None]
    pos = np.array(positions, dtype=np.int32).reshape(-1, 3)
    r = satan_gamma(nx, ny, nz, cp.ncpml, pos, None, e_ff, e_bb, normalize=normalize, residual=res)
    return r["grad"] * (1.0 if normalize else cp.dx * cp.dy * cp.dz), ecal


def compare(g_ref: np.ndarray, g: np.ndarray) -> dict:
    """Cosine similarity and least-squares-scaled relative L2 of two gradients."""
    a, b = g_ref.ravel(), g.ravel()
    cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))
    s = float(a @ b / (b @ b))
    return {"cosine": cos, "ls_scale": s, "ls_rel_l2": float(np.linalg.norm(a - s * b) / np.linalg.norm(a))}
