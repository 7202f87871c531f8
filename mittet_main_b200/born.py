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


def satan_formula_gradient(wl, obs: np.ndarray, normalize: bool = False, shot: int = 0, current_factor: bool = True):
    """Born gradient of one shot of workload ``wl`` (satan_i calc_gamma form).

    obs: [nshot, nrec, nf] observed spectra at wl.receivers / wl.omega.
    Returns (grad [nz, ny, nx], ecal [nrec, nf]).  Only electric receivers
    contribute, as in satan_i."""
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
    shots, weights = [], []
    for (x, y, z) in positions:
        for d in _DIRS:
            q = index.get((x, y, z, d))
            if q is None:
                continue
            shots.append(Shot(points=[(x, y, z, d, SRC_ELECTRIC, 1.0)]))
            weights.append(np.conj(dE[q]))  # [nf]
    nf = len(wl.omega)
    eback = np.zeros_like(eff)
    sense = np.zeros(eff.shape[2:]) if normalize else None
    if shots:
        back = replace(wl, shots=shots, volume_dft="xyz")
        with W.make_solver(back) as s:
            s.forward(wl.nt)
            for k, wgt in enumerate(weights):
                for c, name in enumerate(_DIRS):
                    g = s.volume_dft(k, name)  # [nf, nz, ny, nx]
                    eback[c] += g * wgt[:, None, None, None]
                    if normalize:
                        sense += np.abs(eff[c] * g).sum(axis=0)
    jw = f_to_d(np.asarray(wl.wavelet[:wl.nt], dtype=np.float64)[None], cp.dt, cp.omega0, wl.omega,
                h_factor=current_factor)[0]
    prod = (eff * eback).sum(axis=0)  # [nf, nz, ny, nx]
    grad = np.real(prod / jw[:, None, None, None]).sum(axis=0) * (cp.dx * cp.dy * cp.dz)
    if normalize:
        grad = grad / np.where(sense > 0, sense, 1.0)
    nc = cp.ncpml
    out = np.zeros_like(grad)
    out[nc:-nc, nc:-nc, nc:-nc] = grad[nc:-nc, nc:-nc, nc:-nc]
    return out, ecal


def compare(g_ref: np.ndarray, g: np.ndarray) -> dict:
    """Cosine similarity and least-squares-scaled relative L2 of two gradients."""
    a, b = g_ref.ravel(), g.ravel()
    cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))
    s = float(a @ b / (b @ b))
    return {"cosine": cos, "ls_scale": s, "ls_rel_l2": float(np.linalg.norm(a - s * b) / np.linalg.norm(a))}
