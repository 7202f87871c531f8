"""GPU pins of the f_to_d transforms and satan_i's gradient formula to the
reference's own satan_i functions (golden fixtures made by
tests/golden/make_golden.py from the compiled reference):

* laplaceToFreq (fwi3d_cpu_function_v1.4.c:1976-2089): the receiver f_to_d of
  the GPU (mittet_f_to_d, trace_dft_kernel), E spectra and the
  sqrt(-2 w0/(i w)) current factor, FP64 <= 1e-10.
* laplaceToFreq_2 (:2091-2200) over copytoEcal's history (:1652-1686): the
  full-volume f_to_d the GPU accumulates on the fly (ring + FP64 flush) during
  a solve of the same model and source, FP64 <= 1e-10, FP32 <= 1e-4.
* residualE, sensitivity, conv_GdelE, calc_gamma (:2202-2384): the one-pass
  GPU kernel mittet_satan_gamma, FP64 <= 1e-12 (sense normalisation on and off).
"""
import os

import numpy as np
import pytest

from mittet_main_b200 import born
from mittet_main_b200.capi import FLAVOR_SATAN_I, FP32, FP64, SRC_ELECTRIC
from mittet_main_b200.solver import ConstPara, MittetSolver, Shot, f_to_d
from oracle import oracle as O
from tests.conftest import rel_l2
from tests.golden.make_golden import gamma_inputs
from tests.test_reference_pins import _ftod_inputs, _load

pytestmark = pytest.mark.gpu


def test_gpu_f_to_d_matches_reference_laplace_to_freq(golden_dir):
    traces, jx, dt, om0, omegas, f = _ftod_inputs(golden_dir)
    spec = f["spec"]
    got = f_to_d(traces, dt, om0, omegas)  # [nrec, 3, it]
    assert rel_l2(got, spec[:, :3]) <= 1e-10
    for r in range(traces.shape[0]):
        for c in range(3):
            assert rel_l2(got[r, c], spec[r, c]) <= 1e-10, (r, c)
    jw = f_to_d(jx[None], dt, om0, omegas[1:], h_factor=True)[0]
    assert rel_l2(jw, spec[0, 3, 1:]) <= 1e-10


@pytest.mark.parametrize("prec", [FP64, FP32])
def test_gpu_volume_dft_matches_reference_laplace_to_freq_2(golden_dir, prec):
    g = _load(golden_dir, "satan_volume")
    ix, iy, iz = (int(v) for v in g["shape"])
    d, nt, nvol = float(g["d"]), int(g["nt"]), int(g["nvol"])
    om0 = float(g["omega0"])
    cp = ConstPara(nx=ix, ny=iy, nz=iz, dx=d, dy=d, dz=d, ncpml=int(g["ncpml"]), dt=float(g["dt"]),
                   cmax=float(g["cmax"]), omega0=om0, mu0=O.MU0_C, flavor=FLAVOR_SATAN_I, precision=prec,
                   check_cfl=False)
    # the reference transforms it = nt + 1 samples (its last one never written, zero)
    om = 2.0 * np.pi / (nt + 1) / cp.dt
    w = np.arange(1, nvol)
    omegas = om * w
    src = [int(v) for v in g["src"]]
    with MittetSolver(cp) as s:
        s.set_model(g["sigma"])
        s.set_shots([Shot(points=[(src[0], src[1], src[2], "ex", SRC_ELECTRIC, 1.0)])])
        s.set_wavelet(g["wavelet"])
        s.set_receivers([])
        s.set_freqs(omegas)
        s.set_volume_dft("xyz")
        s.forward(nt)
        vol = np.stack([s.volume_dft(0, c).reshape(len(w), -1)[:, g["cells"]] for c in ("ex", "ey", "ez")])
    # G = E / J with J = sqrt(-2 w0/(i w)) (a unit current impulse) and out_True = 1
    jfac = np.sqrt(2.0 * om0 / omegas) * np.exp(1j * np.pi / 4)
    ref = g["vol"] * jfac[None, :, None]
    assert np.abs(ref).max() > 0
    tol = 1e-10 if prec == FP64 else 1e-4
    assert rel_l2(vol, ref) <= tol
    for c in range(3):
        assert rel_l2(vol[c], ref[c]) <= tol * 10, c


@pytest.mark.parametrize("normalize", [True, False])
def test_gpu_satan_gamma_matches_reference(golden_dir, normalize):
    a = gamma_inputs()
    ref = _load(golden_dir, "satan_gamma")
    ix, iy, iz = a["shape"]
    shp = (iz, iy, ix)
    nf = a["e_ff"].shape[1]
    nrec = len(a["rec_pos"])
    r = born.satan_gamma(ix, iy, iz, a["ncpml"], a["rec_pos"], a["obs"],
                         a["e_ff"].reshape(3, nf, *shp), a["e_bb"].reshape(3, nrec, 3, nf, *shp),
                         normalize=normalize)
    assert r["err_sum"] == pytest.approx(float(ref["err_sum"]), rel=1e-12)
    assert rel_l2(r["de"], ref["de"]) <= 1e-12
    assert rel_l2(r["sense"].ravel(), ref["sense"]) <= 1e-12
    assert rel_l2(r["e_back"].reshape(3, nf, -1), ref["e_back"]) <= 1e-12
    if normalize:
        assert rel_l2(r["grad"].ravel(), ref["grad"]) <= 1e-12
    else:
        want = np.where(ref["grad"] != 0, ref["grad"] * ref["sense"], 0.0)
        assert rel_l2(r["grad"].ravel(), want) <= 1e-12
    # grad accumulates (calc_gamma's +=) and the residual can be given directly
    r2 = born.satan_gamma(ix, iy, iz, a["ncpml"], a["rec_pos"], None, a["e_ff"].reshape(3, nf, *shp),
                          a["e_bb"].reshape(3, nrec, 3, nf, *shp), normalize=normalize, grad=r["grad"],
                          residual=r["de"])
    assert rel_l2(r2["grad"], 2 * r["grad"]) <= 1e-12
