"""CPU pins of the oracle's restatements to the reference's own satan_i code.

The golden fixtures are outputs of the reference's functions compiled from
their sources (tests/golden/make_golden.py, oracle/ref_satan_driver.c):

* laplaceToFreq (fwi3d_cpu_function_v1.4.c:1976-2089): the damped DFT of
  receiver traces and the sqrt(-2 w0/(i w)) current factor -> oracle.dft.
* residualE, sensitivity, conv_GdelE, calc_gamma (:2202-2384)
  -> oracle.satan_gamma.
* calc_phi, calc_alpha, update_para2 (:2565-2603, 2757-2832)
  -> oracle.calc_phi, oracle.update_para2.
* Text files the reference wrote in those runs (spectrum_*_SSS_RRR.dat,
  gradient_III.dat, sig_III.dat) -> mittet_main_b200.formats readers.
"""
import os

import numpy as np
import pytest

from mittet_main_b200 import formats
from oracle import oracle as O
from tests.conftest import rel_l2
from tests.golden.make_golden import gamma_inputs, update_inputs


def _load(golden_dir, name):
    return dict(np.load(os.path.join(golden_dir, name + ".npz")))


def _ftod_inputs(golden_dir):
    g = _load(golden_dir, "satan_ex")
    f = _load(golden_dir, "satan_ftod")
    rec = g["receivers"]
    traces = np.stack([np.stack([g["traces"][[q for q, r in enumerate(rec) if tuple(r[:3]) == tuple(p) and r[3] == c][0]]
                                 for c in range(3)]) for p in f["positions"]])
    it = traces.shape[2]
    dt, om0 = float(g["dt"]), float(g["omega0"])
    om = 2.0 * np.pi / it / dt  # laplaceToFreq's om = 2.f*M_PI/it/dt
    return traces, g["wavelet"][:it], dt, om0, om * np.arange(it), f


def test_oracle_dft_matches_reference_laplace_to_freq(golden_dir):
    traces, jx, dt, om0, omegas, f = _ftod_inputs(golden_dir)
    spec = f["spec"]  # [nrec, 4 (EX_w EY_w EZ_w JX_w), it]
    for r in range(traces.shape[0]):
        for c in range(3):
            got = O.dft(traces[r, c], dt, om0, omegas)
            assert rel_l2(got, spec[r, c]) <= 1e-12, (r, c)
    # the current factor sqrt(-2 w0/(i w)) (JX_w; w = 0 is overwritten by the reference)
    got = O.dft(jx, dt, om0, omegas[1:], h_factor=True)
    assert rel_l2(got, spec[0, 3, 1:]) <= 1e-12
    assert spec[0, 3, 0] == pytest.approx(2 * om0)


def test_oracle_satan_gamma_matches_reference(golden_dir):
    a = gamma_inputs()
    ref = _load(golden_dir, "satan_gamma")
    got = O.satan_gamma(a["shape"], a["ncpml"], a["rec_pos"], a["obs"], a["e_ff"], a["e_bb"])
    assert got["err_sum"] == pytest.approx(float(ref["err_sum"]), rel=1e-13)
    for k in ("de", "sense", "e_back", "grad"):
        assert rel_l2(got[k], ref[k]) <= 1e-13, k
    ix, iy, iz = a["shape"]
    g = ref["grad"].reshape(iz, iy, ix)
    nc = a["ncpml"]
    inner = np.zeros_like(g, dtype=bool)
    inner[nc:iz - nc, nc:iy - nc, nc:ix - nc] = True
    assert np.all(g[~inner] == 0.0) and np.all(g[inner] != 0.0)  # calc_gamma's range


def test_oracle_model_update_matches_reference(golden_dir):
    a = update_inputs()
    ref = _load(golden_dir, "satan_update")
    ix, iy, iz = a["shape"]
    sig = a["sig"].reshape(iz, iy, ix)
    grad = a["grad"].reshape(iz, iy, ix)
    scaler, sig2 = O.calc_phi(sig, grad, a["iseabed"])
    assert scaler == float(ref["scaler"])
    assert np.array_equal(sig2.ravel(), ref["sig2"])
    cells = [((z - 1) * iy + (y - 1)) * ix + (x - 1) for (x, y, z) in a["rec_pos"]]
    # receiver values in the reference's summation order: receiver, frequency, x y z
    ecal = a["e_ffl"][:, :, cells].transpose(2, 1, 0)
    e2 = a["e_ff2"][:, :, cells].transpose(2, 1, 0)
    obs = a["de"].transpose(1, 2, 0) + ecal
    new, alpha = O.update_para2(sig, grad, obs, ecal, e2, scaler, a["iseabed"], a["minval"], a["maxval"], a["ncpml"])
    assert alpha == pytest.approx(float(ref["alpha"]), rel=1e-13)
    assert rel_l2(new.ravel(), ref["sig"]) <= 1e-15


def test_formats_read_files_the_reference_wrote(golden_dir, tmp_path):
    rf = os.path.join(golden_dir, "ref_files")
    # laplaceToFreq: spectrum_e (EX_w, every frequency of the grid) and
    # spectrum_ex (OBSX_f = EX_w / JX_w * out_True, out_True = 1 here, n < upperF)
    f = _load(golden_dir, "satan_ftod")
    spec = f["spec"][0]
    it = spec.shape[1]
    e = formats.read_spectrum(os.path.join(rf, "spectrum_e_000_000.dat"), it)
    assert e.shape == (it,)
    assert np.allclose(e, spec[0], rtol=1e-5, atol=1e-6 * np.abs(spec[0]).max())
    uf = int(f["upper_f"])
    ex = formats.read_spectrum(os.path.join(rf, "spectrum_ex_000_000.dat"), uf)
    gx = spec[0, :uf] / spec[3, :uf]
    assert np.allclose(ex, gx, rtol=1e-5, atol=1e-6 * np.abs(gx).max())
    # update_para2: gradient_000.dat = alpha * scaler * grad, sig_000.dat = the new model
    a = update_inputs()
    ref = _load(golden_dir, "satan_update")
    ix, iy, iz = a["shape"]
    gr = formats.read_volume(os.path.join(rf, "gradient_000.dat"), ix, iy, iz)
    want = float(ref["alpha"]) * float(ref["scaler"]) * a["grad"].reshape(iz, iy, ix)
    assert np.allclose(gr, want, rtol=1e-5, atol=0)
    sg = formats.read_volume(os.path.join(rf, "sig_000.dat"), ix, iy, iz)
    assert np.allclose(sg, ref["sig"].reshape(iz, iy, ix), rtol=1e-5, atol=0)
    # and the writer produces the same layout
    out = str(tmp_path / "sig_000.dat")
    formats.write_volume(out, ref["sig"].reshape(iz, iy, ix), *a["d"])
    with open(out) as fa, open(os.path.join(rf, "sig_000.dat")) as fb:
        assert fa.read().split() == fb.read().split()
