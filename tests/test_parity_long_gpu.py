"""GPU parity at the benchmark configurations, over thousands of steps.

* The 64^3 CPU configuration exactly (two-layer 0.01 / 1.0 S/m model, Ex
  dipole at (32, 32, 30), Nt = 3000, 32 receivers x 6 components, f_to_d at
  0.25 / 0.5 / 1 / 2 Hz): receiver E and H spectra of the GPU solve against
  the FP64 oracle's, FP64 <= 1e-10 and FP32 <= 1e-4 rel-L2.
  - satan_i flavour: a bounded solve, the parity claim proper.
  - ncver0027 flavour: its negative magnetic CPML conductivity at i = ncpml
    (cpu_cpml4.f90:27) makes this thin-CPML solve grow without bound (trace
    maxima ~1e98 at step 3000), as the reference's would.  FP64 still matches
    the oracle to 1e-10 (both carry the same growing mode); FP32 overflows and
    the solve reports MITTET_ERR_DIVERGED.
* The full-volume f_to_d over Nt = 3000 steps on a 128x128x96 twin of the
  256x256x192 workload (log-normal blocks + resistive body, 16-cell CPML,
  ncver0027 flavour): the accumulated spectra at 48 cells against the
  oracle's DFT of its traces at those cells, FP32 <= 1e-4, FP64 <= 1e-10.
"""
import numpy as np
import pytest

from mittet_main_b200 import workloads as W
from mittet_main_b200.capi import FLAVOR_NCVER0027, FLAVOR_SATAN_I, FP32, FP64, MittetError
from oracle import oracle as O
from tests.conftest import rel_l2
from tests.test_parity_gpu import check_spectra, oracle_run

pytestmark = pytest.mark.gpu
TOL = {FP64: 1e-10, FP32: 1e-4}

_cache = {}


def _c1_oracle(flavor):
    if flavor not in _cache:
        wl = W.plain_cpu(flavor=flavor)
        _cache[flavor] = oracle_run(wl)
    return _cache[flavor]


@pytest.mark.parametrize("prec", [FP64, FP32])
def test_c1_satan_full_length_matches_oracle(prec):
    wl = W.plain_cpu(precision=prec, flavor=FLAVOR_SATAN_I)
    assert wl.nt == 3000 and wl.cp.nx == 64 and len(wl.receivers) == 32 * 6
    ref = _c1_oracle(FLAVOR_SATAN_I)
    with W.make_solver(wl) as s:
        spec, td = s.forward(wl.nt, want_traces=True)
    # the solve is bounded and has decayed well below its peak by the end
    assert np.isfinite(ref[0]).all()
    assert np.abs(ref[0][:, -200:]).max() < 1e-2 * np.abs(ref[0]).max()
    check_spectra(wl, spec, ref, TOL[prec])
    assert rel_l2(td[0], ref[0]) <= TOL[prec] * (1 if prec == FP64 else 10)


def test_c1_ncver_fp64_matches_oracle_while_growing():
    wl = W.plain_cpu(precision=FP64, flavor=FLAVOR_NCVER0027)
    ref = _c1_oracle(FLAVOR_NCVER0027)
    assert np.abs(ref[0]).max() > 1e40  # the reference scheme grows on this grid
    with W.make_solver(wl) as s:
        spec, td = s.forward(wl.nt, want_traces=True)
    check_spectra(wl, spec, ref, TOL[FP64])


def test_c1_ncver_fp32_reports_divergence():
    wl = W.plain_cpu(precision=FP32, flavor=FLAVOR_NCVER0027)
    with W.make_solver(wl) as s:
        with pytest.raises(MittetError) as ex:
            s.forward(wl.nt)
    assert ex.value.name == "MITTET_ERR_DIVERGED"


def _long_case(prec):
    wl = W.plain_gpu(nt=3000, nx=128, ny=128, nz=96, precision=prec, volume=True)
    rng = np.random.default_rng(2026)
    cp = wl.cp
    cells = [(int(rng.integers(1, cp.nx + 1)), int(rng.integers(1, cp.ny + 1)), int(rng.integers(1, cp.nz + 1)))
             for _ in range(40)]
    sx, sy, sz = wl.shots[0].points[0][:3]
    cells += [(sx + dx, sy + dy, sz + dz) for (dx, dy, dz) in
              [(0, 0, 0), (3, 0, 1), (-5, 2, 4), (0, -8, 10), (12, 12, 20), (-20, 6, 30), (1, 1, 50), (30, -30, 5)]]
    return wl, cells


def _long_oracle():
    if "long" not in _cache:
        wl, cells = _long_case(FP64)
        mu = np.full(wl.sigma.shape, wl.cp.mu0)
        from tests.test_parity_gpu import oracle_params
        rec = [(x, y, z, c) for (x, y, z) in cells for c in ("ex", "ey", "ez")]
        tr = O.forward(oracle_params(wl.cp), wl.sigma, mu, wl.shots[0].points, wl.wavelet, rec, wl.nt)
        spec = np.stack([O.dft(t, wl.cp.dt, wl.cp.omega0, wl.omega) for t in tr])  # [ncell*3, nf]
        _cache["long"] = spec.reshape(len(cells), 3, -1)
    return _cache["long"]


@pytest.mark.parametrize("prec", [FP32, FP64])
def test_volume_dft_3000_steps_matches_oracle(prec):
    wl, cells = _long_case(prec)
    ref = _long_oracle()
    with W.make_solver(wl) as s:
        s.forward(wl.nt)
        vol = np.stack([s.volume_dft(0, "e" + c) for c in "xyz"])  # [3, nf, nz, ny, nx]
    got = np.stack([vol[:, :, z - 1, y - 1, x - 1] for (x, y, z) in cells])  # [ncell, 3, nf]
    assert np.abs(ref).max() > 0
    err = rel_l2(got, ref)
    assert err <= TOL[prec], f"volume spectra rel-L2 {err:.3e}"
    # per frequency too: the highest frequency decays fastest, so it carries the least energy
    for f in range(ref.shape[2]):
        ef = rel_l2(got[:, :, f], ref[:, :, f])
        assert ef <= TOL[prec] * 10, f"freq {f}: rel-L2 {ef:.3e}"
