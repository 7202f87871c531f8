"""CPU: the oracle's discrete adjoint gradient against central finite
differences of the oracle forward (the forward is pinned to the reference's
own kernels).  Tolerance: 1e-3 relative, the gradient bar of the workload."""
import numpy as np
import pytest

from oracle import oracle as O


def small_problem(seed=5, nt=120):
    nx, ny, nz, nc = 24, 22, 20, 6
    rng = np.random.default_rng(seed)
    sig = 10 ** rng.normal(np.log10(0.3), 0.2, size=(nz, ny, nx))
    d = 50.0
    om0 = 2 * O.PI_F
    cmax = np.sqrt(2 * om0 / O.MU0_F / sig.min())
    dt = 0.95 * d / (cmax * np.sqrt(3) * 1.16667)
    p = O.Params(nx=nx, ny=ny, nz=nz, dx=d, dy=d, dz=d, dt=dt, ncpml=nc, cmax=cmax)
    fmax = 0.9 * np.sqrt(2 * om0 / O.MU0_F / sig.max()) / (10.4 * d)
    t = np.arange(nt + 2) * dt
    t0, beta = np.pi / fmax, np.pi * fmax ** 2
    w = -2 * beta * (t - t0) * np.sqrt(beta / np.pi) * np.exp(-beta * (t - t0) ** 2)
    src = [(12, 11, 8, "ex", O.SRC_ELECTRIC, 1.0), (8, 8, 12, "hz", O.SRC_MAGNETIC, 1e-3)]
    rec = [(x, y, z, c) for (x, y, z) in [(4, 5, 6), (16, 11, 14), (12, 4, 9), (20, 18, 16)]
           for c in ("ex", "ey", "hz", "hx")]
    omega = 2 * np.pi * np.array([0.5, 1.0, 2.0, 4.0])
    mu = np.full(sig.shape, O.MU0_F)
    return p, sig, mu, src, w, rec, nt, omega


def test_oracle_gradient_matches_finite_differences():
    p, sig, mu, src, w, rec, nt, omega = small_problem()
    rng = np.random.default_rng(1)
    obs = (rng.normal(size=(len(rec), omega.size)) + 1j * rng.normal(size=(len(rec), omega.size))) * 1e-14
    J, g, spec = O.gradient(p, sig, mu, src, w, rec, nt, omega, obs)
    assert J == pytest.approx(O.misfit(p, sig, mu, src, w, rec, nt, omega, obs), rel=1e-12)
    cells = [(5, 6, 7), (12, 11, 8), (10, 10, 16), (8, 8, 12), (14, 9, 6), (3, 3, 3), (19, 17, 15), (12, 11, 9)]
    gmax = np.abs(g).max()
    for (i, j, k) in cells:
        dd = 1e-4 * sig[k, j, i]
        sp = sig.copy(); sp[k, j, i] += dd
        sm = sig.copy(); sm[k, j, i] -= dd
        fd = (O.misfit(p, sp, mu, src, w, rec, nt, omega, obs) - O.misfit(p, sm, mu, src, w, rec, nt, omega, obs)) / (2 * dd)
        assert abs(g[k, j, i] - fd) <= 1e-3 * max(abs(fd), 1e-6 * gmax), (i, j, k, g[k, j, i], fd)


def test_oracle_gradient_is_zero_for_matching_data():
    p, sig, mu, src, w, rec, nt, omega = small_problem(nt=60)
    _, _, spec = O.gradient(p, sig, mu, src, w, rec, nt, omega, np.zeros((len(rec), omega.size)))
    J, g, _ = O.gradient(p, sig, mu, src, w, rec, nt, omega, spec)
    assert J == 0.0 and np.abs(g).max() == 0.0


def test_restated_model_update_on_a_hand_case():
    """oracle.calc_phi / oracle.update_para2 on a 4x4x4 case worked by hand."""
    sig = np.full((4, 4, 4), 0.5)
    sig[0, 0, 0] = 0.25
    sig[1, 1, 1] = 2.0
    grad = np.zeros((4, 4, 4))
    grad[1, 1, 1] = 4.0
    grad[2, 2, 2] = 8.0   # below the seabed (k = 2 > 1): not in the maxima
    scaler, sig2 = O.calc_phi(sig, grad, iseabed=1)
    assert scaler == float(np.float32(0.01)) * 2.0 / 4.0
    assert sig2[1, 1, 1] == 2.0 - scaler * 4.0 and sig2[2, 2, 2] == 0.5 - scaler * 8.0
    obs = np.array([[[1 + 1j]]])
    ecal = np.array([[[0.5 + 0j]]])
    e2 = np.array([[[0.5 + 0.5j]]])
    new, alpha = O.update_para2(sig, grad, obs, ecal, e2, scaler, iseabed=1, minval=0.1, maxval=1.9, ncpml=1)
    k1 = (0.5 + 1j) * 0.5j
    k2 = (0.5j) ** 2
    assert alpha == 3.0 * abs(k1) / abs(k2)
    assert new[1, 1, 1] == 1.9                       # clamped to maxval
    assert new[2, 2, 2] == 0.5                       # below the seabed: only clamped
    assert new[0, 0, 0] == 0.25                      # CPML frame untouched
