"""CPU tests of the oracle: pinned against the reference's own satan_i
kernels (golden fixtures) and restated formulae.  No GPU."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import rel_l2

NAMES = ["ex", "ey", "ez", "hx", "hy", "hz"]


def load(golden_dir, name):
    return dict(np.load(os.path.join(golden_dir, name + ".npz")))


def run_oracle_on_golden(g, want_fields=False):
    ix, iy, iz = (int(v) for v in g["shape"])
    p = O.satan_params(ix, iy, iz, float(g["d"]), float(g["d"]), float(g["d"]), int(g["ncpml"]),
                       float(g["omega0"]), float(g["sigma"].min()))
    p.dt = float(g["dt"])
    p.cmax = float(g["cmax"])
    src = tuple(int(v) for v in g["src"])
    srcs = [(src[0], src[1], src[2], NAMES[int(g["src_comp"])], O.SRC_ELECTRIC, 1.0)]
    rec = [(int(r[0]), int(r[1]), int(r[2]), NAMES[int(r[3])]) for r in g["receivers"]]
    mu = np.full(g["sigma"].shape, O.MU0_C)
    return O.forward(p, g["sigma"], mu, srcs, g["wavelet"], rec, int(g["nt"]), want_fields=want_fields)


@pytest.mark.parametrize("name", ["satan_ex", "satan_ey", "satan_ez"])
def test_oracle_matches_reference_bit_for_bit(golden_dir, name):
    g = load(golden_dir, name)
    want = "fields" in g
    out = run_oracle_on_golden(g, want_fields=want)
    tr = out[0] if want else out
    assert np.array_equal(tr, g["traces"]), f"max diff {np.abs(tr - g['traces']).max()}"
    assert np.abs(g["traces"]).max() > 0
    if want:
        assert np.array_equal(out[1], g["fields"])


def test_golden_fixture_has_signal_in_every_slab(golden_dir):
    g = load(golden_dir, "satan_ex")
    F = g["fields"]
    nc = int(g["ncpml"])
    # CPML psi terms touched the slabs: fields there are non-zero
    assert np.abs(F[:, :, :, 2:nc]).max() > 0
    assert np.abs(F[:, 2:nc, :, :]).max() > 0
    assert np.abs(F[:, :, 2:nc, :]).max() > 0


def test_dft_matches_direct_formula():
    rng = np.random.default_rng(0)
    x = rng.normal(size=300)
    dt, w0 = 1e-3, 2 * np.pi
    om = np.array([0.3, 2.0, 7.5, 40.0])
    got = O.dft(x, dt, w0, om)
    n = np.arange(x.size)
    ref = np.array([np.sum(x * dt * np.exp((1j - 1) * np.sqrt(w0 * w) * n * dt)) for w in om])
    assert rel_l2(got, ref) < 1e-13
    goth = O.dft(x, dt, w0, om, h_factor=True)
    assert rel_l2(goth, ref * np.sqrt(-2 * w0 / 1j / om)) < 1e-13


def test_dft_h_factor_zero_frequency_is_not_finite():
    # ncver0027/cpu_f_to_d_h.f90:146 divides by om*k; row k = 0 is non-finite
    out = O.dft(np.ones(10), 1e-3, 2 * np.pi, np.array([0.0]), h_factor=True)
    assert not np.isfinite(out[0])


def test_ncver_profiles_restated():
    p = O.Params(nx=40, ny=36, nz=30, dx=50., dy=50., dz=50., dt=7e-4, ncpml=10, cmax=31623.)
    pr = O.profiles(p)
    nc = 10
    sig_max = 4.0 * p.cmax * np.log(100.0) / (2 * nc * p.dx)
    # esig_x(i) = sig_max ((ncpml - i)/(ncpml - 1))^3, i 1-based (cpu_cpml4.f90:26)
    for i1 in (1, 5, 10):
        assert pr[0, 0, i1 - 1] == pytest.approx(sig_max * ((nc - i1) / (nc - 1)) ** 3, rel=1e-14)
    # msig at i = ncpml is negative ((-0.5)/(ncpml-1))^3 (cpu_cpml4.f90:27)
    assert pr[0, 1, nc - 1] < 0
    # far side mirrored: esig_x(nx-(i-1)) = esig_x(i)
    assert np.array_equal(pr[0, :, :nc], pr[0, :, p.nx - 1:p.nx - nc - 1:-1])
    # interior: sigma 0, ked = dx
    assert np.all(pr[0, 0, nc:p.nx - nc] == 0) and np.all(pr[0, 6, nc:p.nx - nc] == p.dx)


def test_ncver_ranges_restated():
    p = O.Params(nx=40, ny=36, nz=30, dx=50., dy=50., dz=50., dt=7e-4, ncpml=10, cmax=31623.)
    r = O.ranges(p).reshape(-1)
    upd = r[:36].reshape(6, 2, 3)
    # Ex: k 3..nz-1, j 3..ny-1, i 1..nx (1-based, cpu_eh_field_cpml42.f90:127-129)
    assert upd[0].tolist() == [[0, 2, 2], [40, 35, 29]]
    # Hz: k 1..nz, j 2..ny-2, i 2..nx-2 (:244-246)
    assert upd[5].tolist() == [[1, 1, 0], [38, 34, 30]]
    slabs = r[36:].reshape(6, 10)
    # CPML_E4 x: i 3..ncpml+1 and nx-ncpml+1..nx-1 (cpu_cpml4.f90:283,296)
    assert slabs[0, :4].tolist() == [2, 11, 30, 39]
    # CPML_H4 x: i 2..ncpml and nx-ncpml..nx-2 (:396,409)
    assert slabs[3, :4].tolist() == [1, 10, 29, 38]


def test_psi_hyx_typo_changes_only_h_slab_results():
    p = O.Params(nx=30, ny=28, nz=26, dx=50., dy=50., dz=50., dt=7e-4, ncpml=8, cmax=31623.)
    sig = np.full((26, 28, 30), 0.3)
    sig[:13] = 0.01
    mu = np.full(sig.shape, O.MU0_F)
    w = np.sin(np.arange(62) * 0.2) * np.exp(-((np.arange(62) - 15) / 6.0) ** 2)
    src = [(15, 14, 13, "hz", O.SRC_MAGNETIC, 1.0)]
    rec = [(15, 14, 16, "ex"), (3, 14, 13, "hy")]
    a = O.forward(p, sig, mu, src, w, rec, 60)
    p.psi_hyx_typo = 0
    b = O.forward(p, sig, mu, src, w, rec, 60)
    assert np.abs(a - b).max() > 0  # the typo matters once the wave reaches the x slab
