"""GPU parity of the forward path against the oracle and the reference's
own satan_i kernels (golden fixtures).  Tolerances (rel-L2 over all
receivers and frequencies of a component class):
  FP64 fields: 1e-10    FP32 fields + FP64 DFT: 1e-4
"""
import os
from dataclasses import replace

import numpy as np
import pytest

from mittet_main_b200 import workloads as W
from mittet_main_b200.capi import FLAVOR_NCVER0027, FLAVOR_SATAN_I, FP32, FP64, SRC_ELECTRIC, MittetError
from mittet_main_b200.solver import ConstPara, MittetSolver, Shot, f_to_d
from oracle import oracle as O
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu
NAMES = ["ex", "ey", "ez", "hx", "hy", "hz"]
TOL = {FP64: 1e-10, FP32: 1e-4}


def oracle_params(cp: ConstPara) -> O.Params:
    p = O.Params(nx=cp.nx, ny=cp.ny, nz=cp.nz, dx=cp.dx, dy=cp.dy, dz=cp.dz, dt=cp.dt, ncpml=cp.ncpml,
                 cmax=cp.cmax, omega0=cp.omega0, flavor=cp.flavor, e_sign=cp.e_sign, h_sign=cp.h_sign)
    if cp.flavor == FLAVOR_SATAN_I:
        p.c2, p.psi_hyx_typo = O.C2_C, 0
    return p


def oracle_run(wl: W.Workload, cp=None, want_fields=False):
    cp = cp or wl.cp
    mu = wl.mu if wl.mu is not None else np.full(wl.sigma.shape, cp.mu0)
    outs = []
    for shot in wl.shots:
        srcs = [(x, y, z, c, k, a) for (x, y, z, c, k, a) in shot.points]
        outs.append(O.forward(oracle_params(cp), wl.sigma, mu, srcs, wl.wavelet, wl.receivers, wl.nt,
                              want_fields=want_fields))
    return outs


def split_eh(wl, arr):
    ise = np.array([r[3] in ("ex", "ey", "ez") for r in wl.receivers])
    return arr[..., ise, :], arr[..., ~ise, :]


def check_spectra(wl, got, ref_traces, tol):
    """got: [nshot, nrec, nf]; ref_traces: list of [nrec, nt] oracle traces."""
    for s, tr in enumerate(ref_traces):
        ref = np.stack([O.dft(tr[r], wl.cp.dt, wl.cp.omega0, wl.omega, h_factor=wl.receivers[r][3].startswith("h"))
                        for r in range(len(wl.receivers))])
        ge, gh = split_eh(wl, got[s][None])
        re_, rh = split_eh(wl, ref[None])
        assert rel_l2(ge, re_) <= tol, f"E spectra rel-L2 {rel_l2(ge, re_):.3e}"
        if rh.size:
            assert rel_l2(gh, rh) <= tol, f"H spectra rel-L2 {rel_l2(gh, rh):.3e}"


# ------------------------------------------------ pinned: reference satan_i
@pytest.mark.parametrize("name", ["satan_ex", "satan_ey", "satan_ez"])
@pytest.mark.parametrize("prec", [FP64, FP32])
def test_gpu_matches_reference_satan_kernels(golden_dir, name, prec):
    g = dict(np.load(os.path.join(golden_dir, name + ".npz")))
    ix, iy, iz = (int(v) for v in g["shape"])
    d = float(g["d"])
    cp = ConstPara(nx=ix, ny=iy, nz=iz, dx=d, dy=d, dz=d, ncpml=int(g["ncpml"]), dt=float(g["dt"]),
                   cmax=float(g["cmax"]), omega0=float(g["omega0"]), mu0=O.MU0_C, flavor=FLAVOR_SATAN_I,
                   precision=prec, check_cfl=False)
    nt = int(g["nt"])
    with MittetSolver(cp) as s:
        s.set_model(g["sigma"])
        src = [int(v) for v in g["src"]]
        s.set_shots([Shot(points=[(src[0], src[1], src[2], NAMES[int(g["src_comp"])], SRC_ELECTRIC, 1.0)])])
        s.set_wavelet(g["wavelet"])
        s.set_receivers([(int(r[0]), int(r[1]), int(r[2]), NAMES[int(r[3])]) for r in g["receivers"]])
        _, td = s.forward(nt, want_traces=True)
        ref = g["traces"]
        ise = np.array([int(r[3]) < 3 for r in g["receivers"]])
        assert rel_l2(td[0][ise], ref[ise]) <= TOL[prec]
        assert rel_l2(td[0][~ise], ref[~ise]) <= TOL[prec]
        if "fields" in g:
            F = s.fields(0)
            for c in range(6):
                assert rel_l2(F[c], g["fields"][c]) <= TOL[prec] * 10, NAMES[c]


# ------------------------------------------------ ncver0027 flavour vs oracle
@pytest.mark.parametrize("prec", [FP64, FP32])
@pytest.mark.parametrize("magnetic", [False, True])
def test_gpu_matches_oracle_ncver_small(prec, magnetic):
    wl = W.small_case(nt=240, precision=prec, magnetic=magnetic)
    ref = oracle_run(wl)
    with W.make_solver(wl) as s:
        spec, td = s.forward(wl.nt, want_traces=True)
        assert rel_l2(td[0], ref[0]) <= TOL[prec]
        check_spectra(wl, spec, ref, TOL[prec])


def test_gpu_fp64_final_fields_match_oracle():
    wl = W.small_case(n=(34, 30, 28), ncpml=7, nt=150, precision=FP64, magnetic=True)
    tr, F = oracle_run(wl, want_fields=True)[0]
    with W.make_solver(wl) as s:
        s.forward(wl.nt)
        G = s.fields(0)
    for c in range(6):
        assert rel_l2(G[c], F[c]) <= 1e-10, NAMES[c]


@pytest.mark.parametrize("n,ncpml", [((16, 17, 16), 6), ((33, 17, 16), 6), ((37, 21, 19), 5)])
@pytest.mark.parametrize("flavor", [FLAVOR_NCVER0027, FLAVOR_SATAN_I])
def test_box_layout_edge_cases_match_oracle(n, ncpml, flavor):
    """The smallest grids the CPML allows (2 ncpml + 4 cells per axis): no
    interior box in x (every cell in the general body), an interior box of
    three or four rows and planes, and odd sizes: final fields and traces
    against the oracle (FP64, 1e-10)."""
    wl = W.small_case(n=n, ncpml=ncpml, nt=60, precision=FP64, flavor=flavor, magnetic=True, seed=3)
    tr, F = oracle_run(wl, want_fields=True)[0]
    with W.make_solver(wl) as s:
        _, td = s.forward(wl.nt, want_traces=True)
        G = s.fields(0)
    assert rel_l2(td[0], tr) <= 1e-10
    for c in range(6):
        assert rel_l2(G[c], F[c]) <= 1e-10, NAMES[c]


def test_sign_flipped_bp_updates_match_oracle():
    wl = W.small_case(nt=120, precision=FP64)
    cp = replace(wl.cp, e_sign=-1, h_sign=-1, check_cfl=True)
    wl2 = replace(wl, cp=cp)
    ref = oracle_run(wl2)
    with W.make_solver(wl2) as s:
        _, td = s.forward(wl.nt, want_traces=True)
    assert rel_l2(td[0], ref[0]) <= 1e-10


def test_batched_shots_equal_single_shots():
    wl = W.small_case(nt=150, precision=FP32)
    pts2 = [(wl.cp.nx // 3, wl.cp.ny // 3, wl.cp.nz // 2, "ey", SRC_ELECTRIC, 0.5)]
    wl2 = replace(wl, shots=[wl.shots[0], Shot(points=pts2), wl.shots[0]])
    with W.make_solver(wl2) as s:
        spec, td = s.forward(wl.nt, want_traces=True)
    for k, shot in enumerate(wl2.shots):
        with W.make_solver(replace(wl, shots=[shot])) as s1:
            sp1, td1 = s1.forward(wl.nt, want_traces=True)
        assert np.array_equal(td[k], td1[0])
        assert np.array_equal(spec[k], sp1[0])


@pytest.mark.parametrize("prec", [FP32, FP64])
def test_linearity_in_source_amplitude(prec):
    # Doubling is exact for normal numbers, but the stencil's precursors ahead
    # of the wavefront reach the denormal range, so compare in rel-L2.
    wl = W.small_case(nt=100, precision=prec)
    x, y, z, c, k, a = wl.shots[0].points[0]
    wl2 = replace(wl, shots=[Shot(points=[(x, y, z, c, k, 2.0 * a)])])
    with W.make_solver(wl) as s:
        sp1, t1 = s.forward(wl.nt, want_traces=True)
    with W.make_solver(wl2) as s:
        sp2, t2 = s.forward(wl.nt, want_traces=True)
    assert rel_l2(t2, 2.0 * t1) <= (1e-7 if prec == FP32 else 1e-15)
    assert rel_l2(sp2, 2.0 * sp1) <= (1e-7 if prec == FP32 else 1e-15)


def test_volume_dft_matches_oracle_dft_of_traces():
    wl = W.small_case(nt=200, precision=FP32)
    cells = [(5, 6, 7), (wl.cp.nx // 2, wl.cp.ny // 2, wl.cp.nz // 2 - 2), (wl.cp.nx - 3, 4, wl.cp.nz - 5)]
    rec = [(x, y, z, c) for (x, y, z) in cells for c in ("ex", "ey", "ez")]
    wl2 = replace(wl, receivers=rec, volume_dft="xyz")
    ref = oracle_run(wl2)[0]
    with W.make_solver(wl2) as s:
        s.forward(wl.nt)
        vols = {c: s.volume_dft(0, c) for c in ("ex", "ey", "ez")}
    got = np.stack([vols[c][:, z - 1, y - 1, x - 1] for (x, y, z, c) in rec])
    want = np.stack([O.dft(ref[r], wl.cp.dt, wl.cp.omega0, wl.omega) for r in range(len(rec))])
    assert rel_l2(got, want) <= 1e-4


def test_volume_dft_with_ring_remainder():
    # nt not a multiple of the 16-step ring exercises the partial flush
    wl = W.small_case(nt=37, precision=FP64)
    rec = [(wl.cp.nx // 2 + 1, wl.cp.ny // 2, wl.cp.nz // 2, "ex")]
    wl2 = replace(wl, receivers=rec, volume_dft="x")
    ref = oracle_run(wl2)[0]
    with W.make_solver(wl2) as s:
        s.forward(wl.nt)
        v = s.volume_dft(0, "ex")
    x, y, z, _ = rec[0]
    assert rel_l2(v[:, z - 1, y - 1, x - 1], O.dft(ref[0], wl.cp.dt, wl.cp.omega0, wl.omega)) <= 1e-10


def test_volume_dft_matches_receiver_spectra():
    """Nt = 533 runs four 128-step ring blocks, each folded into the
    accumulators before the ring is rewritten, and a remainder.  The volume
    spectra at 80 random cells (all three components) equal the spectra of
    receivers sampled there, an independent path (traces, then the trace
    DFT), to FP64 rounding, and the oracle at three of them."""
    wl = W.small_case(nt=533, precision=FP64)
    rng = np.random.default_rng(17)
    cells = [(int(rng.integers(1, wl.cp.nx + 1)), int(rng.integers(1, wl.cp.ny + 1)),
              int(rng.integers(1, wl.cp.nz + 1))) for _ in range(80)]
    rec = [(x, y, z, c) for (x, y, z) in cells for c in ("ex", "ey", "ez")]
    wl2 = replace(wl, receivers=rec, volume_dft="xyz")
    with W.make_solver(wl2) as s:
        spec, _ = s.forward(wl.nt, want_traces=True)
        vols = {c: s.volume_dft(0, c) for c in ("ex", "ey", "ez")}
    got = np.stack([vols[c][:, z - 1, y - 1, x - 1] for (x, y, z, c) in rec])
    assert np.abs(got).max() > 0
    assert rel_l2(got, spec[0]) <= 1e-12
    few = replace(wl2, receivers=rec[:9])
    ref = oracle_run(few)[0]
    want = np.stack([O.dft(ref[r], wl.cp.dt, wl.cp.omega0, wl.omega) for r in range(9)])
    assert rel_l2(got[:9], want) <= 1e-10


def test_standalone_f_to_d_matches_oracle():
    rng = np.random.default_rng(3)
    x = rng.normal(size=(5, 700))
    dt, w0 = 7.4e-4, 2 * 3.14159265358979
    om = np.arange(1, 50) * 2 * np.pi / (700 * dt)
    got = f_to_d(x, dt, w0, om)
    ref = np.stack([O.dft(x[r], dt, w0, om) for r in range(5)])
    assert rel_l2(got, ref) <= 1e-12
    goth = f_to_d(x, dt, w0, om, h_factor=True)
    refh = np.stack([O.dft(x[r], dt, w0, om, h_factor=True) for r in range(5)])
    assert rel_l2(goth, refh) <= 1e-12


def test_repeated_forward_is_deterministic():
    wl = W.small_case(nt=64, precision=FP32)
    with W.make_solver(wl) as s:
        a, ta = s.forward(wl.nt, want_traces=True)
        b, tb = s.forward(wl.nt, want_traces=True)
    assert np.array_equal(ta, tb) and np.array_equal(a, b)


def test_edge_source_and_receivers_at_grid_corners():
    wl = W.small_case(nt=80, precision=FP64)
    nx, ny, nz = wl.cp.nx, wl.cp.ny, wl.cp.nz
    rec = [(1, 1, 1, "ez"), (nx, ny, nz, "hx"), (nx, 1, nz // 2, "ey"), (2, ny - 1, 3, "hz")]
    wl2 = replace(wl, receivers=rec, shots=[Shot(points=[(3, 3, 3, "ez", SRC_ELECTRIC, 1.0)])])
    ref = oracle_run(wl2)[0]
    with W.make_solver(wl2) as s:
        _, td = s.forward(wl.nt, want_traces=True)
    assert rel_l2(td[0], ref) <= 1e-10


def test_single_step():
    wl = W.small_case(nt=1, precision=FP64)
    ref = oracle_run(wl)[0]
    with W.make_solver(wl) as s:
        _, td = s.forward(1, want_traces=True)
    assert np.allclose(td[0], ref, rtol=1e-12, atol=0)


@pytest.mark.parametrize("tma_cfg", [0, 4])
@pytest.mark.parametrize("prec", [FP32, FP64])
@pytest.mark.parametrize("flavor", [FLAVOR_NCVER0027, FLAVOR_SATAN_I])
def test_tma_interior_is_bit_identical_to_plain_loads(monkeypatch, prec, flavor, tma_cfg):
    """The TMA-staged interior kernel and the plain-load interior body use the
    same fma forms, so fields, traces and volume spectra agree bit for bit.
    The grid gives the interior partial tiles in x and y, several z chunks
    and two shots; both TMA layouts (own-cell tiles staged or loaded by the
    threads) are pinned in turn."""
    wl = W.small_case(n=(150, 44, 40), ncpml=8, nt=70, precision=prec, flavor=flavor, magnetic=True)
    nx, ny, nz = wl.cp.nx, wl.cp.ny, wl.cp.nz
    second = Shot(points=[(nx // 3, ny // 2 + 3, nz // 2 - 4, "ey", SRC_ELECTRIC, 0.7)])
    wl = replace(wl, volume_dft="xyz", shots=[wl.shots[0], second])
    out = {}
    monkeypatch.setenv("MITTET_TMA_CFG", str(tma_cfg))  # 0: own-cell tiles staged, 4: loaded by the threads
    for mode in ("ldg", "tma"):
        monkeypatch.setenv("MITTET_INTERIOR", mode)
        with W.make_solver(wl) as s:
            spec, td = s.forward(wl.nt, want_traces=True)
            var = s.tuned_variant()
            vols = [s.volume_dft(k, c) for k in (0, 1) for c in ("ex", "ey", "ez")]
            fields = [s.fields(k) for k in (0, 1)]
        out[mode] = (spec, td, vols, fields, var)
    assert out["tma"][4]["e_interior"][0] == 0 and out["tma"][4]["h_interior"][0] == 0, out["tma"][4]
    assert out["ldg"][4]["e_interior"][0] != 0 and out["ldg"][4]["h_interior"][0] != 0, out["ldg"][4]
    a, b = out["ldg"], out["tma"]
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    for va, vb in zip(a[2], b[2]):
        assert np.array_equal(va, vb)
    for fa, fb in zip(a[3], b[3]):
        for c in range(6):
            assert np.array_equal(fa[c], fb[c]), NAMES[c]


@pytest.mark.parametrize("prec,flavor", [(FP32, FLAVOR_NCVER0027), (FP32, FLAVOR_SATAN_I), (FP64, FLAVOR_NCVER0027)])
def test_every_stencil_variant_is_bit_identical(monkeypatch, prec, flavor):
    """Every variant the autotuner may choose (marching and single-plane
    bodies, each tile shape) gives the same fields, traces and volume spectra
    bit for bit: the bodies share their fma forms and only partition the
    cells differently.  The grid gives partial tiles in x and y, ragged z
    chunks, CPML slabs on every face and two shots."""
    from mittet_main_b200.solver import stencil_variants

    wl = W.small_case(n=(150, 44, 40), ncpml=8, nt=40, precision=prec, flavor=flavor, magnetic=True)
    nx, ny, nz = wl.cp.nx, wl.cp.ny, wl.cp.nz
    second = Shot(points=[(nx // 3, ny // 2 + 3, nz // 2 - 4, "ey", SRC_ELECTRIC, 0.7)])
    wl = replace(wl, volume_dft="xyz", shots=[wl.shots[0], second])
    vs = stencil_variants(prec == FP64)
    assert any(c[3] < 0 for c in vs) and any(c[3] > 0 for c in vs), vs
    monkeypatch.setenv("MITTET_INTERIOR", "ldg")
    base = None
    for v, cfg in enumerate(vs):
        monkeypatch.setenv("MITTET_VARIANT", str(v))
        with W.make_solver(wl) as s:
            spec, td = s.forward(wl.nt, want_traces=True)
            used = s.tuned_variant()
            vols = [s.volume_dft(k, c) for k in (0, 1) for c in ("ex", "ey", "ez")]
            fields = [s.fields(k) for k in (0, 1)]
        assert all(u == cfg for u in used.values()), (v, cfg, used)
        if base is None:
            base = (spec, td, vols, fields)
            continue
        assert np.array_equal(spec, base[0]) and np.array_equal(td, base[1]), (v, cfg)
        for va, vb in zip(vols, base[2]):
            assert np.array_equal(va, vb), (v, cfg)
        for fa, fb in zip(fields, base[3]):
            for c in range(6):
                assert np.array_equal(fa[c], fb[c]), (v, cfg, NAMES[c])


def test_residual_reinjection_matches_oracle(tmp_path):
    """read_source_3d_res: the magnetic sources driven by a time-reversed
    residual (difference of two runs), read back from a "t value" file."""
    from mittet_main_b200 import formats, rtm

    wl = W.small_case(nt=120, precision=FP64, magnetic=True)
    pert = wl.sigma.copy()
    pert[10:16, 12:20, 12:18] *= 4.0
    r = len(wl.receivers) // 2
    with W.make_solver(wl) as s:
        _, t0 = s.forward(wl.nt, want_traces=True)
    with W.make_solver(replace(wl, sigma=pert)) as s:
        _, t1 = s.forward(wl.nt, want_traces=True)
    res = rtm.reversed_residual(t1[0, r], t0[0, r])
    path = tmp_path / "residual_wave_abso_rev.d"
    np.savetxt(path, np.c_[np.arange(1, wl.nt + 1) * wl.cp.dt, res])
    _, sig = formats.read_signal(str(path))
    w = rtm.reinjection_wavelet(sig)
    wl2 = replace(wl, wavelet=w)
    ref = oracle_run(wl2)
    with W.make_solver(wl2) as s:
        _, td = s.forward(wl.nt, want_traces=True)
    assert np.abs(res).max() > 0
    assert rel_l2(td[0], ref[0]) <= 1e-10


def test_differential_probe_matches_oracle():
    """source_posi's two Hz coils and pattern-2 receivers; the probe
    differences of the GPU traces equal those of the oracle's."""
    from mittet_main_b200 import probe

    wl = W.small_case(nt=150, precision=FP64, magnetic=True)
    shot, rec = probe.source_posi(sp=14, y0=wl.cp.ny // 2, z_source=wl.cp.nz // 2, l_hori=6, l_sr=3)
    wl2 = replace(wl, shots=[shot], receivers=rec)
    ref = oracle_run(wl2)[0]
    with W.make_solver(wl2) as s:
        _, td = s.forward(wl.nt, want_traces=True)
    assert rel_l2(td[0], ref) <= 1e-10
    for got, want in zip(probe.diff_probe(td[0]), probe.diff_probe(ref)):
        assert rel_l2(got, want) <= 1e-9


@pytest.mark.parametrize("prec", [FP32, FP64])
def test_merged_boundary_launch_is_bit_identical(monkeypatch, prec):
    """The four boundary parts of a phase merged into one launch run the same
    bodies per tile, so every merged shape gives the fields, traces and
    volume spectra of the four separate launches bit for bit."""
    from mittet_main_b200.solver import stencil_variants
    wl = W.small_case(n=(70, 44, 40), ncpml=8, nt=70, precision=prec, magnetic=True)
    second = Shot(points=[(20, 30, 12, "ez", SRC_ELECTRIC, 0.7)])
    wl = replace(wl, volume_dft="xyz", shots=[wl.shots[0], second])
    shapes = {(2, 32, 4), (2, 16, 8), (2, 8, 16)}
    cands = [-1] + [v for v, c in enumerate(stencil_variants(prec == FP64)) if tuple(c[:3]) in shapes and 0 < c[3] < 1000]
    base = None
    for v in cands:
        monkeypatch.setenv("MITTET_BOUNDARY", str(v))
        with W.make_solver(wl) as s:
            spec, td = s.forward(wl.nt, want_traces=True)
            path = s.launch_path()
            vols = [s.volume_dft(k, c) for k in (0, 1) for c in ("ex", "ey", "ez")]
            fields = [s.fields(k) for k in (0, 1)]
        assert (path["e_boundary"] is None) == (v < 0), (v, path)
        if base is None:
            base = (spec, td, vols, fields)
            continue
        assert np.array_equal(spec, base[0]) and np.array_equal(td, base[1]), v
        for va, vb in zip(vols, base[2]):
            assert np.array_equal(va, vb), v
        for fa, fb in zip(fields, base[3]):
            assert np.array_equal(fa, fb), v


@pytest.mark.parametrize("prec", [FP32, FP64])
@pytest.mark.parametrize("n", [(150, 44, 40), (70, 44, 40)])
def test_band_launch_is_bit_identical(monkeypatch, prec, n):
    """The interior and x faces as one band launch run the same bodies per
    tile, so every band depth gives the fields, traces and volume spectra of
    the separate launches bit for bit.  150 cells: a line-aligned interior
    [32, 128) with a partial right-face tile; 70 cells: 4-aligned x edges.
    Depth 3 leaves a ragged last band."""
    monkeypatch.setenv("MITTET_PERSIST", "0")
    wl = W.small_case(n=n, ncpml=8, nt=70, precision=prec, magnetic=True)
    second = Shot(points=[(20, 30, 12, "ez", SRC_ELECTRIC, 0.7)])
    wl = replace(wl, volume_dft="xyz", shots=[wl.shots[0], second])
    base = None
    for zc in (0, 4, 8, 16, 3):
        monkeypatch.setenv("MITTET_BAND", str(zc))
        with W.make_solver(wl) as s:
            spec, td = s.forward(wl.nt, want_traces=True)
            path = s.launch_path()
            vols = [s.volume_dft(k, c) for k in (0, 1) for c in ("ex", "ey", "ez")]
            fields = [s.fields(k) for k in (0, 1)]
        assert path["e_band"] == zc and path["h_band"] == zc, (zc, path)
        if base is None:
            base = (spec, td, vols, fields)
            continue
        assert np.array_equal(spec, base[0]) and np.array_equal(td, base[1]), zc
        for va, vb in zip(vols, base[2]):
            assert np.array_equal(va, vb), zc
        for fa, fb in zip(fields, base[3]):
            assert np.array_equal(fa, fb), zc


@pytest.mark.parametrize("prec", [FP32, FP64])
def test_device_model_equals_host_model(prec):
    """mittet_set_model_device (float64 or float32 CUDA arrays, with mu and
    with electric and magnetic sources) forms the same model words and
    source gains as mittet_set_model given the same values: bit-identical
    spectra and traces.  A zero conductivity is rejected on the device."""
    import torch

    wl = W.small_case(n=(40, 36, 32), ncpml=6, nt=60, precision=prec, magnetic=True)
    wl = replace(wl, shots=[wl.shots[0], Shot(points=[(12, 20, 14, "ey", SRC_ELECTRIC, 0.8)])])
    rng = np.random.default_rng(4)
    mu = wl.cp.mu0 * (1.0 + 0.2 * rng.random(wl.sigma.shape))
    for dt in (torch.float64, torch.float32):
        # the host path gets the values the device path is given
        sig_h = torch.tensor(wl.sigma, dtype=dt).to(torch.float64).numpy()
        mu_h = torch.tensor(mu, dtype=dt).to(torch.float64).numpy()
        with W.make_solver(replace(wl, sigma=sig_h, mu=mu_h)) as s:
            ref_spec, ref_td = s.forward(wl.nt, want_traces=True)
            s.set_model_device(torch.tensor(sig_h, dtype=dt, device="cuda"), torch.tensor(mu_h, dtype=dt, device="cuda"))
            spec, td = s.forward(wl.nt, want_traces=True)
            assert np.array_equal(spec, ref_spec) and np.array_equal(td, ref_td), dt
            bad = torch.tensor(sig_h, dtype=dt, device="cuda")
            bad[3, 4, 5] = 0.0
            with pytest.raises(MittetError):
                s.set_model_device(bad)
            s.set_model_device(torch.tensor(sig_h, dtype=dt, device="cuda"), torch.tensor(mu_h, dtype=dt, device="cuda"))
            again, _ = s.forward(wl.nt)
            assert np.array_equal(again, ref_spec), dt


@pytest.mark.parametrize("prec", [FP32, FP64])
def test_layouts_are_bit_identical(monkeypatch, prec):
    """The whole grid as one box with the general body, and the interior and
    x faces as parts with the slab rows whole (the layouts the autotuner may
    pick besides the partitioned one) give the fields, traces and volume
    spectra of the partitioned layout bit for bit, and the gradient (whose
    adjoint keeps the partitioned boxes) too."""
    monkeypatch.setenv("MITTET_PERSIST", "0")
    wl = W.small_case(n=(70, 44, 40), ncpml=8, nt=70, precision=prec, magnetic=True)
    second = Shot(points=[(20, 30, 12, "ez", SRC_ELECTRIC, 0.7)])
    wl = replace(wl, volume_dft="xyz", shots=[wl.shots[0], second])
    rng = np.random.default_rng(3)
    obs = (rng.normal(size=(2, len(wl.receivers), len(wl.omega)))
           + 1j * rng.normal(size=(2, len(wl.receivers), len(wl.omega)))) * 1e-12
    out = {}
    for lay in ("0", "1", "2"):
        monkeypatch.setenv("MITTET_LAYOUT", lay)
        with W.make_solver(wl) as s:
            spec, td = s.forward(wl.nt, want_traces=True)
            path = s.launch_path()
            vols = [s.volume_dft(k, c) for k in (0, 1) for c in ("ex", "ey", "ez")]
            fields = [s.fields(k) for k in (0, 1)]
            grad = s.gradient(wl.nt, obs, checkpoint_every=25)
        assert path["e_layout"] == int(lay) and path["h_layout"] == int(lay), path
        out[lay] = (spec, td, vols, fields, grad)
    a = out["0"]
    for lay in ("1", "2"):
        b = out[lay]
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), lay
        for va, vb in zip(a[2], b[2]):
            assert np.array_equal(va, vb), lay
        for fa, fb in zip(a[3], b[3]):
            assert np.array_equal(fa, fb), lay
        assert a[4][0] == pytest.approx(b[4][0], rel=1e-13) and np.array_equal(a[4][1], b[4][1]), lay
