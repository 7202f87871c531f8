"""The reference's text formats: round trips and a synthetic satan_i data
directory turned into a workload (CPU only)."""
import os

import numpy as np

from mittet_main_b200 import formats as F


def test_model_env_round_trip(tmp_path):
    e = F.ModelEnv(ix=31, iy=31, iz=31, dx=50.0, dy=50.0, dz=50.0, dt_ratio=1.0, it=1302, mstep=100, trstep=10,
                   omega_0=6.283185307179586, fmax_w=5.0, glim=10.4, ncpml=6, unused=[1.0, 2.0, 3.0, 4.0, 5.0],
                   start_f=1, upper_f=20, shots=[(16, 16, 8), (10, 16, 8)], receivers=[(20, 16, 8), (22, 16, 8)])
    p = tmp_path / "model_env.dat"
    F.write_model_env(str(p), e)
    assert F.read_model_env(str(p)) == e


def test_model_env_parses_whitespace_like_fscanf(tmp_path):
    text = "8 9 10\n25.0 25.0 20.0 1.0\n500 10 5 6.2831853 4.0 10.4 3\n0 0 0 0 0\n1 6 1\n4  5  6\n2\n3 3 3\n5 5 5\n"
    p = tmp_path / "model_env.dat"
    p.write_text(text)
    e = F.read_model_env(str(p))
    assert (e.ix, e.iy, e.iz, e.dz, e.it, e.ncpml, e.start_f, e.upper_f) == (8, 9, 10, 20.0, 500, 3, 1, 6)
    assert e.shots == [(4, 5, 6)] and e.receivers == [(3, 3, 3), (5, 5, 5)]


def test_conductivity_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    sig = np.round(rng.uniform(0.01, 4.0, size=(4, 5, 6)), 6)
    p = tmp_path / "conductivity.dat"
    F.write_conductivity(str(p), sig, 50.0, 50.0, 25.0)
    first = p.read_text().splitlines()[1].split()
    assert [float(v) for v in first[:3]] == [50.0, 0.0, 0.0]  # x fastest, k outermost
    assert np.array_equal(F.read_conductivity(str(p), 6, 5, 4), sig)


def test_spectra_and_volumes_round_trip(tmp_path):
    rng = np.random.default_rng(2)
    spec = rng.normal(size=(2, 4, 3)) + 1j * rng.normal(size=(2, 4, 3))
    recs = [(3, 3, 3, "ex"), (3, 3, 3, "ey"), (3, 3, 3, "ez"), (5, 5, 5, "ex")]
    F.write_observed(str(tmp_path), spec, recs, np.array([0.25, 0.5, 1.0]))
    assert sorted(os.listdir(tmp_path))[:3] == ["spectrum_ex_000_000.dat", "spectrum_ex_000_001.dat",
                                                "spectrum_ex_001_000.dat"]
    back = F.read_spectrum(str(tmp_path / "spectrum_ey_001_000.dat"), 3)
    assert np.allclose(back, spec[1, 1], rtol=1e-6)
    vol = rng.normal(size=(3, 4, 5)) * 1e-12
    F.write_volume(str(tmp_path / "gradient_001.dat"), vol, 50.0, 50.0, 50.0)
    line = (tmp_path / "gradient_001.dat").read_text().splitlines()[0]
    assert line.startswith("      0.00          0.00          0.00    ")
    assert np.allclose(F.read_volume(str(tmp_path / "gradient_001.dat"), 5, 4, 3), vol, rtol=1e-6)


def test_f_to_d_files(tmp_path):
    ex = np.array([1 + 2j, 3 - 1j])
    jz = np.array([2 + 0j, 1 + 1j])
    F.write_f_to_d(str(tmp_path), "1010", np.array([0.0, 0.5]), ex, jz)
    f, g = F.read_f_to_d(str(tmp_path / "GXe_w1010.d"))
    assert np.array_equal(f, [0.0, 0.5]) and np.allclose(g, ex / jz, rtol=1e-15)
    assert (tmp_path / "absEX_w1010.d").exists()


def test_workload_from_satan_data_directory(tmp_path):
    e = F.ModelEnv(ix=20, iy=18, iz=16, dx=50.0, dy=50.0, dz=50.0, dt_ratio=1.0, it=200, mstep=10, trstep=1,
                   omega_0=2 * np.pi, fmax_w=4.0, glim=10.4, ncpml=4, start_f=1, upper_f=4,
                   shots=[(10, 9, 5)], receivers=[(12, 9, 5), (14, 9, 5)])
    F.write_model_env(str(tmp_path / "model_env.dat"), e)
    (tmp_path / "minmax.dat").write_text("0.01 4.0\n")
    sig = np.full((16, 18, 20), 0.5)
    F.write_conductivity(str(tmp_path / "conductivity.dat"), sig, 50.0, 50.0, 50.0)
    t = np.arange(200) * 1e-3
    F.write_waveform(str(tmp_path / "waveformX.dat"), 1e-3, np.sin(t))
    wl = F.workload_from_satan(str(tmp_path))
    assert (wl.cp.nx, wl.cp.ny, wl.cp.nz, wl.cp.ncpml, wl.nt) == (20, 18, 16, 4, 199)
    assert len(wl.shots) == 1 and len(wl.receivers) == 6 and wl.omega.size == 3
    cmax = np.sqrt(2.0 * 2 * np.pi / 12.5663706e-7 / 0.01)
    courant = 1.0 / cmax / np.sqrt(3.0 / 50.0 ** 2)
    assert wl.cp.dt == courant * float(np.float32(6.0 / 7.0)) * float(np.float32(0.999)) or \
        abs(wl.cp.dt / (courant * 6.0 / 7.0 * 0.999) - 1) < 1e-6


def test_time_domain_output_is_fftw_backward_scaled():
    """to_time_domain = FFTW BACKWARD (e^{+2 pi i k n / nd}, unnormalised)
    x 2/(nd dt), cpu_f_to_d_e.f90:281-305, checked against the direct sum."""
    from mittet_main_b200.solver import to_time_domain

    rng = np.random.default_rng(3)
    nd, dt = 37, 7.4e-4
    X = rng.normal(size=nd) + 1j * rng.normal(size=nd)
    n = np.arange(nd)
    direct = np.array([np.sum(X * np.exp(2j * np.pi * n * q / nd)) for q in range(nd)]) * 2.0 / (nd * dt)
    assert np.allclose(to_time_domain(X, dt), direct, rtol=1e-12, atol=0)


def test_time_domain_files(tmp_path):
    z = np.array([1 + 1j, 2 - 3j, 0.5j])
    F.write_f_to_d_time(str(tmp_path), "1010", 1e-3, z, 2 * z, 3 * z)
    a = np.loadtxt(tmp_path / "GXe_t1010.d")
    assert np.allclose(a[:, 0], [0.0, 1e-3, 2e-3]) and np.allclose(a[:, 1] + 1j * a[:, 2], 3 * z)
    assert np.allclose(np.loadtxt(tmp_path / "absJZ_t1010.d")[:, 1], np.abs(2 * z))


def test_probe_positions_and_differences(tmp_path):
    """source_posi's pattern-2 geometry and diff_probe's two differences."""
    from mittet_main_b200 import probe

    shot, rec = probe.source_posi(sp=31, y0=20, z_source=15, l_hori=6, l_sr=3)
    assert [p[:4] for p in shot.points] == [(31, 20, 15, "hz"), (37, 20, 15, "hz")]
    assert rec == [(31, 20, 18, "hz"), (31, 20, 12, "hz"), (37, 20, 12, "hz")]
    tr = np.array([[1.0, 2.0, 3.0], [0.5, 1.0, 4.0], [0.25, 3.0, 1.0]])
    d12, d23 = probe.diff_probe(tr)
    assert np.array_equal(d12, [0.5, 1.0, -1.0]) and np.array_equal(d23, [0.25, -2.0, 3.0])
    probe.write_diff_probe(str(tmp_path), "31", 1e-3, tr)
    a = np.loadtxt(tmp_path / "31pattern2_23diff.d")
    assert np.allclose(a[:, 0], [1e-3, 2e-3, 3e-3]) and np.array_equal(a[:, 1], d23)
