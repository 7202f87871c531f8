"""CPU tests of the C ABI: the library loads, exports every declared symbol,
and validates arguments before touching a device.  No GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from mittet_main_b200 import capi
from mittet_main_b200.solver import ConstPara, cmax_of, dt_rule, firstderiv_gauss

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "mittet.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mittet_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = capi.load()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    # and the ctypes table covers them all
    assert set(names) <= set(capi.SIGNATURES)


def test_phys_defaults_restate_reference_constants():
    lib = capi.load()
    p = capi.Phys()
    assert lib.mittet_phys_defaults(capi.FLAVOR_NCVER0027, ctypes.byref(p)) == 0
    assert p.c1 == 1.125 and p.c2 == -0.04167 and p.mu0 == 1.2566370614e-6 and p.psi_hyx_typo == 1
    assert p.omega0 == 2.0 * 3.14159265358979
    assert lib.mittet_phys_defaults(capi.FLAVOR_SATAN_I, ctypes.byref(p)) == 0
    assert p.c2 == float(np.float32(-0.04167)) and p.mu0 == 12.5663706e-7 and p.cpml_opt_to_max_x == 10.0
    assert lib.mittet_phys_defaults(7, ctypes.byref(p)) == -1


def test_reference_dt_rules():
    lib = capi.load()
    g = capi.Grid(101, 101, 101, 4.5e-3, 4.5e-3, 4.5e-3, 10)
    cmax = 1234.5
    assert lib.mittet_reference_dt(0, ctypes.byref(g), cmax) == pytest.approx(0.999 * 4.5e-3 / cmax / np.sqrt(3) / 1.16667, rel=1e-15)
    courant = 1.0 / cmax / np.sqrt(3.0 / 4.5e-3 ** 2)
    assert lib.mittet_reference_dt(1, ctypes.byref(g), cmax) == pytest.approx(courant * 6 / 7 * float(np.float32(0.999)), rel=1e-15)


def test_freq_grid_ref():
    lib = capi.load()
    om = np.zeros(5)
    assert lib.mittet_freq_grid_ref(100, 1e-3, 5, om.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0
    assert np.allclose(om, np.arange(5) * 2 * 3.14159265358979 / 100 / 1e-3, rtol=1e-15)


def test_create_rejects_bad_arguments_before_the_device():
    lib = capi.load()
    h = ctypes.c_void_p()
    p = capi.Phys()
    lib.mittet_phys_defaults(0, ctypes.byref(p))
    p.dt, p.cmax = 1e-4, 1000.0
    bad = capi.Grid(4, 40, 40, 50., 50., 50., 10)
    assert lib.mittet_create(ctypes.byref(bad), ctypes.byref(p), ctypes.byref(h)) == -1
    assert "at least 8" in capi.last_error()
    g = capi.Grid(40, 40, 40, 50., 50., 50., 25)
    assert lib.mittet_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(h)) == -1
    # CFL: dt above the (2,4) Taylor limit (cpu_set_condition.f90:279-286)
    g = capi.Grid(40, 40, 40, 50., 50., 50., 8)
    p.dt = 1.01 * 50.0 / 1000.0 / np.sqrt(3) / 1.16667
    assert lib.mittet_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(h)) == -2


def test_forward_on_null_handle_is_an_error():
    lib = capi.load()
    assert lib.mittet_forward(None, 10, None, None) == -1
    assert lib.mittet_set_model(None, None, None) == -1


def test_no_cpu_fallback_without_a_device():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    cp = ConstPara(nx=24, ny=24, nz=24, dx=50., dy=50., dz=50., ncpml=6, dt=dt_rule(50., 31623.), cmax=31623.)
    from mittet_main_b200.solver import MittetSolver
    with pytest.raises(capi.MittetError) as e:
        MittetSolver(cp)
    assert e.value.code == -6


def test_wavelet_is_reference_gaussian_derivative():
    dt, fmax = 1e-3, 5.0
    w = firstderiv_gauss(100, dt, fmax)
    pi = 3.14159265358979
    beta, t0 = pi * fmax ** 2, pi / fmax
    t = 37 * dt
    assert w[37] == pytest.approx(-(2 * beta * (t - t0) * np.sqrt(beta / pi)) * np.exp(-beta * (t - t0) ** 2), rel=1e-14)
