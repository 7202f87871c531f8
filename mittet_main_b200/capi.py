"""ctypes binding of the C ABI in ``include/mittet.h`` (libmittet_b200.so).

The library is built in-tree by ``mittet_main_b200/build.py``.  There is no
CPU fallback: if the library cannot be loaded, or no CUDA device is present,
every call raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmittet_b200.so")

MITTET_OK = 0
ERRORS = {
    -1: "MITTET_ERR_INVALID_ARG",
    -2: "MITTET_ERR_CFL",
    -3: "MITTET_ERR_OOM",
    -4: "MITTET_ERR_DIVERGED",
    -5: "MITTET_ERR_DEVICE_TIMEOUT",
    -6: "MITTET_ERR_CUDA",
    -7: "MITTET_ERR_STATE",
}
FLAVOR_NCVER0027 = 0
FLAVOR_SATAN_I = 1
FP32 = 0
FP64 = 1
EX, EY, EZ, HX, HY, HZ = range(6)
COMP = {"ex": EX, "ey": EY, "ez": EZ, "hx": HX, "hy": HY, "hz": HZ}
SRC_MAGNETIC = 0
SRC_ELECTRIC = 1


class MittetError(RuntimeError):
    """A C-ABI call returned a negative status."""

    def __init__(self, code: int, message: str):
        self.code = code
        self.name = ERRORS.get(code, f"status {code}")
        super().__init__(f"{self.name}: {message}")


class CflError(MittetError):
    pass


class DivergedError(MittetError):
    pass


class Grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
                ("ncpml", ctypes.c_int32)]


class Phys(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("omega0", ctypes.c_double), ("cmax", ctypes.c_double),
                ("mu0", ctypes.c_double), ("c1", ctypes.c_double), ("c2", ctypes.c_double),
                ("flavor", ctypes.c_int32), ("psi_hyx_typo", ctypes.c_int32),
                ("e_sign", ctypes.c_int32), ("h_sign", ctypes.c_int32),
                ("cpml_nn", ctypes.c_double), ("cpml_order", ctypes.c_double),
                ("cpml_kappa_max", ctypes.c_double), ("cpml_a_max", ctypes.c_double),
                ("cpml_ma", ctypes.c_double), ("cpml_rcoef", ctypes.c_double),
                ("cpml_opt_to_max_x", ctypes.c_double),
                ("precision", ctypes.c_int32), ("device", ctypes.c_int32), ("check_cfl", ctypes.c_int32)]


class PointSource(ctypes.Structure):
    _fields_ = [("shot", ctypes.c_int32), ("ix", ctypes.c_int32), ("iy", ctypes.c_int32),
                ("iz", ctypes.c_int32), ("comp", ctypes.c_int32), ("kind", ctypes.c_int32),
                ("amp", ctypes.c_double)]


class Receiver(ctypes.Structure):
    _fields_ = [("ix", ctypes.c_int32), ("iy", ctypes.c_int32), ("iz", ctypes.c_int32), ("comp", ctypes.c_int32)]


# Every function the header declares, with its ctypes signature.
_P = ctypes.POINTER
_VP = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int32
SIGNATURES = {
    "mittet_phys_defaults": (ctypes.c_int, [_I, _P(Phys)]),
    "mittet_reference_dt": (_D, [_I, _P(Grid), _D]),
    "mittet_freq_grid_ref": (ctypes.c_int, [_I, _D, _I, _P(_D)]),
    "mittet_create": (ctypes.c_int, [_P(Grid), _P(Phys), _P(_VP)]),
    "mittet_destroy": (None, [_VP]),
    "mittet_set_model": (ctypes.c_int, [_VP, _P(_D), _P(_D)]),
    "mittet_set_sources": (ctypes.c_int, [_VP, _I, _I, _P(PointSource)]),
    "mittet_set_wavelet": (ctypes.c_int, [_VP, _I, _P(_D)]),
    "mittet_set_receivers": (ctypes.c_int, [_VP, _I, _P(Receiver)]),
    "mittet_set_freqs": (ctypes.c_int, [_VP, _I, _P(_D), _I]),
    "mittet_set_volume_dft": (ctypes.c_int, [_VP, ctypes.c_uint32]),
    "mittet_forward": (ctypes.c_int, [_VP, _I, _P(_D), _P(_D)]),
    "mittet_get_volume_dft": (ctypes.c_int, [_VP, _I, _I, _P(_D)]),
    "mittet_get_fields": (ctypes.c_int, [_VP, _I, _P(_D)]),
    "mittet_f_to_d": (ctypes.c_int, [_I, _I, _I, _D, _D, _P(_D), _I, _P(_D), _I, _P(_D)]),
    "mittet_gradient": (ctypes.c_int, [_VP, _I, _P(_D), _I, _P(_D), _P(_D)]),
    "mittet_release_gradient_buffers": (ctypes.c_int, [_VP]),
    "mittet_fwi_update": (ctypes.c_int, [_VP, _I, _P(_D), _P(_D), _P(_D), _I, _D, _D, _P(_D), _P(_D)]),
    "mittet_satan_gamma": (ctypes.c_int, [_I, _P(Grid), _I, _P(_I), _I, _P(_D), _P(_D), _P(_D), _I, _P(_D),
                                          _P(_D), _P(_D), _P(_D), _P(_D)]),
    "mittet_set_model_device": (ctypes.c_int, [_VP, _VP, _VP, _I]),
    "mittet_forward_device": (ctypes.c_int, [_VP, _I, _VP, _VP]),
    "mittet_time_kernels": (ctypes.c_int, [_VP, _I, _P(_D)]),
    "mittet_tuned_variant": (ctypes.c_int, [_VP, _P(_I), _P(_I)]),
    "mittet_tuned_variants": (ctypes.c_int, [_VP, _P(_I)]),
    "mittet_stencil_variants": (ctypes.c_int, [_I, _P(_I), _P(_I), _I]),
    "mittet_last_launch_count": (ctypes.c_int64, [_VP]),
    "mittet_persistent_variant": (ctypes.c_int, [_VP, _P(_I), _P(_I)]),
    "mittet_boundary_variant": (ctypes.c_int, [_VP, _P(_I), _P(_I)]),
    "mittet_band_variant": (ctypes.c_int, [_VP, _P(_I), _P(_I)]),
    "mittet_layout_variant": (ctypes.c_int, [_VP, _P(_I), _P(_I)]),
    "mittet_forward_noalloc": (ctypes.c_int, [_P(Grid), _P(Phys), _VP, _I, _P(PointSource), _I, _VP, _I,
                                               _P(Receiver), _I, _P(_D), _I, _VP, _VP]),
    "mittet_last_error": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t]),
}

_lib = None
_lock = threading.Lock()


def load(build_if_missing: bool = True):
    """Load the in-tree library, building it first only if it does not exist
    (rebuilds are explicit: ``python mittet_main_b200/build.py``)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if build_if_missing and not os.path.exists(LIB_PATH):
            from . import build as _build
            _build.build(force=True)
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    load().mittet_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc == MITTET_OK:
        return
    msg = last_error()
    if rc == -2:
        raise CflError(rc, msg)
    if rc == -4:
        raise DivergedError(rc, msg)
    raise MittetError(rc, msg)
