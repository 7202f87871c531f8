"""B200-native Mittet fictitious-wave FDTD forward solve and FWI gradient.

The numerical path is ``libmittet_b200.so`` (hand-written sm_100a CUDA behind
the C ABI in ``include/mittet.h``); this package is its host-side front end.
"""
from .capi import (COMP, EX, EY, EZ, FLAVOR_NCVER0027, FLAVOR_SATAN_I, FP32, FP64, HX, HY, HZ,
                   SRC_ELECTRIC, SRC_MAGNETIC, CflError, DivergedError, MittetError)
from .solver import (ConstPara, MittetSolver, Shot, cmax_of, dt_rule, f_to_d, f_to_d_e, f_to_d_h,
                     firstderiv_gauss, freq_grid_ref)

__all__ = [
    "COMP", "EX", "EY", "EZ", "HX", "HY", "HZ", "FLAVOR_NCVER0027", "FLAVOR_SATAN_I", "FP32", "FP64",
    "SRC_ELECTRIC", "SRC_MAGNETIC", "CflError", "DivergedError", "MittetError", "ConstPara", "MittetSolver",
    "Shot", "cmax_of", "dt_rule", "f_to_d", "f_to_d_e", "f_to_d_h", "firstderiv_gauss", "freq_grid_ref",
]
