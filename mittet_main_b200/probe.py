"""The differential-probe set-up and products of the ncver0027 driver.

source_posi (ncver0027/cpu_source_posi.f90:8-39) places two Hz point sources
(the probe's coils) a distance L_hori apart along x, and three Hz receivers
in "pattern 2": (1) above the left source by L_sr, (2) below it by L_sr,
(3) below the right source by L_sr.  output_EH_J (cpu_output.f90:53-55)
records Hz at the three receivers, and diff_probe (cpu_diff_probe.f90:1-58)
writes the differential signals (1)-(2) ("12diff", the absolute probe) and
(2)-(3) ("23diff", the differential probe).  The solve itself is the
ordinary forward path; this module only places the points and forms the
products.  Positions are 1-based like the reference's.
"""
from __future__ import annotations

import os

import numpy as np

from .capi import SRC_MAGNETIC
from .solver import Shot


def source_posi(sp: int, y0: int, z_source: int, l_hori: int, l_sr: int):
    """(shot, receivers) of source_posi for source position sp: the two
    magnetic Hz sources (amplitude 1 each, read_source_3d) and the three
    pattern-2 Hz receivers, in the order (1), (2), (3)."""
    x_source2 = sp + l_hori
    shot = Shot(points=[(sp, y0, z_source, "hz", SRC_MAGNETIC, 1.0),
                        (x_source2, y0, z_source, "hz", SRC_MAGNETIC, 1.0)])
    receivers = [(sp, y0, z_source + l_sr, "hz"),           # (1)
                 (sp, y0, z_source - l_sr, "hz"),           # (2)
                 (sp + l_hori, y0, z_source - l_sr, "hz")]  # (3)
    return shot, receivers


def diff_probe(traces: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """traces [3, nt] of receivers (1), (2), (3) -> (12diff, 23diff)."""
    tr = np.asarray(traces, dtype=np.float64)
    return tr[0] - tr[1], tr[1] - tr[2]


def write_diff_probe(dirname: str, prefix: str, dt: float, traces: np.ndarray) -> None:
    """<prefix>pattern2_12diff.d and <prefix>pattern2_23diff.d, one "t value"
    line per step, t = istep dt for istep = 1..nt (as output_EH_J's t)."""
    d12, d23 = diff_probe(traces)
    t = np.arange(1, d12.size + 1) * dt
    for name, d in (("pattern2_12diff.d", d12), ("pattern2_23diff.d", d23)):
        with open(os.path.join(dirname, prefix + name), "w") as f:
            for tv, v in zip(t, d):
                f.write(f"  {tv:.17g}  {v:.17g}\n")
