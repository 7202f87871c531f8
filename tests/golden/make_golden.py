"""Generate the golden fixtures of the satan_i forward path.

Runs the reference's own satan_i C kernels, compiled from their sources by
oracle/Makefile into oracle/_ref/satan_ref, on small seeded cases and stores
inputs and outputs under tests/golden/.  Needs the reference tree (it is not
read at test time): ``python tests/golden/make_golden.py``.
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

CASES = [
    # name, (ix, iy, iz), ncpml, nt, source comp, source (1-based), seed, with_fields
    ("satan_ex", (26, 24, 22), 8, 160, 0, (13, 12, 11), 11, True),
    ("satan_ey", (24, 26, 20), 7, 120, 1, (9, 14, 10), 12, False),
    ("satan_ez", (22, 22, 24), 6, 120, 2, (11, 11, 13), 13, False),
]


def receivers_for(ix, iy, iz, nc):
    pts = [(2, 2, 2), (ix // 2, iy // 2, iz // 2 + 2), (ix - 1, iy // 2, iz // 2), (ix // 3, iy - 2, 3),
           (nc, nc + 1, iz - nc), (ix - 2, iy - 2, iz - 2), (nc + 2, iy // 2, 2), (ix // 2, 3, iz - 3)]
    return [(x, y, z, c) for (x, y, z) in pts for c in range(6)]


def main():
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    for name, (ix, iy, iz), nc, nt, scomp, src, seed, with_fields in CASES:
        rng = np.random.default_rng(seed)
        sig = 10.0 ** rng.normal(np.log10(0.3), 0.3, size=(iz, iy, ix))
        d = 50.0
        om0 = 2.0 * np.pi
        cmin = np.sqrt(2 * om0 / O.MU0_C / sig.max())
        fmax = 0.9 * cmin / (10.4 * d)
        p = O.satan_params(ix, iy, iz, d, d, d, nc, om0, sig.min())
        t = np.arange(nt + 1) * p.dt
        t0, beta = np.pi / fmax, np.pi * fmax ** 2
        # satan_i/fwi3d_cpu_waveform_v1.4.c:132-142, sampled at i dt from i = 0
        w = -2.0 * beta * (t - t0) * np.sqrt(beta / np.pi) * np.exp(-beta * (t - t0) ** 2)
        rec = receivers_for(ix, iy, iz, nc)
        dt, cmax, tr, F = O.run_satan_reference(ix, iy, iz, d, d, d, nc, om0, sig, w, nt, src, scomp, rec)
        out = dict(shape=np.array([ix, iy, iz]), ncpml=nc, nt=nt, d=d, omega0=om0, sigma=sig, wavelet=w,
                   src=np.array(src), src_comp=scomp, receivers=np.array(rec), dt=dt, cmax=cmax, traces=tr)
        if with_fields:
            out["fields"] = F
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, "max|trace|", np.abs(tr).max())


if __name__ == "__main__":
    main()
