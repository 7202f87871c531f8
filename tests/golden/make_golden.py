"""Generate the golden fixtures of the satan_i path.

Runs the reference's own satan_i C functions, compiled from their sources by
oracle/Makefile into oracle/_ref/satan_ref, on small seeded cases and stores
inputs and outputs under tests/golden/:

  satan_e[xyz].npz   the forward time loop (traces, final fields)
  satan_ftod.npz     laplaceToFreq on the satan_ex traces (receiver f_to_d,
                     the sqrt(-2 w0/(i w)) current factor)
  satan_volume.npz   laplaceToFreq_2 on copytoEcal's history (full-volume
                     transform), at sampled cells
  satan_gamma.npz    residualE, sensitivity, conv_GdelE, calc_gamma on seeded
                     spectra (gamma_inputs)
  satan_update.npz   calc_phi, calc_alpha, update_para2 on seeded inputs
                     (update_inputs)
  ref_files/         text files the reference itself wrote in those runs
                     (spectrum, gradient and conductivity files)

Needs the reference tree (it is not read at test time):
``python tests/golden/make_golden.py``.
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


def _cnormal(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def gamma_inputs(seed=41):
    """Seeded spectra in satan_i's layouts for residualE .. calc_gamma."""
    rng = np.random.default_rng(seed)
    shape, ncpml, nf = (9, 8, 7), 2, 3
    n = shape[0] * shape[1] * shape[2]
    rec_pos = np.array([(3, 3, 3), (5, 4, 2), (7, 6, 5)], dtype=np.int32)
    obs = _cnormal(rng, (3, len(rec_pos), nf))
    e_ff = _cnormal(rng, (3, nf, n))
    e_bb = _cnormal(rng, (3, len(rec_pos), 3, nf, n))
    return dict(shape=shape, ncpml=ncpml, rec_pos=rec_pos, d=(50.0, 40.0, 30.0), obs=obs, e_ff=e_ff, e_bb=e_bb)


def update_inputs(seed=43):
    """Seeded model, gradient and receiver spectra for calc_phi .. update_para2."""
    rng = np.random.default_rng(seed)
    shape, ncpml, nf = (10, 8, 6), 1, 3
    ix, iy, iz = shape
    n = ix * iy * iz
    rec_pos = np.array([(3, 3, 2), (6, 4, 3), (8, 6, 4), (4, 7, 2)], dtype=np.int32)
    sig = 10.0 ** rng.normal(np.log10(0.3), 0.3, size=n)
    grad = rng.standard_normal(n) * 1e-3
    de = _cnormal(rng, (3, len(rec_pos), nf))
    e_ffl = _cnormal(rng, (3, nf, n))
    e_ff2 = e_ffl + 0.1 * _cnormal(rng, (3, nf, n))
    return dict(shape=shape, ncpml=ncpml, iseabed=3, rec_pos=rec_pos, d=(25.0, 25.0, 20.0), minval=0.05,
                maxval=2.0, sig=sig, grad=grad, de=de, e_ffl=e_ffl, e_ff2=e_ff2)


def _write_ref_files(texts):
    d = os.path.join(HERE, "ref_files")
    os.makedirs(d, exist_ok=True)
    for name, text in texts.items():
        with open(os.path.join(d, name), "w") as f:
            f.write(text)


def make_ftod():
    g = dict(np.load(os.path.join(HERE, "satan_ex.npz")))
    rec = g["receivers"]
    pos = [tuple(r[:3]) for r in rec if r[3] == 0]
    tr = g["traces"]
    traces = np.stack([np.stack([tr[[q for q, r in enumerate(rec) if tuple(r[:3]) == p and r[3] == c][0]]
                                 for c in range(3)]) for p in pos])  # [npos, 3, nt]
    # strongest receiver first: the reference's files are written for receiver 000
    order = np.argsort(-np.abs(traces).max(axis=(1, 2)), kind="stable")
    traces = traces[order]
    pos = [pos[q] for q in order]
    it = traces.shape[2]
    upper_f = 8
    jx = g["wavelet"][:it]
    files = ["spectrum_e_000_000.dat", "spectrum_j_000_000.dat", "spectrum_ex_000_000.dat"]
    spec, texts = O.run_satan_ftod(traces, jx, float(g["dt"]), float(g["omega0"]), upper_f, files)
    np.savez_compressed(os.path.join(HERE, "satan_ftod.npz"), positions=np.array(pos), upper_f=upper_f, spec=spec)
    _write_ref_files(texts)
    print("satan_ftod", spec.shape)


def make_volume():
    ix, iy, iz, nc, nt, nvol = 18, 16, 14, 5, 150, 5
    rng = np.random.default_rng(17)
    sig = 10.0 ** rng.normal(np.log10(0.3), 0.3, size=(iz, iy, ix))
    d, om0 = 50.0, 2.0 * np.pi
    cmin = np.sqrt(2 * om0 / O.MU0_C / sig.max())
    fmax = 0.9 * cmin / (10.4 * d)
    p = O.satan_params(ix, iy, iz, d, d, d, nc, om0, sig.min())
    t = np.arange(nt + 1) * p.dt
    t0, beta = np.pi / fmax, np.pi * fmax ** 2
    w = -2.0 * beta * (t - t0) * np.sqrt(beta / np.pi) * np.exp(-beta * (t - t0) ** 2)
    src = (9, 8, 7)
    dt, cmax, tr, F, vol = O.run_satan_reference(ix, iy, iz, d, d, d, nc, om0, sig, w, nt, src, 0, [], nvol=nvol)
    cells = np.sort(rng.choice(ix * iy * iz, size=256, replace=False))
    vs = vol.reshape(3, nvol - 1, -1)[:, :, cells]
    np.savez_compressed(os.path.join(HERE, "satan_volume.npz"), shape=np.array([ix, iy, iz]), ncpml=nc, nt=nt, d=d,
                        omega0=om0, sigma=sig, wavelet=w, src=np.array(src), src_comp=0, dt=dt, cmax=cmax,
                        nvol=nvol, cells=cells, vol=vs)
    print("satan_volume", vs.shape, np.abs(vs).max())


def make_gamma():
    a = gamma_inputs()
    out, _ = O.run_satan_gamma(a["shape"], a["ncpml"], a["rec_pos"], a["d"], a["obs"], a["e_ff"], a["e_bb"])
    np.savez_compressed(os.path.join(HERE, "satan_gamma.npz"), seed=41, **out)
    print("satan_gamma err_sum", out["err_sum"])


def make_update():
    a = update_inputs()
    files = ["gradient_000.dat", "sig_000.dat"]
    out, texts = O.run_satan_update(a["shape"], a["ncpml"], a["iseabed"], a["rec_pos"], a["d"], a["minval"],
                                    a["maxval"], a["sig"], a["grad"], a["de"], a["e_ffl"], a["e_ff2"], files)
    np.savez_compressed(os.path.join(HERE, "satan_update.npz"), seed=43, scaler=out["scaler"], k1=out["k1"],
                        k2=out["k2"], alpha=out["alpha"], sig2=out["sig2"], sig=out["sig"])
    _write_ref_files(texts)
    print("satan_update alpha", out["alpha"], "scaler", out["scaler"])


def main():
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    if "--post" not in sys.argv:
        make_forward()
    make_ftod()
    make_volume()
    make_gamma()
    make_update()


def make_forward():
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
