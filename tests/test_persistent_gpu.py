"""The persistent multi-shot launch (one cooperative launch per block of 128
steps, persistent.cuh) against the stepped graph of part kernels.

Both run the same cell bodies with the same fma forms, so traces, final
fields and full-volume spectra must be bit-identical, for a batch of shots
with electric and magnetic sources, in FP32 and FP64, with a remainder block
shorter than 128 steps.  A grid barrier that cannot complete (it waits for
one CTA more than the grid has) gives up after its time limit and the solve
reports MITTET_ERR_DEVICE_TIMEOUT; a new handle then solves normally.
"""
from dataclasses import replace

import numpy as np
import pytest

from mittet_main_b200 import workloads as W
from mittet_main_b200.capi import FP32, FP64, SRC_ELECTRIC, SRC_MAGNETIC, MittetError
from mittet_main_b200.solver import Shot

pytestmark = pytest.mark.gpu


def _batch(prec, nt=150):
    wl = W.small_case(n=(40, 36, 32), ncpml=7, nt=nt, precision=prec, magnetic=True, seed=11)
    shots = [wl.shots[0],
             Shot(points=[(14, 12, 15, "ex", SRC_ELECTRIC, 1.0)]),
             Shot(points=[(25, 20, 10, "ey", SRC_ELECTRIC, 0.5), (20, 20, 20, "hz", SRC_MAGNETIC, 1.0)]),
             Shot(points=[(30, 9, 22, "ez", SRC_ELECTRIC, 1.0)])]
    return replace(wl, shots=shots, volume_dft="xyz")


def _solve(wl, monkeypatch, persist):
    monkeypatch.setenv("MITTET_PERSIST", persist)
    with W.make_solver(wl) as s:
        spec, td = s.forward(wl.nt, want_traces=True)
        path = s.launch_path()
        fields = [s.fields(k) for k in range(len(wl.shots))]
        vol = [s.volume_dft(k, "ex") for k in range(len(wl.shots))]
    return spec, td, fields, vol, path


@pytest.mark.parametrize("prec", [FP32, FP64])
def test_persistent_launch_is_bit_identical_to_stepped(monkeypatch, prec):
    wl = _batch(prec)
    a = _solve(wl, monkeypatch, "1")
    b = _solve(wl, monkeypatch, "0")
    assert a[4]["persistent"] and not b[4]["persistent"]
    assert np.abs(b[1]).max() > 0
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(a[0], b[0])
    for k in range(len(wl.shots)):
        assert np.array_equal(a[2][k], b[2][k]), k
        assert np.array_equal(a[3][k], b[3][k]), k


def test_persistent_barrier_timeout_reports_and_recovers(monkeypatch):
    wl = _batch(FP32, nt=150)
    monkeypatch.setenv("MITTET_PERSIST", "1")
    monkeypatch.setenv("MITTET_PERSIST_STALL", "1")
    monkeypatch.setenv("MITTET_PERSIST_WAIT_MS", "20")
    with W.make_solver(wl) as s:
        with pytest.raises(MittetError) as ex:
            s.forward(wl.nt)
        assert ex.value.name == "MITTET_ERR_DEVICE_TIMEOUT"
    monkeypatch.delenv("MITTET_PERSIST_STALL")
    monkeypatch.delenv("MITTET_PERSIST_WAIT_MS")
    a = _solve(wl, monkeypatch, "1")
    b = _solve(wl, monkeypatch, "0")
    assert np.array_equal(a[1], b[1])
