"""Failure detection on the GPU, driven from the host without any GPU fault.

* MITTET_ERR_DIVERGED: a time step three times the (2,4) CFL limit, with the
  host-side CFL check switched off, makes the scheme unstable; the receiver
  traces overflow to Inf/NaN within a few hundred steps and the non-finite
  check of the traces reports it (the reference only prints or exits on its
  stability checks, satan_i/fwi3d_cpu_function_v1.4.c:1374-1405).
* MITTET_ERR_DEVICE_TIMEOUT: the TMA-staged interior waits on mbarriers for
  its tile copies.  MITTET_TMA_SPIN_LIMIT shortens every such wait to a few
  non-blocking polls, so the waits give up before the copies land; each CTA
  then drains its copies in flight with the normal (bounded) drain limit and
  returns, and the host reports the timeout.  A new handle without the limit
  then solves normally and matches the FP64 oracle.
"""
from dataclasses import replace

import numpy as np
import pytest

from mittet_main_b200 import workloads as W
from mittet_main_b200.capi import FP32, FP64, MittetError
from mittet_main_b200.solver import firstderiv_gauss
from tests.conftest import rel_l2
from tests.test_parity_gpu import oracle_run

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [FP32, FP64])
def test_unstable_time_step_reports_diverged(prec):
    wl = W.small_case(nt=600, precision=prec)
    cp = replace(wl.cp, dt=wl.cp.dt / 0.95 * 3.0, check_cfl=False)
    wl = replace(wl, cp=cp, wavelet=firstderiv_gauss(wl.nt + 1, cp.dt, wl.fmax))
    with W.make_solver(wl) as s:
        with pytest.raises(MittetError) as ex:
            s.forward(wl.nt)
    assert ex.value.name == "MITTET_ERR_DIVERGED"


def test_cfl_check_rejects_the_same_step():
    wl = W.small_case(nt=20)
    cp = replace(wl.cp, dt=wl.cp.dt / 0.95 * 3.0)
    with pytest.raises(MittetError) as ex:
        W.make_solver(replace(wl, cp=cp))
    assert ex.value.name == "MITTET_ERR_CFL"


def test_tma_wait_limit_reports_timeout_then_recovers(monkeypatch):
    # a grid of its own, so no autotune choice cached for another test is reused
    wl = W.small_case(n=(44, 40, 36), ncpml=6, nt=64, precision=FP32)
    monkeypatch.setenv("MITTET_INTERIOR", "tma")
    monkeypatch.setenv("MITTET_TMA_SPIN_LIMIT", "2")
    with W.make_solver(wl) as s:
        with pytest.raises(MittetError) as ex:
            s.forward(wl.nt)
        assert ex.value.name == "MITTET_ERR_DEVICE_TIMEOUT"
        assert s.tuned_variant()["e_interior"][0] == 0  # the TMA interior ran
    monkeypatch.delenv("MITTET_TMA_SPIN_LIMIT")
    with W.make_solver(wl) as s:
        _, td = s.forward(wl.nt, want_traces=True)
        assert s.tuned_variant()["e_interior"][0] == 0
    ref = oracle_run(wl)[0]
    assert rel_l2(td[0], ref) <= 1e-4
