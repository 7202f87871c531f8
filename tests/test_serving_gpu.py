"""GPU: requests of different grids, shot counts and modes served together
give the same results as each request solved alone."""
import numpy as np
import pytest

from mittet_main_b200 import workloads as W
from mittet_main_b200.capi import FP32
from mittet_main_b200.serving import MittetServer, Request, run_request

pytestmark = pytest.mark.gpu


def requests():
    out = []
    specs = [((32, 30, 28), 80, 1), ((40, 36, 32), 120, 2), ((32, 30, 28), 60, 1), ((36, 36, 36), 100, 3),
             ((40, 36, 32), 90, 1), ((32, 30, 28), 70, 2)]
    for i, (n, nt, ns) in enumerate(specs):
        wl = W.small_case(n=n, ncpml=6, nt=nt, precision=FP32, seed=20 + i)
        from dataclasses import replace
        from mittet_main_b200.solver import Shot
        shots = [Shot(points=[(n[0] // 2 - s, n[1] // 2 + s, n[2] // 2, "ex", 1, 1.0)]) for s in range(ns)]
        wl = replace(wl, shots=shots)
        mode = "gradient" if i % 3 == 2 else "forward"
        obs = np.zeros((ns, len(wl.receivers), len(wl.omega)), dtype=complex) if mode == "gradient" else None
        out.append(Request(i, 0.01 * i, wl, mode, obs, checkpoint_every=25))
    return out


def test_results_alone_equal_results_in_the_mix():
    reqs = requests()
    alone = {r.rid: run_request({}, r) for r in reqs}
    srv = MittetServer(n_slots=3, hbm_budget=40e9)
    res = srv.run(reqs)
    assert srv.max_concurrent >= 2
    for r in res:
        assert r.error is None, r.error
        a = alone[r.rid]
        if isinstance(a, tuple):
            assert r.output[0] == pytest.approx(a[0], rel=1e-6)
            assert np.array_equal(r.output[1], a[1])
        else:
            assert np.array_equal(r.output, a)
