"""CPU tests of the serving loop's admission logic with a stand-in executor
(no GPU): the HBM budget is never exceeded, every request completes once,
requests overlap when slots and memory allow, and a request too large to fit
lets smaller later ones through."""
import threading
import time

import pytest

from mittet_main_b200.serving import MittetServer, Request, percentile, serial_latencies


class FakeWL:
    pass


def make(rid, arrival, size):
    r = Request(rid, arrival, FakeWL())
    r.size = size
    return r


def test_budget_respected_and_all_complete():
    lock = threading.Lock()
    live = {"bytes": 0, "peak": 0}

    def execu(cache, req):
        with lock:
            live["bytes"] += req.size
            live["peak"] = max(live["peak"], live["bytes"])
        time.sleep(0.02)
        with lock:
            live["bytes"] -= req.size
        return req.rid * 10

    reqs = [make(i, 0.002 * i, size=(30 if i % 3 else 70)) for i in range(24)]
    srv = MittetServer(n_slots=4, hbm_budget=100, executor=execu, estimator=lambda r: r.size)
    res = srv.run(reqs)
    assert sorted(r.rid for r in res) == list(range(24))
    assert all(r.output == r.rid * 10 and r.error is None for r in res)
    assert live["peak"] <= 100 and srv.peak_in_use <= 100
    assert srv.max_concurrent >= 2


def test_small_requests_pass_a_blocked_large_one():
    order = []

    def execu(cache, req):
        order.append(req.rid)
        time.sleep(0.05 if req.rid == 0 else 0.01)
        return None

    reqs = [make(0, 0.0, 60), make(1, 0.001, 60), make(2, 0.002, 10), make(3, 0.003, 10)]
    srv = MittetServer(n_slots=4, hbm_budget=100, executor=execu, estimator=lambda r: r.size)
    res = {r.rid: r for r in srv.run(reqs)}
    # request 1 (60) cannot start while 0 (60) runs; 2 and 3 (10 each) can
    assert res[2].start < res[1].start and res[3].start < res[1].start


def test_oversized_request_is_rejected():
    srv = MittetServer(n_slots=2, hbm_budget=10, executor=lambda c, r: None, estimator=lambda r: r.size)
    with pytest.raises(ValueError):
        srv.run([make(0, 0.0, 11)])


def test_serial_latency_model():
    reqs = [make(0, 0.0, 1), make(1, 0.5, 1), make(2, 0.6, 1)]
    lat = serial_latencies(reqs, {0: 1.0, 1: 1.0, 2: 1.0})
    assert lat == {0: 1.0, 1: 1.5, 2: 2.4}
    assert percentile([1, 2, 3, 4], 50) == 2.5


def test_slots_keep_handles_per_grid_within_the_budget():
    """Idle handles of every grid a slot served stay cached and count against
    the budget; a request of a cached grid reuses its slot's handle, and one
    that does not fit next to the cached handles evicts idle ones (LRU)."""
    lock = threading.Lock()
    made = []

    class Handle:
        def __init__(self, key, size):
            self.key, self.size, self.closed = key, size, False

        def close(self):
            self.closed = True

    live = {"bytes": 0, "peak": 0}

    def held_now(caches_seen):
        return sum(h.size for h in caches_seen if not h.closed)

    def execu(cache, req):
        with lock:
            h = cache.get(req.key)
            if h is None:
                h = Handle(req.key, req.size)
                cache[req.key] = h
                made.append(h)
            live["peak"] = max(live["peak"], held_now(made))
        time.sleep(0.01)
        return req.rid

    reqs = []
    for i in range(16):
        r = make(i, 0.02 * i, size=(40 if i % 4 == 3 else 20))
        r.key = "big" if i % 4 == 3 else ("a" if i % 2 else "b")
        reqs.append(r)
    srv = MittetServer(n_slots=2, hbm_budget=100, executor=execu, estimator=lambda r: r.size,
                       keyer=lambda r: r.key, resident_estimator=lambda r: r.size)
    res = srv.run(reqs)
    assert sorted(r.output for r in res) == list(range(16))
    assert srv.peak_in_use <= 100 and live["peak"] <= 100
    assert srv.reuses > 0
    # fewer handles than requests were created: slots reused them
    assert len(made) < len(reqs)


def test_gradient_larger_than_the_budget_runs_alone():
    """A gradient whose all-shots estimate exceeds the budget is admitted for
    the whole budget (its shots then run in groups that fit), alone."""
    running = {"n": 0, "max_with_big": 0}
    lock = threading.Lock()

    def execu(cache, req):
        with lock:
            running["n"] += 1
            if req.mode == "gradient":
                running["max_with_big"] = max(running["max_with_big"], running["n"])
        time.sleep(0.02)
        with lock:
            running["n"] -= 1
        return req.rid

    reqs = [make(i, 0.001 * i, 20) for i in range(6)]
    reqs[2].mode = "gradient"
    reqs[2].size = 500
    srv = MittetServer(n_slots=4, hbm_budget=100, executor=execu, estimator=lambda r: r.size)
    res = srv.run(reqs)
    assert sorted(r.output for r in res) == list(range(6))
    assert running["max_with_big"] == 1 and srv.peak_in_use <= 100


def test_sjf_admits_the_smallest_waiting_request_first():
    """With one slot and a burst of arrivals, policy="sjf" runs the waiting
    requests in order of estimated work; "fcfs" in arrival order."""
    def run(policy):
        order = []

        def execu(cache, req):
            order.append(req.rid)
            time.sleep(0.02)
            return None

        # request 0 occupies the slot while 1..4 arrive
        reqs = [make(0, 0.0, 5), make(1, 0.001, 40), make(2, 0.002, 10), make(3, 0.003, 30), make(4, 0.004, 20)]
        srv = MittetServer(n_slots=1, hbm_budget=100, executor=execu, estimator=lambda r: r.size,
                           policy=policy, work=lambda r: r.size, aging_s=1e6)
        srv.run(reqs)
        return order

    assert run("fcfs") == [0, 1, 2, 3, 4]
    assert run("sjf") == [0, 2, 4, 3, 1]


def test_sjf_ageing_lets_a_long_waiting_request_through():
    """The SJF key divides the work by 1 + waited / aging_s: a large request
    that has waited many ageing periods goes before a small new one."""
    srv = MittetServer(n_slots=1, hbm_budget=100, estimator=lambda r: r.size, policy="sjf",
                       work=lambda r: r.size, aging_s=1.0)
    big, small = make(0, 0.0, 50), make(1, 9.0, 2)
    assert srv.priority(big, 9.0) > srv.priority(small, 9.0)     # 50 / 10 = 5 > 2 / 1
    late = make(2, 29.9, 2)
    assert srv.priority(big, 30.0) < srv.priority(late, 30.0)    # 50 / 31 = 1.61 < 2 / 1.1 = 1.82


def test_unknown_policy_is_rejected():
    with pytest.raises(ValueError):
        MittetServer(policy="lifo")


def test_work_estimate_counts_cell_updates():
    from mittet_main_b200 import workloads as W
    from mittet_main_b200.serving import work_estimate

    wl = W.serving_case(32, 32, 32, 3, 100)
    fwd = Request(0, 0.0, wl)
    grad = Request(1, 0.0, wl, mode="gradient")
    assert work_estimate(fwd) == 32 ** 3 * 100 * 3
    assert work_estimate(grad) == 4.4 * work_estimate(fwd)
