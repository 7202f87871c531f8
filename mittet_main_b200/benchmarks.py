"""Reports of the batching, gradient and serving workloads (``bench.py --mode``).

batching: 64 shots of one 192x192x128 model in one batched solve (one CUDA
  graph per 64 steps, all shots in every launch) against the same 64 shots
  solved one at a time on the same GPU; shot-solves/s of both and the ratio.
gradient: FWI gradient of the 128x128x96 model, 16 shots, Ex/Ey at 3
  frequencies, checkpoints every 200 steps; seconds per gradient and Gcell/s
  of forward-equivalent work.
serving: Poisson arrivals of forward (3) and gradient (1) requests over the
  grid set {64^3, 96^3, 128^3, 160x160x96, 256x256x192} (domain 6.4 km wide),
  1-32 shots, Nt scaled with the grid; p50/p99 latency and shot-solves/s of
  the server against two plain paths on the same GPU: one request at a time
  (its shots batched), and one shot at a time.
Times are device-synchronised wall clock of the public API calls.
"""
from __future__ import annotations

import time
from dataclasses import replace

import numpy as np


def _sync():
    import torch
    torch.cuda.synchronize()


def batching_ratio(wl, repeats: int = 1) -> dict:
    """All shots of ``wl`` in one batched solve against the same shots solved
    one at a time (mittet_set_sources + mittet_forward per shot) on the same
    GPU; best of ``repeats`` timed runs of each after a warm-up."""
    ns = len(wl.shots)
    from mittet_main_b200 import workloads as W
    tb = float("inf")
    with W.make_solver(wl) as s:
        s.forward(wl.nt)  # warm-up (autotune, graph)
        for _ in range(repeats):
            _sync()
            t0 = time.perf_counter()
            spec_b, _ = s.forward(wl.nt)
            _sync()
            tb = min(tb, time.perf_counter() - t0)
    one = replace(wl, shots=[wl.shots[0]])
    tp = float("inf")
    with W.make_solver(one) as s:
        s.forward(wl.nt)
        for _ in range(repeats):
            _sync()
            t0 = time.perf_counter()
            specs = []
            for k in range(ns):
                s.set_shots([wl.shots[k]])
                sp, _ = s.forward(wl.nt)
                specs.append(sp[0])
            _sync()
            tp = min(tp, time.perf_counter() - t0)
    same = all(np.array_equal(spec_b[k], specs[k]) for k in range(ns))
    cells = wl.ncell * wl.nt
    return {"workload": wl.name, "nt": wl.nt, "shots": ns,
            "batched_shot_solves_per_s": ns / tb, "one_at_a_time_shot_solves_per_s": ns / tp,
            "batched_vs_one_at_a_time": tp / tb, "batched_gcell_s": ns * cells / tb / 1e9,
            "one_at_a_time_gcell_s": ns * cells / tp / 1e9, "identical_results": bool(same)}


def batching(args):
    from mittet_main_b200 import workloads as W
    from mittet_main_b200.capi import FP64, FP32
    prec = FP64 if args.precision == "fp64" else FP32
    nt = args.nt or 5000
    kw = {}
    if args.grid:
        kw["nx"], kw["ny"], kw["nz"] = (int(v) for v in args.grid.split("x"))
    if getattr(args, "shots", 0):
        kw["nshot"] = args.shots
    wl = W.batched(nt=nt, precision=prec, **kw)
    return {"report": "batching", **batching_ratio(wl)}


def gradient(args):
    from mittet_main_b200 import workloads as W
    from mittet_main_b200.capi import FP64, FP32
    prec = FP64 if args.precision == "fp64" else FP32
    nt = args.nt or 4000
    nshot = getattr(args, "shots", 0) or 16
    ck = getattr(args, "checkpoint", 0) or 200
    true = W.gradient_case(nt=nt, precision=prec, true_model=True, nshot=nshot)
    start = W.gradient_case(nt=nt, precision=prec, true_model=False, nshot=nshot)
    with W.make_solver(true) as s:
        obs, _ = s.forward(true.nt)
    with W.make_solver(start) as s:
        s.gradient(start.nt, obs, ck)  # warm-up
        _sync()
        t0 = time.perf_counter()
        J, G = s.gradient(start.nt, obs, ck)
        _sync()
        tg = time.perf_counter() - t0
        t0 = time.perf_counter()
        s.forward(start.nt)
        _sync()
        tf = time.perf_counter() - t0
    cells = start.ncell * start.nt * len(start.shots)
    nc = start.cp.ncpml
    body = G[nc:-nc, nc:-nc, nc:-nc]
    return {"report": "gradient", "workload": start.name, "nt": start.nt, "shots": len(start.shots), "checkpoint_every": ck,
            "seconds_per_gradient": tg, "seconds_per_forward": tf, "gradient_over_forward": tg / tf,
            "forward_equivalent_gcell_s": cells / tg / 1e9, "misfit": J,
            "grad_max_abs": float(np.abs(body).max())}


def serving(args):
    from mittet_main_b200 import workloads as W
    from mittet_main_b200.capi import FP32
    from mittet_main_b200.serving import (MittetServer, percentile, poisson_requests, run_request,
                                          serial_latencies)
    grids = [(64, 64, 64), (96, 96, 96), (128, 128, 128), (160, 160, 96), (256, 256, 192)]
    scale = args.nt / 6000.0 if args.nt else 0.1  # Nt = 6000 * nx/256 * scale

    def make(i, rng):
        nx, ny, nz = grids[int(rng.integers(len(grids)))]
        nshot = int(rng.integers(1, 33))
        nt = max(50, int(6000 * nx / 256 * scale))
        return W.serving_case(nx, ny, nz, nshot, nt, seed=int(rng.integers(1 << 30)))

    reqs = poisson_requests(args.requests, args.rate, make)
    # serial plain path: one request at a time on one handle
    service = {}
    cache = {}
    for r in reqs[:1]:
        run_request(cache, r)  # warm-up
    for r in reqs:
        _sync()
        t0 = time.perf_counter()
        run_request(cache, r)
        _sync()
        service[r.rid] = time.perf_counter() - t0
    for s in cache.values():
        s.close()
    ser = serial_latencies(reqs, service)
    # plain one-shot-at-a-time path: every shot of a request solved alone, one
    # after another.  Shots of a request cost the same, so one timed
    # single-shot solve per (grid, Nt, mode) gives the request's service time.
    from mittet_main_b200.serving import Request
    one = {}
    for r in reqs:
        wl = r.workload
        key = (wl.cp.nx, wl.cp.ny, wl.cp.nz, wl.nt, r.mode)
        if key in one:
            continue
        single = Request(-1, 0.0, replace(wl, shots=[wl.shots[0]]), r.mode,
                         None if r.obs is None else r.obs[:1], r.checkpoint_every)
        c = {}
        run_request(c, single)  # warm-up (autotune, graph)
        _sync()
        t0 = time.perf_counter()
        run_request(c, single)
        _sync()
        one[key] = time.perf_counter() - t0
        for sv in c.values():
            sv.close()
    service1 = {r.rid: len(r.workload.shots) * one[(r.workload.cp.nx, r.workload.cp.ny, r.workload.cp.nz,
                                                     r.workload.nt, r.mode)] for r in reqs}
    ser1 = serial_latencies(reqs, service1)
    t1 = 0.0
    for r in sorted(reqs, key=lambda r: r.arrival):
        t1 = max(t1, r.arrival) + service1[r.rid]
    srv = MittetServer(n_slots=4, hbm_budget=150e9)
    t0 = time.perf_counter()
    res = srv.run(reqs)
    wall = time.perf_counter() - t0
    shots = sum(len(r.workload.shots) for r in reqs)
    lat = [r.latency for r in res]
    errors = [r.error for r in res if r.error]
    t = 0.0
    for r in sorted(reqs, key=lambda r: r.arrival):
        t = max(t, r.arrival) + service[r.rid]
    return {"report": "serving", "requests": len(reqs), "rate_per_s": args.rate, "nt_scale": scale,
            "server_p50_s": percentile(lat, 50), "server_p99_s": percentile(lat, 99),
            "server_shot_solves_per_s": shots / wall, "serial_p50_s": percentile(list(ser.values()), 50),
            "serial_p99_s": percentile(list(ser.values()), 99), "serial_shot_solves_per_s": shots / t,
            "one_shot_p50_s": percentile(list(ser1.values()), 50), "one_shot_p99_s": percentile(list(ser1.values()), 99),
            "one_shot_shot_solves_per_s": shots / t1, "server_vs_one_shot": (shots / wall) / (shots / t1),
            "max_concurrent": srv.max_concurrent, "peak_budget_bytes": srv.peak_in_use, "errors": errors[:3]}
