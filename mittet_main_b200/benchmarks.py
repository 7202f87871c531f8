"""Reports of the batching, gradient and serving workloads (``bench.py --mode``).

batching: 64 shots of one 192x192x128 model in one batched solve (one CUDA
  graph per 128 steps, all shots in every launch) against the same 64 shots
  solved one at a time on the same GPU; shot-solves/s of both and the ratio.
gradient: FWI gradient of the 128x128x96 model, 16 shots, Ex/Ey at 3
  frequencies, checkpoints every 200 steps; seconds per gradient and Gcell/s
  of forward-equivalent work.
serving: Poisson arrivals of forward (3) and gradient (1) requests over the
  grid set {64^3, 96^3, 128^3, 160x160x96, 256x256x192} (domain 6.4 km wide),
  1-32 shots, Nt = 6000 nx / 256; p50/p99 latency and shot-solves/s of the
  server against two plain paths served in real time on the same GPU: one
  request at a time (its shots batched), and one shot at a time.
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
        path_b = s.launch_path()
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
        path_p = s.launch_path()
    same = all(np.array_equal(spec_b[k], specs[k]) for k in range(ns))
    cells = wl.ncell * wl.nt
    return {"workload": wl.name, "nt": wl.nt, "shots": ns,
            "batched_shot_solves_per_s": ns / tb, "one_at_a_time_shot_solves_per_s": ns / tp,
            "batched_vs_one_at_a_time": tp / tb, "batched_gcell_s": ns * cells / tb / 1e9,
            "one_at_a_time_gcell_s": ns * cells / tp / 1e9, "identical_results": bool(same),
            "batched_launch": path_b, "one_at_a_time_launch": path_p}


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


def one_shot_at_a_time(solver_cache: dict, req):
    """Executor of the plain one-shot-at-a-time path: every shot of the
    request solved alone on the grid's handle, one after another."""
    from mittet_main_b200.serving import Request, run_request
    wl = req.workload
    outs = []
    for k, shot in enumerate(wl.shots):
        single = Request(req.rid, req.arrival, replace(wl, shots=[shot]), req.mode,
                         None if req.obs is None else req.obs[k:k + 1], req.checkpoint_every)
        outs.append(run_request(solver_cache, single))
    return outs


def serving(args):
    """The serving mix: Poisson arrivals (rate args.rate, args.requests
    requests, seeded), grids {64^3, 96^3, 128^3, 160x160x96, 256x256x192}
    with dx = 6400 m / nx, 1-32 shots, Nt = 6000 nx / 256 (args.nt scales it:
    Nt x args.nt / 6000), forward:gradient = 3:1, 150 GB budget.  Three
    arms, each served in real time from the same arrival process on the same
    GPU: the server (4 slots, continuous batching, smallest estimated work
    first with ageing), one request at a time (one slot, arrival order, its
    shots batched) and one shot at a time (one slot, arrival order, each shot
    solved alone)."""
    from mittet_main_b200 import workloads as W
    from mittet_main_b200.serving import MittetServer, percentile, poisson_requests, run_request
    grids = [(64, 64, 64), (96, 96, 96), (128, 128, 128), (160, 160, 96), (256, 256, 192)]
    scale = args.nt / 6000.0 if args.nt else 1.0

    def make(i, rng):
        nx, ny, nz = grids[int(rng.integers(len(grids)))]
        nshot = int(rng.integers(1, 33))
        nt = max(50, int(6000 * nx / 256 * scale))
        return W.serving_case(nx, ny, nz, nshot, nt, seed=int(rng.integers(1 << 30)))

    n = args.requests
    reqs = poisson_requests(n, args.rate, make)
    shots = sum(len(r.workload.shots) for r in reqs)
    # warm-up: the autotuner's choices are cached per (grid, shots, ...) for
    # the process; fill them for every batch shape the arms meet with short
    # solves, so that no arm pays for tuning the others then reuse
    from mittet_main_b200.serving import Request
    seen = set()
    for r in reqs:
        wl = r.workload
        for ns in (len(wl.shots), 1):
            key = (wl.cp.nx, wl.cp.ny, wl.cp.nz, ns)
            if key in seen:
                continue
            seen.add(key)
            short = replace(wl, shots=wl.shots[:ns], nt=64, wavelet=wl.wavelet[:65])
            run_request({}, Request(-1, 0.0, short))
    _sync()
    out = {"report": "serving", "requests": n, "rate_per_s": args.rate, "nt_scale": scale, "shots": shots,
           "grids": sorted({f"{r.workload.cp.nx}x{r.workload.cp.ny}x{r.workload.cp.nz}" for r in reqs}),
           "modes": {m: sum(r.mode == m for r in reqs) for m in ("forward", "gradient")}}
    arms = [("server", 4, run_request, "sjf"), ("one_request_at_a_time", 1, run_request, "fcfs"),
            ("one_shot_at_a_time", 1, one_shot_at_a_time, "fcfs")]
    for name, slots, ex, policy in arms:
        srv = MittetServer(n_slots=slots, hbm_budget=150e9, executor=ex, policy=policy)
        _sync()
        t0 = time.perf_counter()
        res = srv.run(reqs)
        _sync()
        wall = time.perf_counter() - t0
        lat = [r.latency for r in res]
        errors = [r.error for r in res if r.error]
        out[name] = {"policy": policy, "p50_s": percentile(lat, 50), "p99_s": percentile(lat, 99), "wall_s": wall,
                     "shot_solves_per_s": shots / wall, "max_concurrent": srv.max_concurrent,
                     "peak_budget_bytes": srv.peak_in_use, "handle_reuses": srv.reuses,
                     "evictions": srv.evictions, "errors": errors[:3]}
    out["server_vs_one_shot"] = out["server"]["shot_solves_per_s"] / out["one_shot_at_a_time"]["shot_solves_per_s"]
    out["server_vs_one_request"] = (out["server"]["shot_solves_per_s"] /
                                    out["one_request_at_a_time"]["shot_solves_per_s"])
    return out
