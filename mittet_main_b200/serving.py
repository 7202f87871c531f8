"""Request loop: continuous batching of forward and gradient solves on one GPU.

Requests (each its own model, grid, shots, receivers and time base) arrive
over time.  The server keeps ``n_slots`` worker slots; a waiting request is
admitted as soon as a slot is free and its device-memory estimate fits what
is left of the HBM budget (first come first served, but a request that does
not fit lets later, smaller ones go ahead).  Each slot owns solver handles,
and with them CUDA streams, so admitted requests run concurrently on the GPU.

A slot keeps one handle per grid it has served (model, fields and psi slabs
stay resident on the device) and reuses it for the next request of that
grid, so switching grids never frees device memory: a freed buffer would
synchronise the whole device and stall the other slots' streams.  The memory
those idle handles hold counts against the budget; a request that does not
fit otherwise evicts idle handles of free slots, least recently used first.
The C-ABI calls release the GIL, so slots are host threads.

Waiting requests are considered in arrival order (``policy="fcfs"``) or,
with ``policy="sjf"``, smallest estimated work first (cell-updates; a
gradient counts about four forwards), each request's estimate divided by
1 + (time waited / ``aging_s``) so a large request is not passed over for
ever.  Under a burst of arrivals the small requests then finish first
instead of queueing behind large ones, which lowers the median latency at
the same throughput.

Latency = completion - arrival.  ``serial_latencies`` gives a plain path
for comparison from measured service times: one request at a time, in
arrival order.
"""
from __future__ import annotations

import threading
import time
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np


@dataclass
class Request:
    rid: int
    arrival: float               # seconds after the start of the run
    workload: object             # workloads.Workload
    mode: str = "forward"        # "forward" or "gradient"
    obs: Optional[np.ndarray] = None
    checkpoint_every: int = 200


@dataclass
class Result:
    rid: int
    arrival: float
    start: float
    done: float
    slot: int
    output: object = None
    error: Optional[str] = None

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def estimate_bytes(wl, mode: str = "forward", checkpoint_every: int = 200) -> int:
    """Device memory a request needs on a fresh handle (fields, psi slabs,
    model, traces, DFT ring/accumulators; for gradients the checkpoint and
    segment-history buffers)."""
    cp = wl.cp
    esz = 8 if cp.precision == 1 else 4
    px = -(-cp.nx // 32) * 32
    fshot = px * cp.ny * cp.nz
    ns = len(wl.shots)
    nc = cp.ncpml
    slab = 2 * (nc * cp.ny * cp.nz + cp.nz * nc * px + nc * cp.ny * px)  # both slab groups, rough
    b = ns * (6 * fshot + 4 * slab) * esz + 2 * fshot * esz + cp.nx * cp.ny * cp.nz * 8  # + FP64 model upload stage
    b += ns * len(wl.receivers) * wl.nt * esz + ns * len(wl.receivers) * len(wl.omega) * 16
    if wl.volume_dft:
        b += 128 * 3 * ns * fshot * esz + ns * 3 * len(wl.omega) * fshot * 16  # 128-step ring, FP64 accumulators
    if mode == "gradient":
        K = checkpoint_every
        ncheck = -(-wl.nt // K)
        b += ns * esz * ((K + 1) * 6 * fshot + ncheck * (6 * fshot + 4 * slab) + 19 * fshot) + ns * 8 * fshot
    return int(b)


def grid_key(wl):
    """Handles are interchangeable between requests with the same key."""
    cp = wl.cp
    return (cp.nx, cp.ny, cp.nz, cp.precision, cp.flavor, cp.dx, cp.dy, cp.dz, cp.dt, cp.cmax, cp.ncpml, cp.mu0,
            cp.omega0, cp.device)


def run_request(solver_cache: dict, req: Request):
    """Default executor: solve one request on the cached handle of its grid
    (created on first use; handles of other grids stay cached)."""
    from .solver import MittetSolver

    wl = req.workload
    key = grid_key(wl)
    s = solver_cache.get(key)
    if s is None:
        s = MittetSolver(wl.cp)
        solver_cache[key] = s
    s.set_model(wl.sigma, wl.mu)
    s.set_shots(wl.shots)
    s.set_wavelet(wl.wavelet)
    s.set_receivers(wl.receivers)
    s.set_freqs(wl.omega)
    s.set_volume_dft(wl.volume_dft) if wl.volume_dft else s.set_volume_dft("")
    if req.mode == "gradient":
        try:
            return s.gradient(wl.nt, req.obs, req.checkpoint_every)
        finally:
            # the admission estimate counts the gradient buffers for this
            # request only: hand them back before the slot takes other work
            s.release_gradient_buffers()
    spec, _ = s.forward(wl.nt)
    return spec


def work_estimate(req) -> float:
    """Cell-updates a request performs (a gradient: checkpoint pass,
    recompute and adjoint, about 4.4 forwards)."""
    wl = req.workload
    cp = wl.cp
    w = float(cp.nx * cp.ny * cp.nz) * wl.nt * len(wl.shots)
    return w * (4.4 if req.mode == "gradient" else 1.0)


def _default_key(req):
    try:
        return grid_key(req.workload)
    except AttributeError:
        return None


class MittetServer:
    def __init__(self, n_slots: int = 4, hbm_budget: float = 150e9,
                 executor: Optional[Callable] = None, estimator: Optional[Callable] = None,
                 keyer: Optional[Callable] = None, resident_estimator: Optional[Callable] = None,
                 policy: str = "fcfs", work: Optional[Callable] = None, aging_s: float = 30.0):
        if policy not in ("fcfs", "sjf"):
            raise ValueError(f"unknown admission policy {policy!r}")
        self.n_slots = n_slots
        self.policy = policy
        self.work = work or work_estimate
        self.aging_s = float(aging_s)
        self.budget = float(hbm_budget)
        self.executor = executor or run_request
        self.estimator = estimator or (lambda r: estimate_bytes(r.workload, r.mode, r.checkpoint_every))
        # the handle a request leaves cached: its forward state (gradient
        # buffers are released at the end of a gradient request)
        self.resident_estimator = resident_estimator or (
            estimator if estimator is not None else (lambda r: estimate_bytes(r.workload, "forward")))
        self.keyer = keyer or _default_key
        self._lock = threading.Condition()
        self.peak_in_use = 0.0
        self.max_concurrent = 0
        self.evictions = 0
        self.reuses = 0

    def need(self, req) -> float:
        """Bytes a request is admitted for.  A gradient processes its shots in
        groups sized to the free device memory (mittet_gradient), so one whose
        estimate for all shots at once exceeds the budget is admitted for the
        whole budget: it then runs with nothing else admitted beside it."""
        b = float(self.estimator(req))
        return min(b, self.budget) if getattr(req, "mode", "forward") == "gradient" else b

    def priority(self, req, t: float) -> float:
        """SJF admission key at time t (smaller goes first): the estimated
        work divided by 1 + time waited / aging_s."""
        return float(self.work(req)) / (1.0 + max(0.0, t - req.arrival) / self.aging_s)

    def run(self, requests: list, realtime: bool = True) -> list:
        """Serve ``requests`` (sorted by arrival); returns one Result per request."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        for r in reqs:
            if self.need(r) > self.budget:
                raise ValueError(f"request {r.rid} needs more than the whole HBM budget")
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0  # noqa: E731
        waiting: list = []
        results: dict = {}
        free_slots = list(range(self.n_slots))
        caches = [dict() for _ in range(self.n_slots)]
        resident: dict = {}   # (slot, key) -> bytes the cached handle holds
        last_use: dict = {}   # (slot, key) -> time of its last request
        state = {"extra": 0.0, "running": 0}
        threads = []

        def held():
            return state["extra"] + sum(resident.values())

        def worker(slot, req, key, extra, start):
            out, err = None, None
            try:
                out = self.executor(caches[slot], req)
            except Exception as ex:  # reported per request
                err = f"{type(ex).__name__}: {ex}"
            done = now()
            with self._lock:
                results[req.rid] = Result(req.rid, req.arrival, start, done, slot, out, err)
                state["extra"] -= extra
                if key is not None:
                    resident[(slot, key)] = max(resident.get((slot, key), 0.0), float(self.resident_estimator(req)))
                    last_use[(slot, key)] = done
                state["running"] -= 1
                free_slots.append(slot)
                self._lock.notify_all()

        def evict_for(amount, keep):
            """Close idle cached handles of free slots (LRU) until ``amount``
            more bytes fit; False if they cannot."""
            cands = sorted((k for k in resident if k[0] in free_slots and k != keep), key=lambda k: last_use.get(k, 0))
            while held() + amount > self.budget and cands:
                k = cands.pop(0)
                h = caches[k[0]].pop(k[1], None)
                if h is not None and hasattr(h, "close"):
                    h.close()
                resident.pop(k, None)
                self.evictions += 1
            return held() + amount <= self.budget

        pending = list(reqs)
        with self._lock:
            while pending or waiting or state["running"] > 0:
                t = now()
                while pending and (not realtime or pending[0].arrival <= t):
                    waiting.append(pending.pop(0))
                # admit in policy order; a request that does not fit lets later ones pass
                admitted = True
                while admitted:
                    admitted = False
                    order = list(waiting)
                    if self.policy == "sjf":
                        tnow = now()
                        order.sort(key=lambda q: self.priority(q, tnow))
                    for r in order:
                        if not free_slots:
                            break
                        need = self.need(r)
                        key = self.keyer(r)
                        # a free slot that already holds this grid's handle first
                        slot = next((s for s in free_slots if (s, key) in resident), free_slots[0])
                        extra = max(0.0, need - resident.get((slot, key), 0.0))
                        if held() + extra > self.budget and not evict_for(extra, (slot, key)):
                            continue
                        waiting.remove(r)
                        free_slots.remove(slot)
                        if (slot, key) in resident:
                            self.reuses += 1
                        state["extra"] += extra
                        state["running"] += 1
                        self.peak_in_use = max(self.peak_in_use, held())
                        self.max_concurrent = max(self.max_concurrent, state["running"])
                        th = threading.Thread(target=worker, args=(slot, r, key, extra, now()), daemon=True)
                        threads.append(th)
                        th.start()
                        admitted = True
                        break
                if not pending and not waiting and state["running"] == 0:
                    break
                timeout = None
                if pending and realtime:
                    timeout = max(0.0, pending[0].arrival - now())
                self._lock.wait(timeout=timeout if timeout is not None else 0.5)
        for th in threads:
            th.join()
        for c in caches:
            for s in c.values():
                if hasattr(s, "close"):
                    s.close()
        return [results[r.rid] for r in reqs]


def serial_latencies(requests: list, service_times: dict) -> dict:
    """Plain path: one request at a time in arrival order; returns rid -> latency."""
    t = 0.0
    out = {}
    for r in sorted(requests, key=lambda r: r.arrival):
        start = max(t, r.arrival)
        t = start + service_times[r.rid]
        out[r.rid] = t - r.arrival
    return out


def percentile(xs, q):
    return float(np.percentile(np.asarray(xs, dtype=float), q)) if len(xs) else float("nan")


def poisson_requests(n: int, rate: float, make_workload: Callable[[int, np.random.Generator], object],
                     seed: int = 2026, gradient_every: int = 4) -> list:
    """n requests with Poisson arrivals at ``rate`` per second; every
    ``gradient_every``-th request is a gradient (forward:gradient = 3:1)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        wl = make_workload(i, rng)
        mode = "gradient" if gradient_every and i % gradient_every == gradient_every - 1 else "forward"
        obs = None
        if mode == "gradient":
            obs = np.zeros((len(wl.shots), len(wl.receivers), len(wl.omega)), dtype=complex)
        out.append(Request(i, t, wl, mode, obs, checkpoint_every=max(1, min(200, wl.nt // 4))))
    return out
