#!/usr/bin/env python
"""Benchmark of the Mittet fictitious-wave FDTD forward solve on B200.

One bench "step" is one shot-solve of the workload: the full time loop
(Nt leapfrog steps of the (2,4) Yee + CPML stencil with source injection and
receiver sampling) plus the f_to_d transform (receiver spectra and, for the
default workload, the full-volume f_to_d of Ex/Ey/Ez at 4 frequencies).

Default workload (N=1): 256x256x192 cells, dx 25 m, 16-cell CPML, seeded
log-normal model + resistive body, one Ex dipole, Nt 6000, 256 receivers,
FP32 fields with FP64 DFT accumulators.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).  `value` is whole-job Gcell/s with inputs
resident in HBM; `e2e` is the same metric through the C ABI with host
buffers (H2D of the model and D2H of every spectrum inside the timed region).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        import tempfile
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if "Active" in r[5 + q] and "Not" not in r[5 + q]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def stencil_bytes(wl, esz):
    """Algorithmic bytes of one E-phase launch (the dominant kernel):
    read Ex Ey Ez Hx Hy Hz and the model word, write Ex Ey Ez (10 words per cell),
    + the FP32 ring write of Ex Ey Ez when the full-volume DFT is on,
    + 2 psi read + 2 psi write per cell of each E slab group."""
    cp = wl.cp
    n = cp.nx * cp.ny * cp.nz
    b = 10 * esz * n
    if wl.volume_dft:
        b += len(wl.volume_dft) * esz * n
    nc = cp.ncpml
    # E slab widths of the ncver0027 ranges: (ncpml-1) cells each side
    w = [2 * (nc - 1)] * 3
    slab_cells = w[0] * cp.ny * cp.nz + w[1] * cp.nx * cp.nz + w[2] * cp.nx * cp.ny
    b += 4 * esz * slab_cells
    return b * len(wl.shots)


def stencil_read_bytes(wl, esz):
    """Algorithmic read bytes of one E-phase launch: 6 fields and the model
    word per cell, 2 psi per cell of each E slab group."""
    cp = wl.cp
    n = cp.nx * cp.ny * cp.nz
    nc = cp.ncpml
    slab_cells = 2 * (nc - 1) * (cp.ny * cp.nz + cp.nx * cp.nz + cp.nx * cp.ny)
    return (7 * esz * n + 2 * esz * slab_cells) * len(wl.shots)


def e_phase_profile(esz, volume):
    """DRAM read bytes per cell of the E-phase kernels from the committed ncu
    summary (a one-pass capture of every E-phase launch of a step of the
    256x256x96 twin, FP32 fields with the 3-component volume DFT); None for
    other configurations."""
    import re
    path = os.path.join(ROOT, "profiles", "e_phase_dram_256x256x96.md")
    if esz != 4 or volume != "xyz" or not os.path.exists(path):
        return None
    m = re.search(r"e_phase_dram_read_bytes_per_cell:\s*([0-9.]+)", open(path).read())
    return {"read": float(m.group(1)), "source": "profiles/e_phase_dram_256x256x96.md"} if m else None


def run_cpu_baseline(wl, budget_s=12.0):
    """Oracle (FP64 CPU restatement, all host threads) on a bounded sample of the
    workload: a few time steps of the same grid.  Returns (Gcell/s, sample text, threads)."""
    from oracle import oracle as O
    cp = wl.cp
    p = O.Params(nx=cp.nx, ny=cp.ny, nz=cp.nz, dx=cp.dx, dy=cp.dy, dz=cp.dz, dt=cp.dt, ncpml=cp.ncpml,
                 cmax=cp.cmax, omega0=cp.omega0)
    mu = np.full(wl.sigma.shape, cp.mu0)
    src = wl.shots[0].points
    # size the sample to ~budget_s of CPU work from a 2-step probe (set-up
    # included, so an upper bound on the step time), then time it as the
    # difference of a 5-step and a (5+k)-step run so that set-up cancels
    t0 = time.perf_counter()
    O.forward(p, wl.sigma, mu, src, wl.wavelet, [], 2)
    est = (time.perf_counter() - t0) / 2
    k = int(min(400, max(20, budget_s / max(est, 1e-3))))
    sec = O.time_oracle_steps(p, wl.sigma, mu, src, wl.wavelet, 5, 5 + k)
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    g = cp.nx * cp.ny * cp.nz / sec / 1e9
    return g, (f"oracle FP64, {cp.nx}x{cp.ny}x{cp.nz} grid, {k} time steps "
               f"(difference of 5- and {5 + k}-step runs)"), threads


def run_reference(args, wl):
    """--impl reference: the reference's own satan_i C kernels (oracle/_ref) on
    the host cores, same grid, W+K segments of a few time steps each."""
    from oracle import oracle as O
    cp = wl.cp
    threads = os.cpu_count() or 1
    seg = args.ref_seg_steps
    cx, cy, cz = wl.shots[0].points[0][:3]
    times = O.time_satan_reference(cp.nx, cp.ny, cp.nz, cp.dx, cp.dy, cp.dz, cp.ncpml, cp.omega0, wl.sigma,
                                   seg, args.warmup + args.steps, (cx, cy, cz), 0, threads)
    timed = times[args.warmup:]
    t = float(np.sum(timed))
    ncell = cp.nx * cp.ny * cp.nz
    value = ncell * seg * args.steps / t / 1e9
    sample = (f"satan_i e/h_field_cpml42 + e/hpml_abcs4 (gcc -fopenmp -O3 as satan_i/Makefile:12, "
              f"{threads} threads), "
              f"{cp.nx}x{cp.ny}x{cp.nz} grid, {seg} time steps per bench step")
    return {
        "metric": "Gcell/s", "value": value, "unit": "Gcell/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl.name, "nt_sample": seg, "note": "CPU reference, bounded sample"},
        "shot_solves_per_s": value * 1e9 / (ncell * wl.nt),
        "cpu_baseline": {"value": value, "unit": "Gcell/s", "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "Gcell/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plain_gpu", choices=["plain_gpu", "batched", "plain_cpu"])
    ap.add_argument("--mode", default="solve", choices=["solve", "batching", "gradient", "serving"],
                    help="solve: the headline line; batching/gradient/serving: the other workloads' reports")
    ap.add_argument("--requests", type=int, default=16, help="serving: number of requests")
    ap.add_argument("--rate", type=float, default=20.0, help="serving: Poisson arrival rate per second")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--nt", type=int, default=0, help="override Nt (0 = workload default)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 sub-record")
    ap.add_argument("--no-batching", action="store_true", help="skip the batched-vs-one-at-a-time sub-record")
    ap.add_argument("--ref-seg-steps", type=int, default=4)
    ap.add_argument("--grid", default="", help="NXxNYxNZ override of the workload grid (profiling cases)")
    ap.add_argument("--no-volume", action="store_true", help="disable the full-volume f_to_d")
    ap.add_argument("--shots", type=int, default=0, help="gradient: shots (0 = 16)")
    ap.add_argument("--checkpoint", type=int, default=0, help="gradient: checkpoint interval (0 = 200)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    from mittet_main_b200 import workloads as W
    from mittet_main_b200.capi import FP32, FP64
    prec = FP64 if args.precision == "fp64" else FP32
    mk = {"plain_gpu": W.plain_gpu, "batched": W.batched, "plain_cpu": W.plain_cpu}[args.workload]
    kw = {"precision": prec}
    if args.nt:
        kw["nt"] = args.nt
    if args.grid:
        kw["nx"], kw["ny"], kw["nz"] = (int(v) for v in args.grid.split("x"))
    if args.no_volume and args.workload == "plain_gpu":
        kw["volume"] = False
    wl = mk(**kw)

    if args.impl == "reference":
        if rank != 0:
            return
        print(json.dumps(run_reference(args, wl)), flush=True)
        return
    if args.mode != "solve":
        from mittet_main_b200 import benchmarks
        print(json.dumps(getattr(benchmarks, args.mode)(args)), flush=True)
        return

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    from dataclasses import replace
    wl = replace(wl, cp=replace(wl.cp, device=dev))
    # weak scaling: each rank solves its own shot(s) of the same model
    solver = W.make_solver(wl)
    nf = len(wl.omega)
    nrec = len(wl.receivers)
    out = torch.zeros((len(wl.shots), nrec, nf, 2), dtype=torch.float64, device=f"cuda:{dev}")
    stream = torch.cuda.current_stream()
    t_ms, launches0, clocks = timed_solves(solver, wl, args.steps, args.warmup, dist, dev, out, stream)
    cells = wl.cell_updates()
    total_cells = cells * args.steps * world
    value = total_cells / (t_ms / 1e3) / 1e9
    gpu_launches = launches0 * args.steps

    # per-kernel device times (CUDA events on the launching stream) for the roofline
    kt = solver.time_kernels(min(128, wl.nt))  # one ring period: the flush runs once
    esz = 8 if prec == FP64 else 4
    peak, peak_kind = peaks()
    roof = roofline(wl, esz, kt, peak, peak_kind)

    # end to end through the public C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        # inputs and outputs in pinned host memory, allocated before the timed region
        sig_pinned = torch.from_numpy(np.ascontiguousarray(wl.sigma, dtype=np.float64)).pin_memory()
        sig_host = sig_pinned.numpy()
        vol_out = None
        if wl.volume_dft:
            vol_out = torch.empty((wl.omega.size, wl.cp.nz, wl.cp.ny, wl.cp.nx), dtype=torch.complex128,
                                  pin_memory=True).numpy()
        h2d = sig_host.nbytes
        d2h = len(wl.shots) * nrec * nf * 16
        if wl.volume_dft:
            d2h += len(wl.shots) * len(wl.volume_dft) * nf * wl.ncell * 16
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            solver.set_model(sig_host)
            spec, _ = solver.forward(wl.nt)
            if wl.volume_dft:
                for s in range(len(wl.shots)):
                    for c in wl.volume_dft:
                        solver.volume_dft(s, "e" + c, out=vol_out)
        torch.cuda.synchronize()
        te = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device=f"cuda:{dev}")
        if dist:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        te = float(te.item())
        e2e = {"value": total_cells / te / 1e9, "unit": "Gcell/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h}
    stencil_variant = solver.tuned_variant()
    launch_path = solver.launch_path()
    solver.close()

    extras = {}
    if rank == 0 and world == 1:
        # the same workload with FP64 fields (the reference's precision)
        if not args.no_fp64 and prec == FP32:
            wl64 = replace(wl, cp=replace(wl.cp, precision=FP64))
            s64 = W.make_solver(wl64)
            out64 = torch.zeros_like(out)
            st64, sw64 = max(1, min(args.steps, 2)), 1
            t64, l64, c64 = timed_solves(s64, wl64, st64, sw64, None, dev, out64, stream)
            kt64 = s64.time_kernels(min(128, wl.nt))
            s64.close()
            extras["fp64"] = {"value": cells * st64 / (t64 / 1e3) / 1e9, "unit": "Gcell/s", "steps": st64,
                              "warmup": sw64, "ms_per_step": t64 / st64, "kernel_ms": kt64,
                              "roofline": roofline(wl64, 8, kt64, peak, peak_kind), "clocks": c64}
        # batched against one at a time on the small serving grids (32 shots,
        # Nt scaled with the grid as in the serving mix)
        if not args.no_batching:
            from mittet_main_b200.benchmarks import batching_ratio
            rows = {}
            for g in (64, 96):
                bw = W.serving_case(g, g, g, 32, int(6000 * g / 256))
                rows[f"{g}^3x32"] = batching_ratio(bw, repeats=2)
            extras["batched_vs_one_at_a_time"] = {
                "value": rows["64^3x32"]["batched_vs_one_at_a_time"], "workload": "64^3, 32 shots, Nt 1500",
                "metric": "shot-solves/s batched / one shot at a time", "runs": rows}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            g, sample, thr = run_cpu_baseline(wl)
            cpu = {"value": g, "unit": "Gcell/s", "cores": thr, "kind": "port", "sample": sample}
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "Gcell/s", "cores": 0, "kind": "port", "sample": f"failed: {ex}"}

    if rank == 0:
        line = {
            "metric": "Gcell/s", "value": value, "unit": "Gcell/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if prec == FP32 else "f64",
            "data": "synthetic",
            "config": {"workload": wl.name, "nx": wl.cp.nx, "ny": wl.cp.ny, "nz": wl.cp.nz, "nt": wl.nt,
                       "shots_per_gpu": len(wl.shots), "receivers": nrec, "freqs": nf,
                       "volume_dft": wl.volume_dft or None, "fields": args.precision,
                       "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (fields > 126 MB)"},
            "shot_solves_per_s": len(wl.shots) * args.steps * world / (t_ms / 1e3),
            "gpu_launches": gpu_launches,
            "kernel_ms": kt,
            "stencil_variant": stencil_variant,
            "launch_path": launch_path,
            "roofline": roof,
            "clocks": clocks,
            "e2e": e2e,
            "cpu_baseline": cpu,
            **extras,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def timed_solves(solver, wl, steps, warmup, dist, dev, out, stream):
    """W untimed solves, then K solves bracketed by a barrier and a device
    synchronisation, timed with CUDA events on the launching stream (max over
    ranks).  Returns (ms for the K solves, kernel launches per solve, clocks)."""
    import torch
    for _ in range(warmup):
        solver.forward_device(wl.nt, out, stream)
    torch.cuda.synchronize()
    launches = solver.launch_count()
    sampler = ClockSampler(dev)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        solver.forward_device(wl.nt, out, stream)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    if dist:
        dist.barrier()
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=f"cuda:{dev}")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item()), launches, clocks


def roofline(wl, esz, kt, peak, peak_kind):
    """HBM roofline of the E phase (the largest kernel group): algorithmic
    bytes per launch over its CUDA-event time, against the measured copy
    bandwidth, with the DRAM reads per cell of the profiled E-phase kernels."""
    ebytes = stencil_bytes(wl, esz)
    achieved = ebytes / (kt["e_phase"] / 1e3) / 1e9
    cells = wl.ncell * len(wl.shots)
    alg_reads = stencil_read_bytes(wl, esz) / cells
    prof = e_phase_profile(esz, wl.volume_dft)
    r = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
         "kernel": "E phase (band_kernel / e_part_kernel parts / interior_tma_kernel)", "alg_bytes_per_launch": ebytes,
         "alg_read_bytes_per_cell": alg_reads, "peak_source": peak_kind, "traffic": None}
    if prof:
        r["read_bytes_per_cell"] = prof["read"]
        r["read_amplification"] = prof["read"] / alg_reads
        # DRAM writes of a kernel are partly flushed from L2 during later
        # kernels, so the algorithmic writes stand in for them
        r["traffic"] = prof["read"] * cells + (ebytes - stencil_read_bytes(wl, esz))
        r["traffic_source"] = prof["source"] + " (reads, per cell x cells) + algorithmic writes"
    return r


if __name__ == "__main__":
    main()
