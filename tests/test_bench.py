"""CPU tests of the benchmark script's contract pieces that need no GPU: the
roofline record it builds (algorithmic bytes, the DRAM reads per cell read
from the committed ncu summary, a traffic figure that cannot fall below the
algorithmic bytes), and its options parse."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_roofline_record():
    from mittet_main_b200 import workloads as W
    bench = load_bench()
    wl = W.plain_gpu(nt=64)
    r = bench.roofline(wl, 4, {"e_phase": 0.2}, 6537.3, "measured")
    alg = bench.stencil_bytes(wl, 4)
    assert r["alg_bytes_per_launch"] == alg
    assert abs(r["achieved"] - alg / 0.2e-3 / 1e9) < 1e-6 and abs(r["frac"] - r["achieved"] / 6537.3) < 1e-12
    # 6 fields + model word read per cell, plus the psi of the slab cells
    assert 28.0 < r["alg_read_bytes_per_cell"] < 32.0
    prof = bench.e_phase_profile(4, "xyz")
    if prof is None:
        assert r["traffic"] is None
    else:
        assert r["read_bytes_per_cell"] == prof["read"]
        assert r["traffic"] >= alg and r["read_amplification"] >= 1.0
    assert bench.e_phase_profile(8, "xyz") is None  # only FP32 was captured
    r64 = bench.roofline(wl, 8, {"e_phase": 0.3}, 6537.3, "measured")
    assert r64["traffic"] is None and r64["alg_bytes_per_launch"] == 2 * alg
