"""CPU tests of the benchmark script's contract pieces that need no GPU: the
DRAM traffic it reports for the roofline is read from the committed ncu
summary, and its options parse."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_roofline_traffic_comes_from_the_committed_profile():
    from mittet_main_b200 import workloads as W
    bench = load_bench()
    wl = W.plain_gpu(nt=64)
    t = bench.e_phase_traffic(wl, 4)
    # 40.1 B per cell in the summary, for the 256 x 256 x 192 launch
    assert t is not None and 30 * wl.ncell < t < 60 * wl.ncell
    assert bench.e_phase_traffic(wl, 8) is None  # only FP32 was captured
