"""GPU test of mittet_forward_noalloc, the entry point for callers that cannot
call cudaMalloc: serving code that must not stall its other streams on the
device-wide synchronisation cudaFree brings, and hosts whose device memory
belongs to another allocator.

Both entry points run the same stencil bodies with the same explicit fma
forms (the no-alloc one uses the general body on every cell, the regular one
the interior, face and edge bodies the autotuner picks, all of which give a
cell bit-identical results), the same source gains and the same f_to_d
kernel, so the spectra must be equal bit for bit, with an electric and with a
magnetic source, on two calls in a row (the second call finds the scratch
array full of the first call's state), and a call after the first must
allocate no device memory.  The file is named so pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from mittet_main_b200 import capi
from mittet_main_b200 import workloads as W
from mittet_main_b200.capi import FP32

pytestmark = pytest.mark.gpu


def _noalloc_call(lib, wl, sigma_d, wave_d, out_d):
    g = wl.cp.grid()
    p = wl.cp.phys()
    pts = [capi.PointSource(0, x, y, z, capi.COMP[c], k, a) for (x, y, z, c, k, a) in wl.shots[0].points]
    parr = (capi.PointSource * len(pts))(*pts)
    rs = [capi.Receiver(x, y, z, capi.COMP[c]) for (x, y, z, c) in wl.receivers]
    rarr = (capi.Receiver * len(rs))(*rs)
    om = np.ascontiguousarray(wl.omega, dtype=np.float64)
    rc = lib.mittet_forward_noalloc(ctypes.byref(g), ctypes.byref(p), ctypes.c_void_p(sigma_d.data_ptr()),
                                    len(pts), parr, wl.nt, ctypes.c_void_p(wave_d.data_ptr()), len(rs), rarr,
                                    om.size, om.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1,
                                    ctypes.c_void_p(out_d.data_ptr()), None)
    capi.check(rc)


@pytest.mark.parametrize("magnetic", [False, True])
def test_noalloc_forward_matches_regular_entry_point_twice(magnetic):
    import torch

    wl = W.small_case(n=(40, 36, 32), ncpml=8, nt=200, precision=FP32, magnetic=magnetic)
    with W.make_solver(wl) as s:
        ref, _ = s.forward(wl.nt)
    ref = ref[0]  # [nrec, nf]
    assert np.abs(ref).max() > 0

    lib = capi.load()
    dev = torch.device("cuda:0")
    sigma_d = torch.from_numpy(np.ascontiguousarray(wl.sigma, dtype=np.float64)).to(dev)
    wave_d = torch.from_numpy(np.ascontiguousarray(wl.wavelet, dtype=np.float64)).to(dev)
    outs = []
    free_after = []
    for _ in range(2):
        out_d = torch.zeros((len(wl.receivers), len(wl.omega), 2), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(0)[0]
        _noalloc_call(lib, wl, sigma_d, wave_d, out_d)
        torch.cuda.synchronize()
        free_after.append((free_before, torch.cuda.mem_get_info(0)[0]))
        o = out_d.cpu().numpy()
        outs.append(o[..., 0] + 1j * o[..., 1])
    for got in outs:
        assert np.array_equal(got, ref), f"max |diff| {np.abs(got - ref).max():.3e}"
    # the second call allocates nothing on the device
    assert free_after[1][1] == free_after[1][0]


def test_noalloc_rejects_a_solve_larger_than_its_array():
    import torch

    wl = W.small_case(n=(200, 200, 200), ncpml=8, nt=4, precision=FP32)
    lib = capi.load()
    dev = torch.device("cuda:0")
    sigma_d = torch.ones(1, dtype=torch.float64, device=dev)
    wave_d = torch.zeros(wl.nt + 1, dtype=torch.float64, device=dev)
    out_d = torch.zeros((len(wl.receivers), len(wl.omega), 2), dtype=torch.float64, device=dev)
    with pytest.raises(capi.MittetError) as e:
        _noalloc_call(lib, wl, sigma_d, wave_d, out_d)
    assert e.value.code == -1 and "scratch" in str(e.value)
