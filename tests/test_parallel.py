"""CPU, world_size 2 (gloo): shot sharding and the gradient all-reduce of the
multi-GPU path, with a deterministic stand-in for the per-shot solve."""
import os
import socket

import numpy as np
import pytest

from mittet_main_b200.parallel import distributed_gradient, shard_shots


def test_shard_shots_partitions_every_shot_once():
    for nshot in (1, 5, 16, 64):
        for world in (1, 2, 3, 8):
            parts = [shard_shots(nshot, r, world) for r in range(world)]
            flat = [s for p in parts for s in p]
            assert flat == list(range(nshot))
            assert max(map(len, parts)) - min(map(len, parts)) <= 1


def fake_shot(s):
    rng = np.random.default_rng(100 + s)
    return float(s + 1), rng.normal(size=(4, 5, 6))


def local(shots):
    mis, g = 0.0, np.zeros((4, 5, 6))
    for s in shots:
        m, gs = fake_shot(s)
        mis += m
        g += gs
    return mis, g


def _worker(rank, world, port, nshot, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mis, g = distributed_gradient(local, nshot)
        q.put((rank, mis, g))
    finally:
        dist.destroy_process_group()


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("nshot", [5, 16])
def test_distributed_gradient_equals_serial_sum(nshot):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, nshot, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    mis0, g0 = local(range(nshot))
    for _, mis, g in res:
        assert mis == pytest.approx(mis0, rel=1e-15)
        np.testing.assert_allclose(g, g0, rtol=1e-14, atol=1e-14)
