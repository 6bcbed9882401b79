"""The N > 1 path on CPU: two gloo ranks build disjoint instance sets, solve
nothing on the GPU, and aggregate timing (max) and counts (sum) the way
bench.py does under torchrun."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from field_b200 import configs
    from field_b200.shard import aggregate, instance_seeds
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        seeds = instance_seeds(rank, 3, configs.BASE_SEED)
        # a host-side stand-in for the timed solve: rank r "takes" 1 + r seconds, solves 3 + r
        t, n = aggregate(1.0 + rank, 3 + rank, world)
        out.put((rank, seeds, t, n))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_aggregate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (r0, s0, t0, n0), (r1, s1, t1, n1) = res
    assert not set(s0) & set(s1)               # disjoint instances
    assert t0 == t1 == 2.0                      # max over ranks
    assert n0 == n1 == 7.0                      # total solves


def test_seed_capacity_guard():
    from field_b200.shard import instance_seeds
    with pytest.raises(ValueError):
        instance_seeds(0, 5000, 0)
