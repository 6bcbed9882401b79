"""The N > 1 path on CPU: two gloo ranks split uneven instances by cost,
solve their shares (with the CPU oracle standing in for the device solve),
gather the results and aggregate timing (max) and counts (sum) the way
bench.py does under torchrun.  The union of the ranks' results must equal a
single-rank run, instance by instance."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

SWEEP = dict(count=12, n_range=(20, 60), N_range=(5, 60))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _solve_one(spec, x0):
    from oracle.oracle import Oracle
    o = Oracle(spec)
    x, rc, it, err = o.solve_diis(x0, tol=1e-9, maxit=3000, m=5, eta=0.1)
    return {"x": x, "rc": rc, "it": it}


def _worker(rank, world, port, out):
    import time

    import torch.distributed as dist
    from field_b200 import configs
    from field_b200.shard import aggregate, estimate_cost, gather_results, partition
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        inst = configs.sweep1d(**SWEEP)
        parts = partition([estimate_cost(s) for s, _ in inst], world)
        t0 = time.perf_counter()
        local = {i: _solve_one(*inst[i]) for i in parts[rank]}
        elapsed = time.perf_counter() - t0
        results = gather_results(local, world)
        t, n = aggregate(elapsed, sum(1 for r in local.values() if r["rc"] == 0), world)
        out.put((rank, parts, results, t, n, elapsed))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_solve_disjoint_shares_and_match_one_rank():
    from field_b200 import configs
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in procs], key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, parts0, res0, t0, n0, e0), (_, parts1, res1, t1, n1, e1) = res
    assert parts0 == parts1
    assert not set(parts0[0]) & set(parts0[1])
    assert sorted(parts0[0] + parts0[1]) == list(range(SWEEP["count"]))
    assert t0 == t1 == max(e0, e1)                      # max over ranks
    single = {i: _solve_one(s, x) for i, (s, x) in enumerate(configs.sweep1d(**SWEEP))}
    assert n0 == n1 == sum(1 for r in single.values() if r["rc"] == 0)
    for r in (res0, res1):                              # both ranks hold the union
        assert sorted(r) == sorted(single)
        for i in single:
            assert r[i]["rc"] == single[i]["rc"] and r[i]["it"] == single[i]["it"]
            np.testing.assert_array_equal(r[i]["x"], single[i]["x"])


@pytest.mark.parametrize("world", [2, 4, 8])
def test_cost_partition_balances_the_c4_sweep(world):
    """The 256 uneven C4 instances (N 20..1000, M 52..402) split within 2 %
    of perfect balance by estimated cost; an equal-count split is far off."""
    from field_b200 import configs
    from field_b200.shard import estimate_cost, load_imbalance, partition
    costs = [estimate_cost(s) for s, _ in configs.sweep1d(count=256)]
    parts = partition(costs, world)
    assert sorted(i for p in parts for i in p) == list(range(256))
    assert load_imbalance(costs, parts) < 1.02
    naive = [list(range(r, 256, world)) for r in range(world)]
    assert load_imbalance(costs, naive) > load_imbalance(costs, parts)


def test_seed_capacity_guard():
    from field_b200.shard import instance_seeds
    with pytest.raises(ValueError):
        instance_seeds(0, 5000, 0)
