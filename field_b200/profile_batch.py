"""One launch of the persistent batched solver on a chosen number of
instances, as a small, self-contained target for ncu captures.

    python -m field_b200.profile_batch --case c2 --instances 16

Cases: c2 (Lat2DCyl1stO 128x128, A20B20 + W, seeded micelle starts,
Pure_DIIS m = 10) and c4 (the first instances of the uneven 1D sweep, from
x = 0, m = 5).  After one warm-up launch, times one launch with CUDA events
and prints one JSON line (device ms, instances converged, mean iterations).
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import configs
from .batch import BatchSolver
from .shard import instance_seeds


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="c2", choices=["c2", "c4"])
    ap.add_argument("--instances", type=int, default=16)
    ap.add_argument("--threads", type=int, default=0, help="threads per block (0: the library's default)")
    a = ap.parse_args()
    if a.case == "c2":
        insts = [configs.cyl_micelle(seed=sd) for sd in instance_seeds(0, a.instances, configs.BASE_SEED + 2)]
        m, maxit = 10, 2000
    else:
        insts = configs.sweep1d(count=256)[:a.instances]
        m, maxit = 5, 5000
    bs = BatchSolver([s for s, _ in insts], m=m, eta=0.1)
    if a.threads:
        bs.set_launch(a.threads, True)
    x = np.concatenate([x for _, x in insts])
    for _ in range(2):
        bs.load(x)
        bs.solve_resident(1e-7, maxit)
        r = bs.results()
    print(json.dumps({"case": a.case, "instances": a.instances, "kernel_ms": bs.kernel_ms(),
                      "converged": int(r.converged.sum()), "mean_iterations": float(np.mean(r.iterations))}))


if __name__ == "__main__":
    main()
