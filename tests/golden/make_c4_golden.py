"""Writes tests/golden/c4_reference.npz: the 256 uneven Lat1DFlat1stO
instances of the batching configuration (field_b200.configs.sweep1d_inputs:
layers 50..400, N 20..1000 log-uniform, chi_AW on a shuffled grid over
[0, 1], phibulk 1e-4..1e-1, chi_AS -2..0) solved by SFbox itself -- the
reference's own sources built by oracle/refbuild, driven by oracle/_ref/sfref
-- with Pure_DIIS (its defaults m = 5, deltamax 0.1; iteration limit 20000)
to |g| <= 1e-12 from x = 0.

  x        all instances' final iteration variables, concatenated
  offsets  start of each instance in x (count + 1 entries)
  gnorm    |g| at the final x (SFbox's Pure_DIIS stops at |g| <= tolerance)
  iterations  Pure_DIIS iterations taken
  F        free energy at the final x

    python tests/golden/make_c4_golden.py
"""
import multiprocessing as mp
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)

SFREF = os.path.join(ROOT, "oracle", "_ref", "sfref")
OUT = os.path.join(HERE, "c4_reference.npz")
COUNT = 256
TOL = 1e-12
MAXIT = 20000


def _solve(args):
    i, text = args
    sys.path.insert(0, HERE)
    from make_reference_golden import run_sfref
    with tempfile.TemporaryDirectory() as wd:
        d = run_sfref("solve", text, None, wd, f"c4_{i}")
    return i, d["x"], float(np.linalg.norm(d["g"])), float(d["F"][0]), int(d["diis_iterations"][0])


def main():
    from field_b200.configs import sweep1d_inputs
    texts = [t.replace("start\n", f"newton : isaac : iterationlimit : {MAXIT}\nstart\n")
             for t in sweep1d_inputs(count=COUNT, tolerance=TOL)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(os.cpu_count() or 1) as pool:
        res = sorted(pool.map(_solve, list(enumerate(texts))))
    xs = [r[1] for r in res]
    offsets = np.cumsum([0] + [len(x) for x in xs])
    np.savez_compressed(OUT, x=np.concatenate(xs), offsets=offsets, gnorm=np.array([r[2] for r in res]),
                        F=np.array([r[3] for r in res]), iterations=np.array([r[4] for r in res]))
    print("wrote", OUT, "converged", int(np.sum(np.array([r[2] for r in res]) <= TOL)), "of", COUNT)


if __name__ == "__main__":
    if not os.path.exists(SFREF):
        sys.exit("build the reference first: make -C oracle/refbuild")
    main()
