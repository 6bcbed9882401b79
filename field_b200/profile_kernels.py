"""Time the propagator kernels of one system with CUDA events, for roofline
figures and as a small, self-contained target for ncu captures.

    python -m field_b200.profile_kernels --case c3 --reps 50

Cases: c2 (Lat2DCyl1stO 128x128, A20B20), c3 (Lat3D1stO 128^3, A50B50),
c5 (Lat3D2ndO 96^3 brush, N=200; --n to shrink).  Prints one JSON line with
the average device time and algorithmic bytes of a forward step and of a
backward step with fused composition, and the achieved GB/s.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import configs
from .batch import measured_peaks
from .system import System


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="c3", choices=["c2", "c3", "c5"])
    ap.add_argument("--reps", type=int, default=50)
    ap.add_argument("--n", type=int, default=0, help="lattice size override")
    ap.add_argument("--tile", type=int, default=0, help="3D x-chunk depth (0: autotune)")
    ap.add_argument("--form", default="pipelined", choices=["pipelined", "plain", "pipelined2"],
                    help="3D first-order step form when --tile is given")
    a = ap.parse_args()
    if a.case == "c2":
        spec, x = configs.cyl_micelle(**({"nx": a.n, "ny": a.n} if a.n else {}))
    elif a.case == "c3":
        spec, x = configs.melt3d(**({"n": a.n} if a.n else {}))
    else:
        spec, x = configs.brush3d(**({"n": a.n} if a.n else {}))
    s = System(spec)
    s.residual(x)
    tune = None
    if a.tile:
        s.set_tile(a.tile)
        s.set_tile_pipelined({"plain": 0, "pipelined": 1, "pipelined2": 2}[a.form])
    else:
        tune = s.autotune(reps=max(5, a.reps // 5))
    p = s.profile_propagator(reps=a.reps)
    peak, kind = measured_peaks()
    out = {"case": a.case, "M": s.M, "K": s.K, "reps": a.reps, "tile": a.tile or tune,
           "form": a.form if a.tile else "autotuned", **p,
           "gbs_fwd": p["bytes_fwd"] / (p["ms_fwd"] / 1e3) / 1e9,
           "gbs_bwd": p["bytes_bwd"] / (p["ms_bwd"] / 1e3) / 1e9, "peak_gbs": peak, "peak_kind": kind}
    out["frac_fwd"] = out["gbs_fwd"] / peak
    out["frac_bwd"] = out["gbs_bwd"] / peak
    print(json.dumps(out))


if __name__ == "__main__":
    main()
