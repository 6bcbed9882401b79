"""Writes tests/golden/oracle_cases.npz: for a set of the seeded parity
systems, the iteration variables x, and the oracle's residual, segment
profiles, lnGN per molecule and free energy at x.

SFbox itself cannot be built here (its container library fenk is not
available), so these fixtures come from the oracle; they pin the oracle
against later edits and give the GPU tests fixed numbers to meet.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cases import CASES, random_x  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

GOLDEN_CASES = ["1d_surface", "1d_periodic_restricted", "1d_sphere_colloid", "2d_cylinder", "2d_flat_surface",
                "3d_mirror_mix", "3d_2nd_brush", "1d_2nd_lumped", "2d_cyl_2nd_lumped", "3d_fcc_colloid",
                "3d_hex_mirror", "1d_dendrimer"]
SEED = 20261203


def golden_arrays():
    out = {}
    for k in GOLDEN_CASES:
        spec = CASES[k]()
        o = Oracle(spec)
        x = random_x(spec, seed=SEED, scale=0.2)
        f = o.residual(x)
        out[f"{k}/x"] = x
        out[f"{k}/f"] = f
        out[f"{k}/phi"] = np.stack([o.phi(i) for i in range(len(spec.segments))])
        out[f"{k}/lngn"] = np.array([o.lngn(m) for m in range(len(spec.molecules))])
        out[f"{k}/F"] = np.array([o.free_energy()])
    return out


if __name__ == "__main__":
    np.savez_compressed(os.path.join(HERE, "oracle_cases.npz"), **golden_arrays())
    print("wrote", os.path.join(HERE, "oracle_cases.npz"))
