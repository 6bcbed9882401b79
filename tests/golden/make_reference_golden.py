"""Writes tests/golden/reference_cases.npz from SFbox 2.1 itself: the
reference's own C++ sources built by oracle/refbuild (make -C oracle/refbuild),
driven by oracle/_ref/sfref on the input files of reference_inputs.py.

For every case:
  <case>/x       seeded iteration variables (normal, sd 0.3)
  <case>/g       SF_Solve::residuals at x (SF_Solve.cpp:647-651)
  <case>/phi     state volume fractions at x, one row per segment in the
                 input reader's segment order
  <case>/lngn    SF_Molecule::GetLnGN per molecule, input order
  <case>/F       SF_MoleculeList::GetFreeEnergy
  <case>/Omega   SF_MoleculeList::GetGrandPotential
and for the cases of SOLVE_CASES, SFbox's Pure_DIIS (SF_Solve::Iterate,
tolerance 1e-12) from the seeded start x0 (normal, sd 0.1):
  <case>/solve_x0, solve_x, solve_phi, solve_F, solve_Omega, solve_g
and for NEWTON_CASES, SFbox's Newton iteration (newton : method pseudohessian,
its default, and hessian; tolerance 1e-12) from x = 0:
  <case>/newton_<method>_x, _phi, _F, _iterations

    python tests/golden/make_reference_golden.py
"""
import os
import subprocess
import sys
import tempfile
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)

from reference_inputs import INPUTS  # noqa: E402
from field_b200.sfinput import build_system, parse_input  # noqa: E402

SFREF = os.path.join(ROOT, "oracle", "_ref", "sfref")
OUT = os.path.join(HERE, "reference_cases.npz")

SOLVE_CASES = ["1d_flat_surface", "1d_flat_c1", "1d_flat_mirror2", "1d_flat_periodic", "2d_cylinder",
               "2d_cylinder_core", "2d_flat_surface", "3d_periodic_melt", "3d_mirror_colloid", "3d_2nd_brush",
               "3d_fcc_colloid", "3d_hex_colloid", "3d_stencils_colloid", "1d_cylinder", "1d_sphere_colloid",
               "1d_2nd_lumped", "2d_2nd_lumped", "1d_cyl_2nd", "1d_sphere_2nd", "2d_cyl_2nd", "1d_flat_overflow",
               "2d_cyl_overflow", "1d_dendrimer", "1d_force", "3d_2nd_stiff_range", "3d_2nd_palindrome",
               "1d_branched", "1d_branched_restricted", "2d_branched", "3d_branched", "1d_comb", "1d_ring",
               "1d_asym_dendrimer", "1d_comb_branched_side", "1d_charged", "1d_charged_eps",
               "1d_cyl_charged", "1d_sphere_charged", "2d_flat_charged", "2d_flat_charged_walls", "2d_cyl_charged",
               "2d_cyl_charged_axis", "3d_charged_colloid", "1d_2nd_charged", "3d_2nd_charged",
               "1d_charged_overflow"]


NEWTON_CASES = ["1d_flat_c1", "1d_flat_surface", "1d_sphere_colloid", "2d_cylinder_core", "2d_flat_surface",
                "1d_dendrimer", "1d_2nd_lumped", "1d_force", "1d_charged"]
NEWTON_METHODS = ["pseudohessian", "hessian"]


def newton_input(text, method):
    """The case's input file with its newton method replaced."""
    return text.replace("newton : isaac : method : Pure_DIIS", f"newton : isaac : method : {method}")


def case_seed(name):
    return 20261203 + zlib.crc32(name.encode()) % 100000


def read_dump(path):
    out = {}
    with open(path) as f:
        for line in f:
            p = line.split()
            out[p[0]] = np.array([float(v) for v in p[2:]])
    return out


def run_sfref(mode, text, x, workdir, tag):
    inp = os.path.join(workdir, tag + ".in")
    with open(inp, "w") as f:
        f.write(text)
    xf = "-"
    if x is not None:
        xf = os.path.join(workdir, tag + ".x")
        np.asarray(x, dtype="<f8").tofile(xf)
    out = os.path.join(workdir, tag + ".out")
    r = subprocess.run([SFREF, mode, inp, xf, out], capture_output=True, text=True, cwd=workdir)
    if r.returncode != 0:
        raise RuntimeError(f"sfref {mode} {tag} failed ({r.returncode}):\n{r.stdout[-1500:]}\n{r.stderr[-1500:]}")
    d = read_dump(out)
    # Pure_DIIS reports its iterations only on the console ("i = <k> |g| = ...")
    its = [int(ln.split()[2]) for ln in r.stdout.splitlines() if ln.startswith("i = ")]
    if its:
        d["diis_iterations"] = np.array([float(its[-1])])
    return d


def state_rows(spec, dump, prefix=""):
    return np.stack([dump[f"state_{s.name}_phi"] for s in spec.segments])


def reference_arrays():
    data = {}
    with tempfile.TemporaryDirectory() as wd:
        for name, text in INPUTS.items():
            spec, _ = build_system(parse_input(text)[0])
            rng = np.random.default_rng(case_seed(name))
            x = rng.normal(0.0, 0.3, spec.n_itvar())
            d = run_sfref("eval", text, x, wd, name)
            assert int(d["nvar"][0]) == x.size, name
            data[f"{name}/x"] = x
            data[f"{name}/g"] = d["g"]
            data[f"{name}/phi"] = state_rows(spec, d)
            data[f"{name}/lngn"] = np.array([d[f"mol_{m.name}_lngn"][0] for m in spec.molecules])
            data[f"{name}/F"] = d["F"]
            data[f"{name}/Omega"] = d["Omega"]
            if name in SOLVE_CASES:
                x0 = rng.normal(0.0, 0.1, spec.n_itvar())
                if spec.charged:
                    # a potential of 0.1 V is ~4 kT/e: from such a start SFbox's
                    # Pure_DIIS overflows on its first step, so charged systems
                    # start from x = 0
                    x0 = np.zeros(spec.n_itvar())
                s = run_sfref("solve", text, x0, wd, name + "_solve")
                assert np.isfinite(s["g"]).all() and np.linalg.norm(s["g"]) <= 1e-10, name
                data[f"{name}/solve_x0"] = x0
                data[f"{name}/solve_x"] = s["x"]
                data[f"{name}/solve_g"] = s["g"]
                data[f"{name}/solve_phi"] = state_rows(spec, s)
                data[f"{name}/solve_F"] = s["F"]
                data[f"{name}/solve_Omega"] = s["Omega"]
            if name in NEWTON_CASES:
                for meth in NEWTON_METHODS:
                    s = run_sfref("solve", newton_input(text, meth), np.zeros(spec.n_itvar()), wd,
                                  f"{name}_{meth}")
                    data[f"{name}/newton_{meth}_x"] = s["x"]
                    data[f"{name}/newton_{meth}_phi"] = state_rows(spec, s)
                    data[f"{name}/newton_{meth}_F"] = s["F"]
                    data[f"{name}/newton_{meth}_iterations"] = s["iterations"]
    return data


if __name__ == "__main__":
    if not os.path.exists(SFREF):
        sys.exit("build the reference first: make -C oracle/refbuild")
    np.savez_compressed(OUT, **reference_arrays())
    print("wrote", OUT)
