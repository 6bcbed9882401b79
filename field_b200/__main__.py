"""Command line: ``python -m field_b200 input.in [--outdir DIR] [--waves W]``.

Runs an SFbox input file the way ``sfbox input.in`` does for the SCF path
(SF_Box.cpp:98-177): every calculation of the file in order, the points of a
``var :`` sweep in order, each point started from the previous point's
result (``newton : initial_guess : previous_result``, the default), and
``ana`` / ``kal`` output files written after every point
(field_b200.output).  ``vtk`` and ``profiles`` files are written one per
calculation under numbered names.  Sweeps of first-order systems are solved as batched
instances (field_b200.sweep): ``--waves`` sets how many batched launches the
sweep is split into (default: one per point, SFbox's chain).  Solver: the
file's newton : method -- SFbox's Newton iteration (pseudohessian, the
default, or hessian) over the device residual, or Pure_DIIS on the device --
with its tolerance, iterationlimit, deltamax (and m for Pure_DIIS).  Newton
sweeps are solved point after point.  Exit status 0 when every point
converged, 1 otherwise.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m field_b200", description=__doc__.split("\n\n")[0])
    ap.add_argument("input")
    ap.add_argument("--outdir", default=None, help="directory for the output files (default: the input's)")
    ap.add_argument("--waves", type=int, default=0, help="batched launches per sweep (0: one per point)")
    a = ap.parse_args(argv)
    from .output import (numbered_filename, output_lines, output_requests, read_template, write_ana, write_kal,
                         write_profiles, write_vtk)
    from .desc import LATTICE_HEX
    from .sfinput import build_system, parse_input
    from .sweep import batchable, solve_sweep, sweep_calculations
    from .system import System

    with open(a.input) as f:
        text = f.read()
    outdir = a.outdir or os.path.dirname(os.path.abspath(a.input))
    os.makedirs(outdir, exist_ok=True)
    written = set()
    calc_number = 0
    x_prev = None
    all_ok = True
    calcs = parse_input(text)
    indir = os.path.dirname(os.path.abspath(a.input))
    for ci, calc in enumerate(calcs, start=1):
        var, points = sweep_calculations(calc)
        built = [build_system(p) for p in points]
        st = built[0][1]
        newton = st.method in ("pseudohessian", "hessian")
        if len(points) > 1 and not newton and all(batchable(s) for s, _ in built):
            waves = a.waves if a.waves > 0 else len(points)
            same = x_prev is not None and len(x_prev) == built[0][0].n_itvar()
            res = solve_sweep(calc, waves=waves, x0=x_prev if same else None, tol=st.tolerance,
                              maxit=st.iterationlimit, m=st.m, eta=st.deltamax)
            results = [(res.x[i], int(res.iterations[i]), int(res.status[i])) for i in range(len(points))]
        else:
            results = []
            x = x_prev
            for spec, _ in built:
                if x is None or len(x) != spec.n_itvar():
                    x = np.zeros(spec.n_itvar())
                if newton:
                    r = System(spec).solve_newton(x, tol=st.tolerance, maxit=st.iterationlimit,
                                                  pseudohessian=st.method == "pseudohessian", deltamax=st.deltamax)
                else:
                    r = System(spec).solve(x, tol=st.tolerance, maxit=st.iterationlimit, m=st.m, eta=st.deltamax)
                results.append((r.x, r.iterations, r.status))
                x = r.x
        for pi, ((spec, stp), (x, its, status), p) in enumerate(zip(built, results, points)):
            calc_number += 1
            all_ok &= status == 0
            sys_ = System(spec)
            err = float(np.linalg.norm(sys_.residual(x)))
            # SFbox's Pure_DIIS counts its iterations on the console only: the
            # newton iterations line of its output stays 0 (sfnewton.cpp:566-664)
            lines = output_lines(p, spec, sys_, x, its if newton else 0, err, stp.tolerance, stp.iterationlimit,
                                 calc_number)
            for name, kind, params in output_requests(p):
                path = os.path.join(outdir, name)
                first = path not in written
                if params.get("write", "true") == "false":
                    continue
                if kind == "ana":
                    write_ana(path, lines, first, params.get("write_bounds", "true") != "false",
                              spec.lattice.shape)
                elif kind == "kal":
                    write_kal(path, lines, first)
                else:
                    tmpl = params.get("template")
                    tmpl = read_template(os.path.join(indir, tmpl)) if tmpl else None
                    vpath = os.path.join(outdir, numbered_filename(name, ci, len(calcs), var,
                                                                   var.values[pi] if var else None))
                    if kind == "profiles":
                        write_profiles(vpath, lines, spec.lattice.shape, tmpl,
                                       params.get("write_bounds", "true") != "false",
                                       params.get("write_blank_lines", "true") != "false")
                    else:
                        write_vtk(vpath, lines, spec.lattice.shape, tmpl,
                                  spec.lattice.gradients == 3 and spec.lattice.lattice_type == LATTICE_HEX)
                written.add(path)
            print(f"calculation {calc_number}: {'converged' if status == 0 else 'NOT converged'} "
                  f"in {its} iterations, |f| = {err:.3g}", flush=True)
            x_prev = x
    return 0 if all_ok else 1


if __name__ == "__main__":
    sys.exit(main())
