"""``python -m field_b200 input.in``: an SFbox input with a sweep and ana/kal
outputs, run end to end on the GPU."""
import os
import subprocess
import sys

import numpy as np
import pytest

from field_b200 import configs
from field_b200.sfinput import build_system, parse_input
from field_b200.sweep import sweep_calculations
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

INPUT = (configs.C1_INPUT.format(n=30, N=15, phib=0.01, chi_aw=0.2, chi_as=-1.0).replace("start\n", "").replace("tolerance : 1e-7", "tolerance : 1e-9")
         + "var : mon : A : chi - W\nvar : mon : step : 0.2\nvar : mon : end_value : 0.8\nvar : mon : type : real\n"
         + "newton : isaac : m : 8\n"
         + "output : run.ana : type : ana\noutput : run.kal : type : kal\n"
         + "output : run.vtk : type : vtk\noutput : run.vtk : template : tmpl.in\nstart\n")


def test_cli_sweep_writes_ana_and_kal(gpu_lib, tmp_path):
    inp = tmp_path / "sweep.in"
    inp.write_text(INPUT)
    (tmp_path / "tmpl.in").write_text("mon : A : phi : profile\n")
    r = subprocess.run([sys.executable, "-m", "field_b200", str(inp)], capture_output=True, text=True,
                       timeout=600, cwd=os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    assert r.returncode == 0, r.stdout + r.stderr
    # one calculation swept over chi - W = 0.2, 0.4, 0.6, 0.8
    rows = [l.split("\t") for l in (tmp_path / "run.kal").read_text().splitlines()]
    hdr = rows[0]
    assert len(rows) == 1 + 4
    ichi = hdr.index("chi list : A : chi - W")
    assert [float(r[ichi]) for r in rows[1:]] == pytest.approx([0.2, 0.4, 0.6, 0.8])
    iF = hdr.index("sys : noname : free energy")
    iO = hdr.index("sys : noname : grand potential")
    calcs = sweep_calculations(parse_input(INPUT)[0])[1]
    for row, calc in zip(rows[1:], calcs):
        spec, st = build_system(calc)
        o = Oracle(spec)
        x, rc, it, err = o.solve_diis(np.zeros(spec.n_itvar()), tol=1e-10, maxit=5000, m=8, eta=0.1)
        assert rc == 0
        o.residual(x)
        F, Om, _, _ = o.thermo()
        assert float(row[iF]) == pytest.approx(F, rel=1e-6, abs=1e-8)
        assert float(row[iO]) == pytest.approx(Om, rel=1e-6, abs=1e-8)
    # one vtk file per sweep point, named by the varied value; the A profile
    # of layers 1..n-1 (0-based)
    for v in ("0.20000e0", "0.40000e0", "0.60000e0", "0.80000e0"):
        vt = (tmp_path / f"run_chi - W={v}.vtk").read_text().splitlines()
        assert vt[4] == "DIMENSIONS30" and len(vt) == 10 + 29
    ana = (tmp_path / "run.ana").read_text().splitlines()
    assert ana.count("system delimiter") == 1 + 4
    assert sum(l.startswith("mon : A : phi : profile") for l in ana) == 4
