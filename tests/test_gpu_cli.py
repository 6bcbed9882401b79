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


SFBOX = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "sfbox")


def _read_profiles(path):
    rows = [l.split("\t") for l in open(path).read().splitlines() if l.strip()]
    head = [h for h in rows[0] if h]
    data = {}
    for r in rows[1:]:
        vals = [v for v in r if v != ""]
        ncoord = sum(h.startswith("layer") for h in head)
        key = tuple(int(v) for v in vals[:ncoord])
        data[key] = dict(zip(head[ncoord:], (float(v) for v in vals[ncoord:])))
    return head, data


@pytest.mark.skipif(not os.path.exists(SFBOX), reason="oracle/_ref/sfbox is built where the reference sources are")
@pytest.mark.parametrize("case", ["1d_flat_surface", "2d_flat_surface"])
def test_cli_profiles_file_meets_sfbox(gpu_lib, tmp_path, case):
    """The profiles file of `python -m field_b200` against the one SFbox
    itself writes for the same input: the same coordinates and, for every
    profile both write, the same values (both converged to 1e-12); SFbox
    also writes density profiles this library leaves out."""
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from reference_inputs import INPUTS
    text = INPUTS[case].replace("start\n", "output : prof : type : profiles\nstart\n")
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    ref.mkdir()
    (ours / "a.in").write_text(text)
    (ref / "a.in").write_text(text)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-m", "field_b200", str(ours / "a.in")], capture_output=True, text=True,
                       timeout=600, cwd=root)
    assert r.returncode == 0, r.stdout + r.stderr
    r2 = subprocess.run([SFBOX, "a.in"], capture_output=True, text=True, timeout=600, cwd=str(ref))
    assert r2.returncode == 0, r2.stdout[-2000:]
    h1, d1 = _read_profiles(ours / "prof")
    h2, d2 = _read_profiles(ref / "prof")
    assert set(d1) == set(d2)
    common = [h for h in h1 if h in h2 and not h.startswith("layer")]
    assert any(h.endswith(": phi") for h in common) and len(common) >= 4, common
    for h in common:
        a = np.array([d1[k][h] for k in sorted(d1)])
        b = np.array([d2[k][h] for k in sorted(d2)])
        assert np.max(np.abs(a - b)) <= 1e-8 * max(np.max(np.abs(b)), 1e-300) + 1e-11, h


def _read_ana(path):
    out = {}
    for l in open(path).read().splitlines():
        parts = l.split(" : ")
        if len(parts) == 4 and parts[3] != "profile":
            out[tuple(parts[:3])] = parts[3]
    return out


@pytest.mark.skipif(not os.path.exists(SFBOX), reason="oracle/_ref/sfbox is built where the reference sources are")
@pytest.mark.parametrize("case", ["1d_flat_surface", "2d_cylinder_core"])
def test_cli_ana_lines_meet_sfbox(gpu_lib, tmp_path, case):
    """Every scalar line this library writes to an ana file against the same
    line of the ana file SFbox itself writes for the input: the same key,
    the same text, or the same number to 1e-8 (both converged to 1e-12)."""
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from reference_inputs import INPUTS
    text = INPUTS[case].replace("start\n", "output : out.ana : type : ana\nstart\n")
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    ref.mkdir()
    (ours / "a.in").write_text(text)
    (ref / "a.in").write_text(text)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-m", "field_b200", str(ours / "a.in")], capture_output=True, text=True,
                       timeout=600, cwd=root)
    assert r.returncode == 0, r.stdout + r.stderr
    r2 = subprocess.run([SFBOX, "a.in"], capture_output=True, text=True, timeout=600, cwd=str(ref))
    assert r2.returncode == 0, r2.stdout[-2000:]
    a, b = _read_ana(ours / "out.ana"), _read_ana(ref / "out.ana")
    bad = []
    for k, v in a.items():
        if k not in b:
            bad.append((k, v, None))
            continue
        try:
            x, y = float(v), float(b[k])
            ok = abs(x - y) <= 1e-8 * max(abs(y), 1.0)
        except ValueError:
            ok = v == b[k]
        if not ok:
            bad.append((k, v, b[k]))
    assert not bad, bad
