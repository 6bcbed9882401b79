"""ana / kal writers and output statements (host logic, no GPU)."""
import numpy as np
import pytest

from field_b200.output import OutputLine, output_requests, write_ana, write_kal
from field_b200.sfinput import parse_input


def _lines(F):
    return [OutputLine("sys", "noname", "free energy", f"{F:.7g}"),
            OutputLine("sys", "noname", "free energy density", "profile", np.array([0.0, 1.5, 2.25, 0.0])),
            OutputLine("mol", "pol", "theta", "3.5")]


def test_ana_blocks_and_profiles(tmp_path):
    p = str(tmp_path / "out.ana")
    write_ana(p, _lines(-1.25), first=True)
    write_ana(p, _lines(-2.5), first=False)
    text = open(p).read().splitlines()
    assert text[0] == "system delimiter" and text[1] == ""
    assert text[2] == "sys : noname : free energy : -1.25"
    assert text[3] == "sys : noname : free energy density : profile"
    # reals as SFbox's streams print them: scientific, accuracy - 1 decimals
    assert text[4:8] == ["0.00000000000e+00", "1.50000000000e+00", "2.25000000000e+00", "0.00000000000e+00"]
    assert text.count("system delimiter") == 3
    assert "sys : noname : free energy : -2.5" in text
    write_ana(p, _lines(-1.0), first=True, write_bounds=False, lattice_shape=(4,))
    text = open(p).read().splitlines()
    assert text[4:6] == ["1.50000000000e+00", "2.25000000000e+00"] and text[6] == "mol : pol : theta : 3.5"


def test_kal_header_once_then_rows(tmp_path):
    p = str(tmp_path / "out.kal")
    for i, F in enumerate([-1.0, -2.0, -3.0]):
        write_kal(p, _lines(F), first=(i == 0))
    rows = [r.split("\t") for r in open(p).read().splitlines()]
    assert rows[0] == ["sys : noname : free energy", "mol : pol : theta"]
    assert [r[0] for r in rows[1:]] == ["-1", "-2", "-3"] and all(len(r) == 2 for r in rows)


def test_output_requests():
    calc = parse_input("output : run.ana : type : ana\noutput : run.kal : type : kal\n"
                       "output : run.kal : append : true\n")[0]
    req = output_requests(calc)
    assert [(n, t) for n, t, _ in req] == [("run.ana", "ana"), ("run.kal", "kal")]
    with pytest.raises(ValueError):
        output_requests(parse_input("output : x.ave : type : ave\n")[0])
    assert output_requests(parse_input("output : x.prf : type : profiles\n")[0])[0][1] == "profiles"


class _OracleSystem:
    """The parts of field_b200.system.System that output_lines reads, served
    by the oracle on a flat 1D lattice (interior weights 1, boundaries 0)."""

    def __init__(self, spec):
        from oracle.oracle import Oracle
        self.o, self.spec = Oracle(spec), spec

    def residual(self, x):
        return self.o.residual(x)

    def thermo(self):
        return self.o.thermo()

    def lattice_weights(self):
        w = np.ones(self.o.M)
        w[0] = w[-1] = 0.0
        return w, w

    def mol_scalars(self, m):
        return {"lngn": self.o.lngn(m), "phibulk": self.o.phibulk(m), "lnc": 0.0}

    def phi(self, s):
        return self.o.phi(s)

    def swf(self, s):
        return self.o.swf(s)

    def mol_phi(self, m, s):
        return self.o.mol_phi(m, s)


def test_output_lines_keys_and_sums():
    """SFbox's keys in SFbox's order; theta sums over interior sites,
    segment theta excess = theta - sites * phibulk (SF_Segment.cpp:370-392),
    molecule theta excess over phi > 0 only (SF_Molecule.cpp:727-749)."""
    from field_b200 import configs
    from field_b200.output import output_lines
    from field_b200.sfinput import build_system
    n = 20
    calc = parse_input(configs.C1_INPUT.format(n=n, N=10, phib=0.01, chi_aw=0.5, chi_as=-1.0))[0]
    spec, st = build_system(calc)
    sys_ = _OracleSystem(spec)
    x, rc, it, err = sys_.o.solve_diis(np.zeros(spec.n_itvar()), tol=1e-9, maxit=3000, m=5, eta=0.1)
    assert rc == 0
    lines = output_lines(calc, spec, sys_, x, it, err, st.tolerance, st.iterationlimit, 1)
    d = {(l.cls, l.name, l.key): l for l in lines}
    assert [l.cls for l in lines][:2] == ["sys", "sys"]
    acc = int(-np.log10(st.tolerance) + 0.5)
    assert d[("sys", "noname", "free energy")].value == f"{sys_.o.thermo()[0]:.{acc - 1}e}"
    order = []
    for l in lines:
        if not order or order[-1] != l.cls:
            order.append(l.cls)
    assert order == ["sys", "lat", "mol", "chi list", "mon", "newton"]   # SFbox's class order
    assert float(d[("chi list", "A", "chi - W")].value) == 0.5
    assert float(d[("chi list", "A", "chi - S")].value) == -1.0
    phiA = sys_.o.phi(1)
    theta = phiA[1:-1].sum()
    assert float(d[("mon", "A", "theta")].value) == pytest.approx(theta, rel=1e-6)
    assert float(d[("mon", "A", "theta excess")].value) == pytest.approx(theta - n * 0.01, rel=1e-6)
    assert float(d[("mol", "pol", "theta")].value) == pytest.approx(theta, rel=1e-6)
    assert float(d[("mol", "pol", "n")].value) == pytest.approx(theta / 10, rel=1e-6)
    assert float(d[("mol", "pol", "phi-av")].value) == pytest.approx(theta / n, rel=1e-6)
    assert d[("mol", "pol", "composition")].value == "(A)10"
    assert d[("newton", "isaac", "iterations")].value == str(it)
    assert d[("mon", "S", "freedom")].value == "frozen" and ("mon", "S", "G") not in d
    mol_keys = [l.key for l in lines if l.cls == "mol" and l.name == "pol"]
    assert mol_keys[:8] == ["freedom", "phibulk", "log(phibulk)", "phi-av", "theta", "theta excess", "n", "n exc"]


def test_vtk_1d_and_2d_layout(tmp_path):
    """OutputVtkProfiles as SFbox writes it: 1D puts the selected profiles side
    by side for the layers 1..n-1 (0-based) under 'DIMENSIONS<n>'; 2D writes
    the template's first profile at (x, y-1), y outer, x inner."""
    from field_b200.output import write_vtk
    prof = np.arange(7, dtype=float)          # 1D, n = 5 interior layers
    lines = [OutputLine("mon", "A", "theta", "1"), OutputLine("mon", "A", "phi", "profile", prof)]
    p = str(tmp_path / "a.vtk")
    write_vtk(p, lines, (7,))
    text = open(p).read().splitlines()
    assert text[:4] == ["# vtk DataFile Version 3.0", "vtk output", "ASCII", "DATASET STRUCTURED_POINTS"]
    assert text[4] == "DIMENSIONS5" and text[7] == "POINT_DATA 5"
    assert text[8] == "SCALARS SFBox_profile double" and text[9] == "LOOKUP_TABLE default "
    assert text[10:] == [f"{v:.11e}" for v in (1.0, 2.0, 3.0, 4.0)]
    grid = np.arange(5 * 4, dtype=float).reshape(5, 4)   # nx = 3, ny = 2
    lines2 = [OutputLine("mon", "A", "phi", "profile", grid.ravel()),
              OutputLine("mon", "B", "phi", "profile", -grid.ravel())]
    p2 = str(tmp_path / "b.vtk")
    write_vtk(p2, lines2, (5, 4), template=[("mon", "B", "*")])
    t2 = open(p2).read().splitlines()
    assert t2[4] == "DIMENSIONS 3 2 1" and t2[7] == "POINT_DATA 6"
    vals = [float(v) for v in t2[10:]]
    want = [-grid[x, y - 1] for y in (1, 2) for x in (1, 2, 3)]
    assert vals == want
    with pytest.raises(ValueError):
        write_vtk(p2, lines2, (5, 4))


def test_numbered_filenames_and_sweep_values():
    from field_b200.output import numbered_filename
    from field_b200.sweep import expand_variation
    assert numbered_filename("run.vtk", 3, 12) == "run_03.vtk"
    assert numbered_filename("run.vtk", 1, 1) == "run.vtk"
    calc = parse_input("mon : A : chi - W : 0.2\nvar : mon : A : chi - W\nvar : mon : step : 0.2\n"
                       "var : mon : end_value : 0.8\nvar : mon : type : real\n")[0]
    var = expand_variation(calc)
    assert numbered_filename("run.vtk", 1, 1, var, 0.4) == "run_chi - W=0.40000e0.vtk"
    calc = parse_input("lat : l : n_layers : 20\nvar : lat : l : n_layers\nvar : lat : step : 5\n"
                       "var : lat : end_value : 40\nvar : lat : type : integer\n")[0]
    var = expand_variation(calc)
    assert numbered_filename("p.vtk", 2, 3, var, 25) == "p_2_n_layers=25.vtk"


def test_template_wildcards():
    from field_b200.output import in_template
    ln = OutputLine("mon", "A", "phi", "profile", np.zeros(3))
    assert in_template([("mon", "*", "phi")], ln)
    assert in_template([("m*", "A", "p*")], ln)
    assert not in_template([("mol", "*", "phi")], ln)


def test_profiles_layout(tmp_path):
    """OutputProfiles as SFbox writes it: a header of the coordinate names and
    'c : n : k' of each profile, then one row per site, every field followed
    by a tab; boundary sites only with write_bounds; in 2D a blank line after
    each x row and one more at the end; in 3D interior sites only."""
    from field_b200.output import write_profiles
    a, b = np.arange(5, dtype=float), -np.arange(5, dtype=float)
    lines = [OutputLine("sys", "noname", "free energy", "1"), OutputLine("mon", "A", "phi", "profile", a),
             OutputLine("mol", "m", "phi", "profile", b)]
    p = str(tmp_path / "p")
    write_profiles(p, lines, (5,))
    t = open(p).read().split("\n")
    assert t[0] == "layer\tmon : A : phi\tmol : m : phi\t"
    assert t[1] == f"0\t{0.0:.11e}\t{-0.0:.11e}\t" and t[5].startswith("4\t") and t[6] == ""
    write_profiles(p, lines, (5,), write_bounds=False, template=[("mol", "*", "*")])
    t = open(p).read().split("\n")
    assert t[0] == "layer\tmol : m : phi\t" and [r.split("\t")[0] for r in t[1:4]] == ["1", "2", "3"]
    g2 = np.arange(12, dtype=float)                     # (4, 3)
    write_profiles(p, [OutputLine("mon", "A", "phi", "profile", g2)], (4, 3), write_bounds=False)
    t = open(p).read().split("\n")
    assert t[0] == "layer x\tlayer y\tmon : A : phi\t"
    # interior (1, 1) and (2, 1); each of the four x rows closed by a blank
    # line, one more at the end
    assert t[1:] == ["", f"1\t1\t{4.0:.11e}\t", "", f"2\t1\t{7.0:.11e}\t", "", "", "", ""]
    g3 = np.arange(27, dtype=float)                     # (3, 3, 3): one interior site
    write_profiles(p, [OutputLine("mon", "A", "phi", "profile", g3)], (3, 3, 3))
    t = open(p).read().split("\n")
    assert t == ["layer x\tlayer y\tlayer z\tmon : A : phi\t", f"1\t1\t1\t{13.0:.11e}\t", ""]
