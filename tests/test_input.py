"""SFbox input-file reader and system builder (host logic, no GPU)."""
import numpy as np
import pytest

from field_b200 import configs
from field_b200.desc import BOUND_MIRROR1, BOUND_SURFACE, MOL_FREE, MOL_SOLVENT, SEG_FROZEN
from field_b200.sfinput import build_system, parse_composition, parse_input


def test_parse_c1_input():
    text = configs.C1_INPUT.format(n=100, N=100, phib=0.01, chi_aw=0.5, chi_as=-1.0)
    calcs = parse_input(text)
    assert len(calcs) == 1
    spec, st = build_system(calcs[0])
    assert spec.lattice.M == 102
    assert spec.lattice.bound_lo[0] == BOUND_SURFACE and spec.lattice.bound_hi[0] == BOUND_MIRROR1
    assert [s.name for s in spec.segments] == ["S", "A", "W"]
    assert spec.segments[0].freedom == SEG_FROZEN and spec.segments[0].range[0] == 1.0
    assert spec.segments[0].range[1:].sum() == 0
    assert spec.chi[1, 2] == 0.5 and spec.chi[2, 1] == 0.5 and spec.chi[0, 1] == -1.0
    assert spec.molecules[0].N == 100 and spec.molecules[0].freedom == MOL_FREE
    assert spec.molecules[1].freedom == MOL_SOLVENT
    assert spec.n_itvar() == 200
    assert st.tolerance == 1e-7 and st.method == "Pure_DIIS"


def test_start_blocks_inherit_and_override():
    text = """lat : l : gradients : 1
lat : l : n_layers : 10
lat : l : lambda : 0.2
mon : A : freedom : free
mon : W : freedom : free
mol : p : composition : (A)5
mol : p : freedom : free
mol : p : phibulk : 0.1
mol : w : composition : (W)1
mol : w : freedom : solvent
start
mol : p : phibulk : 0.2   // second calculation changes one value
start
"""
    calcs = parse_input(text)
    assert len(calcs) == 2
    s1, _ = build_system(calcs[0])
    s2, _ = build_system(calcs[1])
    assert s1.molecules[0].phibulk == 0.1 and s2.molecules[0].phibulk == 0.2
    assert s2.lattice.n_layers[0] == 10


def test_malformed_lines_rejected():
    with pytest.raises(ValueError):
        parse_input("lat : a : gradients\n")
    with pytest.raises(ValueError):
        parse_input("lat : a : b : c : d\n")


def test_composition():
    assert parse_composition("(A)20(B)20") == [("A", 20), ("B", 20)]
    assert parse_composition("(X)1(A)199") == [("X", 1), ("A", 199)]
    with pytest.raises(ValueError):
        parse_composition("A20")


def test_class_layout_groups_equal_chemistry():
    spec, _ = configs.cyl_micelle(nx=8, ny=8)
    cls, nc = spec.class_layout()
    assert nc == 3 and sorted(cls) == [0, 1, 2]
    # B and W equal when chi_BW equals chi_AW... here B has chi 0 with all, W does not
    spec2, _ = configs.melt3d(n=4, nA=2, nB=2, chi_ab=0.0)
    cls2, nc2 = spec2.class_layout()
    assert nc2 == 1 and cls2 == [0, 0]


def test_synthetic_configs_shapes():
    spec, x = configs.cyl_micelle()
    assert spec.lattice.shape == (130, 130) and x.size == spec.n_itvar() == 128 * 128 * 3
    spec, x = configs.melt3d(n=16)
    assert x.size == 16 ** 3 * 2 and np.all(np.abs(x) <= 0.05)
    inst = configs.sweep1d(count=8)
    assert len(inst) == 8 and all(50 <= s.lattice.n_layers[0] <= 400 for s, _ in inst)
    spec, x = configs.brush3d(n=12, N=20, sigma=0.05)
    assert spec.segments[0].range.sum() == round(0.05 * 144)


@pytest.mark.parametrize("geom,expect", [("spherical", (3 * 20.0 / (4 * np.pi)) ** (1 / 3)),
                                         ("cylindrical", np.sqrt(20.0 / np.pi))])
def test_curved_one_gradient_lattice(geom, expect):
    """One-gradient curved lattices read offset_first_layer (no _x) and
    n_sites_first_layer, which sets the layer adjustment of the first layer
    (Lat1DCylinder.cpp:43-52, Lat1DSphere.cpp:6-12)."""
    from field_b200.desc import GEOM_CYLINDRICAL, GEOM_SPHERICAL
    text = f"""lat : l : gradients : 1
lat : l : geometry : {geom}
lat : l : n_layers : 30
lat : l : lowerbound : mirror1
lat : l : n_sites_first_layer : 20
mon : A : freedom : free
mon : W : freedom : free
mol : p : composition : (A)5
mol : p : freedom : free
mol : p : phibulk : 0.1
mol : w : composition : (W)1
mol : w : freedom : solvent
"""
    spec, _ = build_system(parse_input(text)[0])
    lat = spec.lattice
    assert lat.geometry == (GEOM_SPHERICAL if geom == "spherical" else GEOM_CYLINDRICAL)
    assert lat.layer_adjustment == pytest.approx(expect)
    text2 = text.replace("lat : l : n_sites_first_layer : 20\n", "lat : l : offset_first_layer : 2.5\n")
    spec2, _ = build_system(parse_input(text2)[0])
    assert spec2.lattice.offset_first_layer == 2.5 and spec2.lattice.layer_adjustment == 1.0


def test_overflow_protection_statement():
    """sys : overflow_protection : true selects the log-space lattices; 3D and
    second-order systems reject it as SFbox does (SF_System.cpp:395, :478-481)."""
    from field_b200 import configs
    base = configs.C1_INPUT.format(n=20, N=10, phib=0.01, chi_aw=0.5, chi_as=-1.0).replace("start\n", "")
    spec, _ = build_system(parse_input(base + "sys : noname : overflow_protection : true\nstart\n")[0])
    assert spec.overflow_protection
    spec, _ = build_system(parse_input(base + "start\n")[0])
    assert not spec.overflow_protection
    with pytest.raises(ValueError):
        build_system(parse_input(base + "sys : noname : overflow_protection : maybe\nstart\n")[0])
    with pytest.raises(ValueError):
        build_system(parse_input(base + "sys : noname : overflow_protection : true\n"
                                 "sys : noname : matrix_approach : second_order\nstart\n")[0])


@pytest.mark.parametrize("extra", ["mol : pol : ring : maybe\n", "mon : A : valence : 1\n",
                                   "mon : A : state1 : Ap\n", "reaction : r1 : equation : 2(A)=(B)\n",
                                   "lat : flat : n_layers_extended : 40\n"])
def test_unbuilt_physics_is_refused(extra):
    """Statements that change the physics but are not built are refused by
    name, not ignored."""
    from field_b200 import configs
    base = configs.C1_INPUT.format(n=20, N=10, phib=0.01, chi_aw=0.5, chi_as=-1.0).replace("start\n", "")
    with pytest.raises(ValueError):
        build_system(parse_input(base + extra + "start\n")[0])
    # statements without effect on this path are accepted
    build_system(parse_input(base + "mol : pol : save_memory : true\nmon : A : valence : 0\nstart\n")[0])


def test_branched_compositions_as_bond_trees():
    """SF_ParserBranched's rules (SF_ParserBranched.h:20-45): fragments between
    square brackets, ranks, and every fragment's first segment bonded to the
    last segment of the nearest preceding fragment of lower or equal rank."""
    from field_b200.sfinput import parse_branched, parse_comb
    assert parse_branched("(A)20(B)20") is None
    blocks, parent = parse_branched("(A)3[(B)2](A)3")
    assert blocks == [("A", 3), ("B", 2), ("A", 3)]
    assert parent == [-1, 0, 1, 2, 3, 2, 5, 6]
    # two side fragments at one point ('][')
    _, parent = parse_branched("(A)3[(B)2][(C)2](A)3")
    assert parent == [-1, 0, 1, 2, 3, 2, 5, 2, 7, 8]
    # a branch inside a side fragment: (C) hangs from the end of (B)
    _, parent = parse_branched("(A)2[(B)2[(C)1](B)1](A)1")
    assert parent == [-1, 0, 1, 2, 3, 3, 1]
    # repeated branched groups expand first (ExpandBrackets)
    blocks, parent = parse_branched("((A)2[(B)1])2(A)1")
    assert blocks == [("A", 2), ("B", 1), ("A", 2), ("B", 1), ("A", 1)]
    assert parent == [-1, 0, 1, 1, 3, 4, 4]
    for bad in ("(A)3[[(B)2]](A)3", "(A)3[(B)2](A)3]", "(A)1[(B)2](A)3", "(A)3[](A)3"):
        with pytest.raises(ValueError):
            parse_branched(bad)
    # comb: Main1-(Spacer-[Side])NA-Main2
    blocks, parent = parse_comb("@dend(2. (A)2, (A)1, (B)2, (A)1)")
    assert blocks == [("A", 2), ("A", 1), ("B", 2), ("A", 1), ("B", 2), ("A", 1)]
    assert parent == [-1, 0, 1, 2, 3, 2, 5, 6, 5]
    assert parse_comb("@dend(2, (A)3, 3, (B)2, 2)") is None
    # asymmetric dendrimer: core = the shared first segment of generation 1,
    # every arm end carries the next generation's pair of arms
    from field_b200.sfinput import parse_asym_dendrimer
    blocks, parent = parse_asym_dendrimer("@dend(2; (C)1(A)2, (C)1(A)1, (D)1(B)1, (D)1(B)2)")
    assert sum(n for _, n in blocks) == 12
    assert parent == [-1, 0, 1, 0, 2, 4, 4, 6, 3, 8, 8, 10]
    with pytest.raises(ValueError):
        parse_asym_dendrimer("@dend(2; (A)3, (A)2, (B)2, (A)2)")   # generation 2's fragments start differently
    assert parse_asym_dendrimer("@dend(2, (A)3, 3, (B)2, 2)") is None


def test_rings_and_branched_molecules_in_input_files():
    from field_b200 import configs
    base = configs.C1_INPUT.format(n=20, N=10, phib=0.01, chi_aw=0.5, chi_as=-1.0).replace("start\n", "")
    spec, _ = build_system(parse_input(base + "mol : pol : ring : true\nstart\n")[0])
    assert spec.molecules[0].ring and spec.molecules[0].bond_parent is None
    odd = configs.C1_INPUT.format(n=20, N=11, phib=0.01, chi_aw=0.5, chi_as=-1.0).replace("start\n", "")
    with pytest.raises(ValueError):
        build_system(parse_input(odd + "mol : pol : ring : true\nstart\n")[0])
    text = base.replace("composition : (A)10", "composition : (A)4[(A)2](A)4") + "start\n"
    spec, _ = build_system(parse_input(text)[0])
    assert spec.molecules[0].N == 10 and spec.molecules[0].bond_parent == [-1, 0, 1, 2, 3, 4, 3, 6, 7, 8]
