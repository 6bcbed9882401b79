"""Symmetric dendrimers (SF_Dend1stO, @dend(G, T1, f1, ..., TG, fG)) in the
oracle (no GPU).  A dendrimer whose every functionality beyond the core is 1
is a linear chain, so its profiles must equal the plain chain's; a star and a
two-generation dendrimer keep the u = 0 bulk, lnGN = ln(sites), and the
restricted mass sum rule."""
import numpy as np
import pytest

from cases import random_x
from field_b200.desc import (BOUND_MIRROR1, BOUND_SURFACE, Lattice, Molecule, MOL_FREE, MOL_RESTRICTED,
                             MOL_SOLVENT, Segment, SEG_FROZEN, SystemSpec)
from field_b200.sfinput import build_system, parse_dendrimer, parse_input
from oracle.oracle import Oracle


def _system(mol, n=16, surface=True):
    lat = Lattice(1, [n, 0, 0], [BOUND_SURFACE if surface else BOUND_MIRROR1, 0, 0], [BOUND_MIRROR1, 0, 0],
                  lam=1 / 6)
    r = np.zeros(n + 2)
    r[0] = 1.0
    segs = [Segment("S", SEG_FROZEN, r) if surface else Segment("S"), Segment("A"), Segment("B"), Segment("W")]
    chi = np.zeros((4, 4))
    chi[0, 1] = chi[1, 0] = -1.0
    chi[1, 3] = chi[3, 1] = 0.6
    chi[2, 3] = chi[3, 2] = -0.2
    return SystemSpec(lat, segs, chi, [mol, Molecule("W", [(3, 1)], MOL_SOLVENT)])


@pytest.mark.parametrize("dend,linear", [
    (([(1, 10)], [(1, 1)]), [(1, 10)]),                        # @dend(1, (A)10, 1)
    (([(1, 6)], [(1, 2)]), [(1, 11)]),                         # two arms of 5 around a centre
    (([(1, 3), (2, 2)], [(1, 2), (1, 1)]), [(2, 2), (1, 5), (2, 2)]),   # @dend(2, (A)3, 2, (B)2, 1)
    (([(1, 4), (1, 3)], [(1, 2), (1, 1)]), [(1, 13)]),
])
def test_linear_dendrimers_equal_chains(dend, linear):
    blocks, gens = dend
    mol_d = Molecule("d", blocks, MOL_FREE, phibulk=0.02, generations=gens)
    mol_l = Molecule("d", linear, MOL_FREE, phibulk=0.02)
    assert mol_d.N == mol_l.N
    sd, sl = _system(mol_d), _system(mol_l)
    x = random_x(sd, seed=4, scale=0.3)
    od, ol = Oracle(sd), Oracle(sl)
    fd, fl = od.residual(x), ol.residual(x)
    assert np.max(np.abs(fd - fl)) < 1e-12
    for i in range(4):
        np.testing.assert_allclose(od.phi(i), ol.phi(i), rtol=1e-12, atol=1e-15)
    assert od.lngn(0) == pytest.approx(ol.lngn(0), rel=1e-13)


@pytest.mark.parametrize("text", ["@dend(1, (A)5, 3)", "@dend(2, (A)3, 3, (B)2(A)1, 2)"])
def test_dendrimer_bulk_and_mass(text):
    gens = parse_dendrimer(text)
    names = {"A": 1, "B": 2}
    blocks = [(names[a], n) for bl, _ in gens for a, n in bl]
    g = [(len(bl), f) for bl, f in gens]
    mol = Molecule("d", blocks, MOL_FREE, phibulk=0.05, generations=g)
    spec = _system(mol, surface=False)
    o = Oracle(spec)
    o.residual(np.zeros(spec.n_itvar()))
    sites = spec.itvar_sites()
    N = mol.N
    for seg in (1, 2):
        np.testing.assert_allclose(o.phi(seg)[sites], 0.05 * mol.count(seg) / N, rtol=1e-12)
    assert o.lngn(0) == pytest.approx(np.log(16), rel=1e-13)
    # restricted: sum over the lattice of the molecule's phi is theta
    mol_r = Molecule("d", blocks, MOL_RESTRICTED, theta=1.5, generations=g)
    spec_r = _system(mol_r)
    o_r = Oracle(spec_r)
    o_r.residual(random_x(spec_r, seed=8, scale=0.3))
    w = o_r.site_weights()
    total = sum((o_r.mol_phi(0, s) * w).sum() for s in mol.segment_types())
    assert total == pytest.approx(1.5, rel=1e-12)


def test_dendrimer_input():
    text = """lat : l : n_layers : 20
lat : l : lowerbound : surface
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - S : -1
mol : d : composition : @dend(2, (A)3, 3, (B)2(A)1, 2)
mol : d : freedom : restricted
mol : d : n : 0.1
mol : w : composition : (W)1
mol : w : freedom : solvent
start
"""
    spec, _ = build_system(parse_input(text)[0])
    d = spec.molecules[0]
    assert d.N == 22 and d.count(1) == 13 and d.count(2) == 9
    assert d.theta == pytest.approx(2.2)
    with pytest.raises(ValueError):
        parse_dendrimer("@dend(2; (A)3, (A)2; (A)1, (A)1)")
    with pytest.raises(ValueError):
        parse_dendrimer("@dend(2, (A)3, 3)")
