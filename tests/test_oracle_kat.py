"""Known-answer tests of the CPU oracle (no GPU).

SFbox ships no golden vectors for this path, so the oracle is pinned by
answers that follow from the equations: u = 0 limits, sum rules, symmetry
of the half-chain trick, detailed balance of the cylindrical step
probabilities and the homogeneous-melt free energy.
"""
import numpy as np
import pytest

from field_b200 import configs
from field_b200.desc import (BOUND_MIRROR1, BOUND_MIRROR2, BOUND_PERIODIC, BOUND_SURFACE, GEOM_CYLINDRICAL,
                             Lattice, Molecule, MOL_FREE, MOL_SOLVENT, Segment, SystemSpec)
from oracle.oracle import Oracle


def homopolymer_1d(n=20, N=10, lo=BOUND_MIRROR1, hi=BOUND_MIRROR1, phib=0.05, chi=0.0, lam=1 / 6):
    lat = Lattice(1, [n, 0, 0], [lo, 0, 0], [hi, 0, 0], lam=lam)
    segs = [Segment("A"), Segment("W")]
    c = np.array([[0, chi], [chi, 0.0]])
    mols = [Molecule("p", [(0, N)], MOL_FREE, phibulk=phib), Molecule("w", [(1, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, c, mols)


@pytest.mark.parametrize("N", [2, 3, 10, 11])
@pytest.mark.parametrize("bounds", [(BOUND_MIRROR1, BOUND_MIRROR1), (BOUND_PERIODIC, BOUND_PERIODIC),
                                    (BOUND_MIRROR2, BOUND_MIRROR2)])
def test_u_zero_gives_bulk(N, bounds):
    spec = homopolymer_1d(N=N, lo=bounds[0], hi=bounds[1])
    o = Oracle(spec)
    f = o.residual(np.zeros(o.nvar))
    phiA = o.phi(0)
    sites = spec.itvar_sites()
    np.testing.assert_allclose(phiA[sites], 0.05, rtol=1e-13)
    np.testing.assert_allclose(o.phi(1)[sites], 0.95, rtol=1e-13)
    # lnGN = ln(number of lattice sites) for G = 1 (ideal chain, reflecting walls)
    nsites = o.site_weights().sum()
    assert abs(o.lngn(0) - np.log(nsites)) < 1e-12
    np.testing.assert_allclose(f, 0.0, atol=1e-13)


def test_propagator_1d_single_step_by_hand():
    spec = homopolymer_1d(n=5, lo=BOUND_SURFACE, hi=BOUND_MIRROR1)
    o = Oracle(spec)
    gin = np.array([0.0, 1.0, 2.0, 3.0, 4.0, 5.0, 5.0])
    g = np.array([0.0, 1.0, 1.0, 0.5, 1.0, 2.0, 2.0])
    out = o.propagate(gin, g)
    l = 1 / 6
    want = np.zeros(7)
    for z in range(1, 6):
        want[z] = g[z] * (gin[z] + l * (gin[z - 1] - 2 * gin[z] + gin[z + 1]))
    want[6] = want[5]          # mirror1 upper bound copies layer n
    want[0] = gin[0]           # surface layer keeps its value
    np.testing.assert_allclose(out, want, rtol=1e-15)


def test_cylinder_detailed_balance():
    """L(x) lam_+(x) = L(x+1) lam_-(x+1): the step conserves the L-weighted sum
    of an unweighted (G = 1) distribution between mirror walls."""
    lat = Lattice(2, [12, 9, 0], [BOUND_MIRROR1] * 2 + [0], [BOUND_MIRROR1] * 2 + [0],
                  geometry=GEOM_CYLINDRICAL, lam=1 / 6)
    spec = SystemSpec(lat, [Segment("A"), Segment("W")], np.zeros((2, 2)),
                      [Molecule("p", [(0, 4)], MOL_FREE, phibulk=0.1), Molecule("w", [(1, 1)], MOL_SOLVENT)])
    o = Oracle(spec)
    rng = np.random.default_rng(1)
    gin = o.set_boundaries(rng.uniform(0.5, 1.5, o.M))
    g = np.ones(o.M)
    out = o.propagate(gin, g)
    w = o.site_weights()
    assert abs((w * out).sum() - (w * gin).sum()) < 1e-12 * (w * gin).sum()


def test_homopolymer_half_chain_equals_full_chain():
    """SF_Homopol1stO's symmetric half-chain trick gives the same phi as the
    full copolymer route for a chain of two identical-chemistry blocks."""
    base = configs.flat_adsorption(n=30, N=12)[0]
    rng = np.random.default_rng(5)
    x = rng.normal(0, 0.3, base.n_itvar())
    o1 = Oracle(base)
    o1.residual(x)
    phiA = o1.phi(1)
    # same system with the polymer written as (A)6(A2)6, A2 chemically equal to A
    segs = base.segments + [type(base.segments[1])("A2")]
    chi = np.zeros((4, 4))
    chi[:3, :3] = base.chi
    chi[3, :3] = base.chi[1, :]
    chi[:3, 3] = base.chi[:, 1]
    chi[3, 3] = base.chi[1, 1]
    mols = [Molecule("pol", [(1, 6), (3, 6)], MOL_FREE, phibulk=base.molecules[0].phibulk),
            base.molecules[1]]
    spec2 = SystemSpec(base.lattice, segs, chi, mols)
    cls, nc = spec2.class_layout()
    assert nc == 2 and cls[1] == cls[3]
    o2 = Oracle(spec2)
    f2 = o2.residual(x)
    np.testing.assert_allclose(o2.phi(1) + o2.phi(3), phiA, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(f2, o1.residual(x), rtol=1e-11, atol=1e-12)


def test_melt_homogeneous_free_energy_zero():
    spec, _ = configs.melt3d(n=6, nA=5, nB=5, chi_ab=0.3)
    o = Oracle(spec)
    f = o.residual(np.zeros(o.nvar))
    np.testing.assert_allclose(o.phi(0)[spec.itvar_sites()], 0.5, rtol=1e-13)
    np.testing.assert_allclose(f, 0.0, atol=1e-13)
    assert abs(o.free_energy()) < 1e-11


def test_converged_c1_incompressible():
    spec, x0 = configs.flat_adsorption()
    o = Oracle(spec)
    x, rc, it, err = o.solve_diis(x0, tol=1e-10, maxit=5000, m=10, eta=0.5)
    assert rc == 0 and err < 1e-10
    phit = o.phi(0) + o.phi(1) + o.phi(2)
    sites = spec.itvar_sites()
    np.testing.assert_allclose(phit[sites], 1.0, atol=1e-9)
    # far from the surface the polymer is at its bulk concentration
    assert abs(o.phi(1)[-3] - 0.01) < 1e-6
    # adsorption: excess amount is positive for chi_AS = -1
    assert o.phi(1)[1] > 0.01


def test_second_order_isotropic_limit_reduces_to_first_order_walk_count():
    """With S = L = 0.2 and G = 1 every component of an interior site gets 1
    (five allowed continuations of weight 0.2), so G stays 1 and lnGN is the
    log of the number of sites (Lat3D2ndO.cpp:995-1025)."""
    spec, _ = configs.brush3d(n=5, N=6, sigma=0.2)
    o = Oracle(spec)
    gin = np.ones(6 * o.M)
    out = o.propagate(gin, np.ones(o.M), S=0.2)
    w = o.site_weights() > 0
    for k in range(6):
        np.testing.assert_allclose(out[k * o.M:(k + 1) * o.M][w], 1.0, rtol=1e-15)
