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


def _lumped_and_3d(grad, bx, by=None, n=(7, 6), N=8, S=0.45, seed=5):
    """The same free chain (S stiffness) in solvent on a lumped 1D/2D
    second-order lattice and on the 3D six-direction lattice made homogeneous
    along the lumped gradients (periodic, 3 layers), with potentials that
    depend on the modelled coordinates only."""
    from field_b200.desc import Lattice, Molecule, MOL_FREE, MOL_SOLVENT, Segment, SystemSpec
    segs = [Segment("A"), Segment("W")]
    chi = np.array([[0, 0.7], [0.7, 0]])
    pf = np.full((2, 2), 0.2)
    pf[0, 0] = S
    mols = [Molecule("A", [(0, N)], MOL_FREE, phibulk=0.05), Molecule("W", [(1, 1)], MOL_SOLVENT)]
    P = BOUND_PERIODIC
    if grad == 1:
        lo, hi = [bx[0], 0, 0], [bx[1], 0, 0]
        lat = Lattice(1, [n[0], 0, 0], lo, hi, order=2, lam=1 / 6)
        lat3 = Lattice(3, [n[0], 3, 3], [bx[0], P, P], [bx[1], P, P], order=2)
    else:
        lat = Lattice(2, [n[0], n[1], 0], [bx[0], by[0], 0], [bx[1], by[1], 0], order=2, lam=1 / 6)
        lat3 = Lattice(3, [n[0], n[1], 3], [bx[0], by[0], P], [bx[1], by[1], P], order=2)
    s1 = SystemSpec(lat, segs, chi, mols, pf=pf)
    s3 = SystemSpec(lat3, segs, chi, mols, pf=pf)
    o1, o3 = Oracle(s1), Oracle(s3)
    nc = s1.class_layout()[1]
    x1 = np.random.default_rng(seed).normal(0.0, 0.2, o1.nvar)
    # the 3D sites' potentials: those of the same modelled coordinates
    sites1, sites3 = s1.itvar_sites(), s3.itvar_sites()
    sh1, sh3 = lat.shape, lat3.shape
    key1 = {tuple(np.unravel_index(z, sh1)): j for j, z in enumerate(sites1)}
    x3 = np.empty(o3.nvar)
    for j, z in enumerate(sites3):
        c = np.unravel_index(z, sh3)
        j1 = key1[tuple(c[:grad])]
        x3[j * nc:(j + 1) * nc] = x1[j1 * nc:(j1 + 1) * nc]
    return s1, s3, o1, o3, x1, x3


@pytest.mark.parametrize("grad,bx,by", [(1, (BOUND_MIRROR1, BOUND_MIRROR1), None),
                                        (1, (BOUND_PERIODIC, BOUND_PERIODIC), None),
                                        (2, (BOUND_MIRROR1, BOUND_MIRROR1), (BOUND_PERIODIC, BOUND_PERIODIC)),
                                        (2, (BOUND_PERIODIC, BOUND_PERIODIC), (BOUND_MIRROR1, BOUND_MIRROR1))])
def test_lumped_second_order_equals_3d(grad, bx, by):
    """Lat1D2ndO / Lat2D2ndO lump the bond directions along homogeneous
    gradients (lateral x4, z x2).  On a 3D lattice homogeneous along those
    gradients the six-direction model must give the same profiles, residual
    and free energy per site, and lnGN larger by ln(sites per modelled
    site) -- an independent check of the lumped weights, multiplicities and
    mirror swaps."""
    s1, s3, o1, o3, x1, x3 = _lumped_and_3d(grad, bx, by)
    f1, f3 = o1.residual(x1), o3.residual(x3)
    sh1, sh3 = s1.lattice.shape, s3.lattice.shape
    reps = 3 ** (3 - grad)   # 3D sites per modelled site
    for i in range(2):
        p1 = o1.phi(i).reshape(sh1)
        p3 = o3.phi(i).reshape(sh3)
        inner1 = p1[(slice(1, -1),) * grad]
        for idx in np.ndindex(*sh3[grad:]):
            if any(v == 0 or v == sh3[grad + k] - 1 for k, v in enumerate(idx)):
                continue
            inner3 = p3[(slice(1, -1),) * grad + idx]
            np.testing.assert_allclose(inner3, inner1, rtol=1e-12, atol=1e-15)
    for m in range(2):
        assert o3.lngn(m) == pytest.approx(o1.lngn(m) + np.log(reps), rel=1e-12, abs=1e-12)
    # residual of every 3D site equals that of its modelled site
    nc = s1.class_layout()[1]
    sites1, sites3 = s1.itvar_sites(), s3.itvar_sites()
    key1 = {tuple(np.unravel_index(z, sh1)): j for j, z in enumerate(sites1)}
    for j, z in enumerate(sites3):
        j1 = key1[tuple(np.unravel_index(z, sh3)[:grad])]
        np.testing.assert_allclose(f3[j * nc:(j + 1) * nc], f1[j1 * nc:(j1 + 1) * nc], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("grad", [1, 2])
def test_lumped_second_order_step_conserves_weight(grad):
    """G = 1 and every component 1: each W row sums to S + 4L = 1, so one
    step (forward and backward) keeps every interior component at 1 on a
    periodic lattice."""
    from field_b200.desc import Lattice, Molecule, MOL_SOLVENT, Segment, SystemSpec
    P = BOUND_PERIODIC
    lat = Lattice(grad, [6, 5, 0][:3], [P, P if grad == 2 else 0, 0], [P, P if grad == 2 else 0, 0], order=2)
    spec = SystemSpec(lat, [Segment("W")], np.zeros((1, 1)), [Molecule("W", [(0, 1)], MOL_SOLVENT)])
    o = Oracle(spec)
    K = lat.components
    sh = lat.shape
    for bw in (0, 1):
        out = o.propagate(np.ones(K * o.M), np.ones(o.M), S=0.37, backward=bw).reshape((K,) + sh)
        inner = out[(slice(None),) + (slice(1, -1),) * grad]
        np.testing.assert_allclose(inner, 1.0, rtol=0, atol=1e-15)


@pytest.mark.parametrize("grad", [1, 2])
@pytest.mark.parametrize("freedom", ["free", "restricted"])
def test_lumped_second_order_mass_sum_rule(grad, freedom):
    """With a surface below and mirror1 above (and periodic y in 2D) every
    bond direction is counted once: sum_z w phi_A = phibulk * GN for a free
    chain and = theta for a restricted one.  Surface layers of the stored
    propagators stay 0, so the sum is finite and exact."""
    from field_b200.desc import (Lattice, Molecule, MOL_FREE, MOL_RESTRICTED, MOL_SOLVENT, Segment, SystemSpec,
                                 BOUND_SURFACE)
    if grad == 1:
        lat = Lattice(1, [9, 0, 0], [BOUND_SURFACE, 0, 0], [BOUND_MIRROR1, 0, 0], order=2, lam=1 / 6)
    else:
        lat = Lattice(2, [9, 7, 0], [BOUND_SURFACE, BOUND_PERIODIC, 0], [BOUND_MIRROR1, BOUND_PERIODIC, 0],
                      order=2, lam=1 / 6)
    segs = [Segment("A"), Segment("W")]
    chi = np.array([[0, 0.7], [0.7, 0]])
    pf = np.full((2, 2), 0.3)
    a = (Molecule("A", [(0, 12)], MOL_FREE, phibulk=0.05) if freedom == "free"
         else Molecule("A", [(0, 12)], MOL_RESTRICTED, theta=3.0))
    spec = SystemSpec(lat, segs, chi, [a, Molecule("W", [(1, 1)], MOL_SOLVENT)], pf=pf)
    o = Oracle(spec)
    f = o.residual(np.random.default_rng(1).normal(0.0, 0.3, o.nvar))
    assert np.all(np.isfinite(f))
    tot = float((o.phi(0) * o.site_weights()).sum())
    want = o.phibulk(0) * np.exp(o.lngn(0)) if freedom == "free" else 3.0
    assert tot == pytest.approx(want, rel=1e-13)


@pytest.mark.parametrize("case", ["3d_2nd_brush", "1d_2nd_lumped", "2d_2nd_lumped"])
def test_bond_orientation_slots_sum_to_phi(case):
    """Every direction component lands in one orientation slot (the 2D slot
    selection included), so on interior sites the slots add up to the
    molecule's phi; boundary entries are 0."""
    from cases import CASES, random_x
    spec = CASES[case]()
    o = Oracle(spec)
    o.residual(random_x(spec))
    inner = np.zeros(spec.lattice.shape, bool)
    inner[(slice(1, -1),) * spec.lattice.gradients] = True
    inner = inner.ravel()
    na = 2 if spec.lattice.components == 3 else 3
    for m, mol in enumerate(spec.molecules):
        if sum(n for _, n in mol.blocks) == 1:
            continue
        tot = sum(o.bond_orientation(m, a) for a in range(na))
        phim = sum(o.mol_phi(m, i) for i in sorted({b[0] for b in mol.blocks}))
        np.testing.assert_allclose(tot[inner], phim[inner], rtol=1e-13, atol=1e-16)
        assert not np.any(tot[~inner])


def test_bond_orientation_isotropic_melt():
    """u = 0 on a periodic 3D second-order lattice: every bond direction is
    equally likely, so each of the three axis slots holds phi / 3."""
    from field_b200.desc import Lattice, Molecule, MOL_FREE, MOL_SOLVENT, Segment, SystemSpec
    P = BOUND_PERIODIC
    lat = Lattice(3, [5, 4, 6], [P, P, P], [P, P, P], order=2)
    spec = SystemSpec(lat, [Segment("A"), Segment("W")], np.zeros((2, 2)),
                      [Molecule("A", [(0, 7)], MOL_FREE, phibulk=0.3), Molecule("W", [(1, 1)], MOL_SOLVENT)],
                      pf=np.full((2, 2), 0.35))
    o = Oracle(spec)
    o.residual(np.zeros(o.nvar))
    inner = np.zeros(lat.shape, bool)
    inner[1:-1, 1:-1, 1:-1] = True
    inner = inner.ravel()
    for a in range(3):
        np.testing.assert_allclose(o.bond_orientation(0, a)[inner], 0.1, rtol=1e-13)


@pytest.mark.parametrize("geom", ["cylindrical", "spherical"])
def test_curved_1d_step_by_hand(geom):
    """Lat1DCyl1stO / Lat1DSphere1stO around the centre (no offset, no layer
    adjustment): layer z (1-based radius x = z - 1 at its outer edge) holds
    L = V(x) - V(x - 1) sites with V = pi x^2 (cylinder) or 4/3 pi x^3
    (sphere), and a step goes inward with lambda S(x - 1) / L and outward
    with lambda S(x) / L, S the circumference / surface."""
    from field_b200.desc import GEOM_SPHERICAL
    n, lam = 9, 0.2
    g_ = GEOM_CYLINDRICAL if geom == "cylindrical" else GEOM_SPHERICAL
    lat = Lattice(1, [n, 0, 0], [BOUND_MIRROR1, 0, 0], [BOUND_MIRROR1, 0, 0], geometry=g_, lam=lam)
    spec = SystemSpec(lat, [Segment("A"), Segment("W")], np.zeros((2, 2)),
                      [Molecule("p", [(0, 3)], MOL_FREE, phibulk=0.1), Molecule("w", [(1, 1)], MOL_SOLVENT)])
    o = Oracle(spec)
    rng = np.random.default_rng(8)
    gin = o.set_boundaries(rng.uniform(0.2, 1.5, o.M))
    g = rng.uniform(0.5, 1.5, o.M)
    out = o.propagate(gin, g)
    x = np.arange(o.M, dtype=float)
    if geom == "cylindrical":
        V, S = np.pi * x ** 2, 2 * np.pi * x
    else:
        V, S = 4 / 3 * np.pi * x ** 3, 4 * np.pi * x ** 2
    for z in range(1, n + 1):
        L = V[z] - V[z - 1]
        lm, lp = lam * S[z - 1] / L, lam * S[z] / L
        want = g[z] * (gin[z] + lm * (gin[z - 1] - gin[z]) + lp * (gin[z + 1] - gin[z]))
        assert out[z] == pytest.approx(want, rel=1e-13)
        assert o.site_weights()[z] == pytest.approx(L, rel=1e-14)


@pytest.mark.parametrize("geom", ["cylindrical", "spherical"])
@pytest.mark.parametrize("off,ladj", [(0.0, 1.0), (2.5, 1.0), (0.0, 0.8), (1.5, 1.3)])
def test_curved_1d_detailed_balance(geom, off, ladj):
    """L(z) lam_+(z) = L(z+1) lam_-(z+1), with any core offset and layer
    adjustment: between mirror1 walls a step with G = 1 keeps the L-weighted
    sum, and u = 0 is the bulk with lnGN = ln(sum of L)."""
    from field_b200.desc import GEOM_SPHERICAL
    g_ = GEOM_CYLINDRICAL if geom == "cylindrical" else GEOM_SPHERICAL
    lat = Lattice(1, [14, 0, 0], [BOUND_MIRROR1, 0, 0], [BOUND_MIRROR1, 0, 0], geometry=g_, lam=1 / 6,
                  offset_first_layer=off, layer_adjustment=ladj)
    spec = SystemSpec(lat, [Segment("A"), Segment("W")], np.zeros((2, 2)),
                      [Molecule("p", [(0, 6)], MOL_FREE, phibulk=0.1), Molecule("w", [(1, 1)], MOL_SOLVENT)])
    o = Oracle(spec)
    rng = np.random.default_rng(2)
    gin = o.set_boundaries(rng.uniform(0.5, 1.5, o.M))
    out = o.propagate(gin, np.ones(o.M))
    w = o.site_weights()
    assert abs((w * out).sum() - (w * gin).sum()) < 1e-12 * (w * gin).sum()
    f = o.residual(np.zeros(o.nvar))
    np.testing.assert_allclose(f, 0.0, atol=1e-13)
    np.testing.assert_allclose(o.phi(0)[1:-1], 0.1, rtol=1e-13)
    assert o.lngn(0) == pytest.approx(np.log(w.sum()), rel=1e-13)


def _curved_tables(n, geom):
    """lambda_-/lambda_+ of a curved lattice around the centre (no offset, no
    layer adjustment), lambda = 1/6, by 0-based radial index 0..n+1."""
    x = np.arange(n + 2, dtype=float)
    if geom == "sphere":
        V, S = 4 / 3 * np.pi * x ** 3, 4 * np.pi * x ** 2
    else:
        V, S = np.pi * x ** 2, 2 * np.pi * x
    lm, lp = np.zeros(n + 2), np.zeros(n + 2)
    for z in range(1, n + 2):
        Lz = V[z] - V[z - 1]
        lm[z], lp[z] = S[z - 1] / Lz / 6, S[z] / Lz / 6
    return lm, lp


@pytest.mark.parametrize("geom", ["cylinder", "sphere"])
@pytest.mark.parametrize("backward", [0, 1])
def test_curved_1d_second_order_step_restated(geom, backward):
    """One Lat1DCyl2ndO / Lat1DSphere2ndO step written out component by
    component (three components +x, lateral x4, -x): a radial read mixes
    f * g(neighbour) + (1 - f) * g_reflected(here), f = 6 lambda_-(z) from
    inside, 6 lambda_+(z) from outside; mirror1 walls swap +x and -x."""
    from field_b200.desc import GEOM_SPHERICAL
    n, S = 9, 0.35
    g_ = GEOM_SPHERICAL if geom == "sphere" else GEOM_CYLINDRICAL
    lat = Lattice(1, [n, 0, 0], [BOUND_MIRROR1, 0, 0], [BOUND_MIRROR1, 0, 0], geometry=g_, order=2, lam=1 / 6)
    spec = SystemSpec(lat, [Segment("A"), Segment("W")], np.zeros((2, 2)),
                      [Molecule("p", [(0, 3)], MOL_FREE, phibulk=0.1), Molecule("w", [(1, 1)], MOL_SOLVENT)])
    o = Oracle(spec)
    M = n + 2
    rng = np.random.default_rng(5 + backward)
    gin = rng.uniform(0.2, 1.5, 3 * M)
    G = rng.uniform(0.5, 1.5, M)
    got = o.propagate(gin, G, S=S, backward=backward).reshape(3, M)
    g0, g1, g2 = gin.reshape(3, M).copy()
    g0[0], g2[0], g1[0] = g2[1], g0[1], g1[1]                     # SetBx1(g0,g2), SetBx1(g1)
    g0[-1], g2[-1], g1[-1] = g2[-2], g0[-2], g1[-2]               # SetBxm(g0,g2), SetBxm(g1)
    lm, lp = _curved_tables(n, geom)
    fm, fp = 6 * lm, 6 * lp
    L = (1 - S) / 4
    t = np.arange(1, M - 1)
    if not backward:
        HL0 = fm[t] * g0[t - 1] + (1 - fm[t]) * g2[t]
        HL1 = fm[t] * g1[t - 1] + (1 - fm[t]) * g1[t]
        HU1 = fp[t] * g1[t + 1] + (1 - fp[t]) * g1[t]
        HU2 = fp[t] * g2[t + 1] + (1 - fp[t]) * g0[t]
        want = [S * HL0 + 4 * L * HL1, L * g0[t] + (2 * L + S) * g1[t] + L * g2[t], 4 * L * HU1 + S * HU2]
    else:
        H0 = fp[t] * g0[t + 1] + (1 - fp[t]) * g2[t]
        H2 = fm[t] * g2[t - 1] + (1 - fm[t]) * g0[t]
        want = [S * H0 + 4 * L * g1[t], L * H0 + (2 * L + S) * g1[t] + L * H2, S * H2 + 4 * L * g1[t]]
    for k in range(3):
        np.testing.assert_allclose(got[k, 1:-1], want[k] * G[t], rtol=1e-13)


@pytest.mark.parametrize("backward", [0, 1])
def test_curved_2d_second_order_step_restated(backward):
    """One Lat2DCyl2ndO step written out (components +x, +y, z x2, -y, -x;
    x radial).  Forward: every radial read is mixed with the reflected
    component at the site.  Backward: only the reads of -x are (SFbox builds
    the +x mixture and leaves it unused)."""
    nx, ny, S = 7, 5, 0.3
    lat = Lattice(2, [nx, ny, 0], [BOUND_MIRROR1, BOUND_MIRROR1, 0], [BOUND_MIRROR1, BOUND_MIRROR1, 0],
                  geometry=GEOM_CYLINDRICAL, order=2, lam=1 / 6)
    spec = SystemSpec(lat, [Segment("A"), Segment("W")], np.zeros((2, 2)),
                      [Molecule("p", [(0, 3)], MOL_FREE, phibulk=0.1), Molecule("w", [(1, 1)], MOL_SOLVENT)])
    o = Oracle(spec)
    MX, MY = nx + 2, ny + 2
    rng = np.random.default_rng(9 + backward)
    gin = rng.uniform(0.2, 1.5, 5 * MX * MY)
    G = rng.uniform(0.5, 1.5, (MX, MY))
    got = o.propagate(gin, G.ravel(), S=S, backward=backward).reshape(5, MX, MY)
    g = gin.reshape(5, MX, MY).copy()
    for a, b in ((0, 1), (-1, -2)):          # x walls: swap +x/-x, copy the rest
        g[0, a], g[4, a] = g[4, b].copy(), g[0, b].copy()
        for k in (1, 2, 3):
            g[k, a] = g[k, b]
    for a, b in ((0, 1), (-1, -2)):          # y walls: swap +y/-y, copy the rest
        g[1, :, a], g[3, :, a] = g[3, :, b].copy(), g[1, :, b].copy()
        for k in (0, 2, 4):
            g[k, :, a] = g[k, :, b]
    lm, lp = _curved_tables(nx, "cylinder")
    fm, fp = (6 * lm)[:, None], (6 * lp)[:, None]
    L = (1 - S) / 4
    X, Y = slice(1, -1), slice(1, -1)
    c = lambda k, dx=0, dy=0: g[k, 1 + dx:MX - 1 + dx, 1 + dy:MY - 1 + dy]
    fmi, fpi = fm[X], fp[X]
    if not backward:
        HL = [fmi * c(k, -1) + (1 - fmi) * c(4 if k == 0 else k) for k in range(4)]
        HU = {k: fpi * c(k, 1) + (1 - fpi) * c(0 if k == 4 else k) for k in range(1, 5)}
        want = [S * HL[0] + L * HL[1] + 2 * L * HL[2] + L * HL[3],
                L * c(0, 0, -1) + S * c(1, 0, -1) + 2 * L * c(2, 0, -1) + L * c(4, 0, -1),
                L * c(0) + L * c(1) + S * c(2) + L * c(3) + L * c(4),
                L * c(0, 0, 1) + 2 * L * c(2, 0, 1) + S * c(3, 0, 1) + L * c(4, 0, 1),
                L * HU[1] + 2 * L * HU[2] + L * HU[3] + S * HU[4]]
    else:
        H4 = fmi * c(4, -1) + (1 - fmi) * c(0)
        want = [S * c(0, 1) + L * c(1, 0, 1) + 2 * L * c(2) + L * c(3, 0, -1),
                L * c(0, 1) + S * c(1, 0, 1) + 2 * L * c(2) + L * H4,
                L * c(0, 1) + L * c(1, 0, 1) + S * c(2) + L * c(3, 0, -1) + L * H4,
                L * c(0, 1) + 2 * L * c(2) + S * c(3, 0, -1) + L * H4,
                L * c(1, 0, 1) + 2 * L * c(2) + L * c(3, 0, -1) + S * H4]
    for k in range(5):
        np.testing.assert_allclose(got[k, X, Y], want[k] * G[X, Y], rtol=1e-13)


@pytest.mark.parametrize("case", ["1d_cyl", "1d_sphere", "2d_cyl"])
def test_curved_second_order_u_zero_is_bulk(case):
    """Every mixture f + (1 - f) = 1, so with G = 1 between mirror walls the
    all-ones distribution stays all ones: u = 0 is the bulk, and lnGN is
    ln(sum of L)."""
    from field_b200.desc import GEOM_SPHERICAL
    g_ = GEOM_SPHERICAL if case == "1d_sphere" else GEOM_CYLINDRICAL
    if case == "2d_cyl":
        lat = Lattice(2, [9, 6, 0], [BOUND_MIRROR1, BOUND_MIRROR2, 0], [BOUND_MIRROR1, BOUND_MIRROR1, 0],
                      geometry=g_, order=2, lam=1 / 6, offset_first_layer=1.5)
    else:
        lat = Lattice(1, [12, 0, 0], [BOUND_MIRROR1, 0, 0], [BOUND_MIRROR2, 0, 0], geometry=g_, order=2,
                      lam=1 / 6, offset_first_layer=2.0)
    spec = SystemSpec(lat, [Segment("A"), Segment("W")], np.zeros((2, 2)),
                      [Molecule("p", [(0, 7)], MOL_FREE, phibulk=0.2), Molecule("w", [(1, 1)], MOL_SOLVENT)],
                      pf=np.full((2, 2), 0.4))
    o = Oracle(spec)
    f = o.residual(np.zeros(o.nvar))
    np.testing.assert_allclose(f, 0.0, atol=1e-13)
    np.testing.assert_allclose(o.phi(0)[spec.itvar_sites()], 0.2, rtol=1e-13)
    assert o.lngn(0) == pytest.approx(np.log(o.site_weights().sum()), rel=1e-13)


def test_curved_second_order_large_radius_is_flat():
    """Far from the axis the mixing fractions tend to 1 and Lat1DCyl2ndO
    becomes Lat1D2ndO: profiles agree to the order of 1/R."""
    from field_b200.desc import GEOM_FLAT
    segs = [Segment("A"), Segment("W")]
    chi = np.array([[0, 0.8], [0.8, 0]])
    mols = [Molecule("p", [(0, 10)], MOL_FREE, phibulk=0.05), Molecule("w", [(1, 1)], MOL_SOLVENT)]
    pf = np.full((2, 2), 0.5)
    curved = Lattice(1, [15, 0, 0], [BOUND_MIRROR1, 0, 0], [BOUND_MIRROR1, 0, 0], geometry=GEOM_CYLINDRICAL,
                     order=2, lam=1 / 6, offset_first_layer=1e6)
    flat = Lattice(1, [15, 0, 0], [BOUND_MIRROR1, 0, 0], [BOUND_MIRROR1, 0, 0], geometry=GEOM_FLAT, order=2,
                   lam=1 / 6)
    oc = Oracle(SystemSpec(curved, segs, chi, mols, pf=pf))
    of = Oracle(SystemSpec(flat, segs, chi, mols, pf=pf))
    x = np.random.default_rng(4).normal(0.0, 0.3, of.nvar)
    oc.residual(x)
    of.residual(x)
    np.testing.assert_allclose(oc.phi(0)[1:-1], of.phi(0)[1:-1], rtol=1e-4)


def _grand_potential2(spec, o):
    """F - sum_i n_i mu_i with n_i mu_i of SF_MolList1stO::GetNumMolTimesChemPot
    (SF_MolList1stO.cpp:463-521; molecules without pinned or grafted
    segments, no reactions), restated here independently of the oracle."""
    F = o.thermo()[0]
    ns = len(spec.segments)
    chi = np.asarray(spec.chi, dtype=float)
    mols = spec.molecules
    w = o.site_weights()
    N = [sum(n for _, n in mol.blocks) for mol in mols]
    cnt = np.zeros((len(mols), ns))
    for m, mol in enumerate(mols):
        for seg, n in mol.blocks:
            cnt[m, seg] += n
    phib_m = [o.phibulk(m) for m in range(len(mols))]
    phib_s = np.array([sum(phib_m[m] * cnt[m, i] / N[m] for m in range(len(mols))) for i in range(ns)])
    cib = chi @ phib_s
    total = 0.0
    for m in range(len(mols)):
        used = [i for i in range(ns) if cnt[m, i] > 0]
        th_seg = {i: float((o.mol_phi(m, i) * w).sum()) for i in used}
        th = sum(th_seg.values())
        f = cnt[m] / N[m]
        cref = 0.5 * sum(f[i] * f[j] * chi[i, j] for i in used for j in used)
        v = (np.log(phib_m[m]) + 1) * th / N[m]
        v += th * (-sum(phib_m[k] / N[k] for k in range(len(mols))))
        v += sum(th_seg[i] * cib[i] for i in used) - th * cref
        v -= 0.5 * th * float((phib_s * cib).sum())
        total += v
    return F - total


@pytest.mark.parametrize("which", ["adsorption", "2d_surface", "sphere", "3d_fcc_colloid", "3d_hex_colloid",
                                   "3d_stencils_colloid"])
def test_grand_potential_equals_F_minus_n_mu_at_convergence(which):
    """At the self-consistent solution the grand potential summed from its
    density equals F - sum n mu (SFbox prints both, 'grand potential' and
    'grand potential2'); away from it they differ."""
    from cases import CASES
    spec = {"adsorption": lambda: configs.flat_adsorption(n=40, N=21)[0],
            "2d_surface": CASES["2d_flat_surface"], "sphere": CASES["1d_sphere_colloid"],
            **{k: CASES[k] for k in ("3d_fcc_colloid", "3d_hex_colloid", "3d_stencils_colloid")}}[which]()
    o = Oracle(spec)
    x, rc, it, err = o.solve_diis(np.zeros(spec.n_itvar()), tol=1e-11, maxit=20000, m=10, eta=0.3)
    assert rc == 0
    o.residual(x)
    F, Om, fe, gp = o.thermo()
    assert Om == pytest.approx(_grand_potential2(spec, o), abs=1e-9 * max(1.0, abs(F)))
    assert abs(Om) > 1e-6          # a surface excess, not the bulk
    o.residual(x + 0.05)
    assert abs(o.thermo()[1] - _grand_potential2(spec, o)) > 1e-4


def test_grand_potential_density_vanishes_in_the_bulk():
    """u = 0 between mirrors is the bulk: omega(z) = 0 everywhere."""
    spec = homopolymer_1d(n=15, N=7, chi=0.6)
    o = Oracle(spec)
    o.residual(np.zeros(o.nvar))
    F, Om, fe, gp = o.thermo()
    np.testing.assert_allclose(gp, 0.0, atol=1e-15)
    assert abs(Om) < 1e-13
