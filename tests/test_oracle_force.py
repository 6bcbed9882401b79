"""The constant-force ensemble (mol : force) in the oracle (no GPU): forward
steps biased by +f, backward by -f, so reflecting the lattice and the field
turns f into -f; the biased steps keep constants on the flat 1D, 2D
cylindrical and 3D lattices, so u = 0 stays the bulk; homopolymers and the
2D flat lattice refuse a force as SFbox does."""
import numpy as np
import pytest

from field_b200.desc import (BOUND_MIRROR1, BOUND_PERIODIC, GEOM_CYLINDRICAL, Lattice, Molecule, MOL_FREE,
                             MOL_SOLVENT, Segment, SystemSpec)
from oracle.oracle import Oracle


def _spec(f, lat=None, comp=((0, 4), (1, 3), (0, 2))):
    lat = lat or Lattice(1, [15, 0, 0], [BOUND_MIRROR1, 0, 0], [BOUND_MIRROR1, 0, 0], lam=0.2)
    segs = [Segment("A"), Segment("B"), Segment("W")]
    chi = np.zeros((3, 3))
    chi[0, 2] = chi[2, 0] = 0.8
    chi[1, 2] = chi[2, 1] = -0.2
    mols = [Molecule("c", list(comp), MOL_FREE, phibulk=0.04, force=f), Molecule("W", [(2, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, chi, mols)


def test_reflection_turns_f_into_minus_f():
    f = 0.7
    sa, sb = _spec(f), _spec(-f)
    nc = 3
    x = np.random.default_rng(5).normal(0, 0.3, sa.n_itvar())
    xr = x.reshape(-1, nc)[::-1].reshape(-1)          # sites 1..n reflected
    oa, ob = Oracle(sa), Oracle(sb)
    oa.residual(x)
    ob.residual(xr)
    for i in range(3):
        np.testing.assert_allclose(oa.phi(i)[1:-1], ob.phi(i)[1:-1][::-1], rtol=1e-12)
    assert oa.lngn(0) == pytest.approx(ob.lngn(0), rel=1e-13)
    # and the force does something
    o0 = Oracle(_spec(0.0))
    o0.residual(x)
    assert np.max(np.abs(o0.phi(0) - oa.phi(0))) > 1e-3


@pytest.mark.parametrize("lat", [
    Lattice(1, [15, 0, 0], [BOUND_MIRROR1, 0, 0], [BOUND_MIRROR1, 0, 0], lam=0.2),
    Lattice(2, [8, 9, 0], [BOUND_MIRROR1, BOUND_PERIODIC, 0], [BOUND_MIRROR1, BOUND_PERIODIC, 0],
            geometry=GEOM_CYLINDRICAL, lam=0.2),
    Lattice(3, [5, 4, 6], [BOUND_PERIODIC] * 3, [BOUND_PERIODIC] * 3),
])
def test_force_keeps_the_bulk(lat):
    spec = _spec(1.3, lat=lat)
    o = Oracle(spec)
    o.residual(np.zeros(spec.n_itvar()))
    sites = spec.itvar_sites()
    np.testing.assert_allclose(o.phi(0)[sites], 0.04 * 6 / 9, rtol=1e-12)
    np.testing.assert_allclose(o.phi(1)[sites], 0.04 * 3 / 9, rtol=1e-12)


def test_force_refusals():
    with pytest.raises(ValueError):
        Oracle(_spec(0.5, comp=((0, 9),)))           # homopolymer
    flat2 = Lattice(2, [6, 6, 0], [BOUND_MIRROR1] * 2 + [0], [BOUND_MIRROR1] * 2 + [0], lam=0.2)
    with pytest.raises(ValueError):
        Oracle(_spec(0.5, lat=flat2))                 # 2D flat lattice
