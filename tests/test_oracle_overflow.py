"""Overflow protection (sys : overflow_protection) in the oracle (no GPU).

The *1stOS lattices compute the same chain statistics in logarithms, so on
systems that stay inside the range of a double the profiles, residuals and
lnGN equal the plain first-order ones to rounding.  Where they differ, the
differences are the reference's: its 1D flat ComputeLnGN drops the layer
adjustment (Lat1DFlat1stOS.cpp:441-478), and its 2D ComputeLnGN halves the
column y = MY-2 (1-based) for an upper mirror2 in y (Lat2DFlat1stOS.cpp:482-488).
A restricted chain of 2000 segments in a uniform field of -1 overflows the
plain path and stays exact in logarithms.
"""
import numpy as np
import pytest

from cases import CASES, random_x
from field_b200.desc import (BOUND_MIRROR1, BOUND_MIRROR2, BOUND_SURFACE, Lattice, Molecule, MOL_FREE,
                             MOL_RESTRICTED, MOL_SOLVENT, Segment, SystemSpec)
from oracle.oracle import Oracle

LOG_CASES = ["1d_surface", "1d_lambda_chi", "1d_periodic_restricted", "1d_cylinder", "1d_sphere_colloid",
             "2d_cylinder", "2d_flat_surface"]


def _rel(a, b):
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("case", LOG_CASES)
def test_log_space_equals_plain(case):
    spec = CASES[case]()
    x = random_x(spec, seed=17, scale=0.25)
    plain = Oracle(spec)
    f0 = plain.residual(x)
    spec.overflow_protection = True
    logo = Oracle(spec)
    f1 = logo.residual(x)
    assert np.max(np.abs(f1 - f0)) < 1e-13
    for i in range(len(spec.segments)):
        assert _rel(logo.phi(i), plain.phi(i)) < 1e-13
    for m in range(len(spec.molecules)):
        assert abs(logo.lngn(m) - plain.lngn(m)) < 1e-12 * max(1.0, abs(plain.lngn(m)))


def test_overflow_protection_only_on_first_order_1d_2d():
    for case in ("3d_mirror_mix", "1d_2nd_lumped", "3d_2nd_brush"):
        spec = CASES[case]()
        spec.overflow_protection = True
        with pytest.raises(ValueError):
            Oracle(spec)


def _chain_in_uniform_field(N, overflow, n=20):
    lat = Lattice(1, [n, 0, 0], [BOUND_MIRROR1, 0, 0], [BOUND_MIRROR1, 0, 0], lam=1 / 6)
    segs = [Segment("A"), Segment("W")]
    mols = [Molecule("p", [(0, N)], MOL_RESTRICTED, theta=2.0), Molecule("w", [(1, 1)], MOL_SOLVENT)]
    spec = SystemSpec(lat, segs, np.zeros((2, 2)), mols, overflow_protection=overflow)
    # A and W have equal chi rows and share one class: u = -1 on every site,
    # G = e, G^N = e^2000
    assert spec.n_itvar() == n
    return spec, -np.ones(spec.n_itvar())


def test_long_chain_overflows_plain_and_not_in_logs():
    spec, x = _chain_in_uniform_field(2000, overflow=False)
    plain = Oracle(spec)
    with np.errstate(all="ignore"):
        plain.residual(x)
    assert not np.all(np.isfinite(plain.phi(0)))
    spec, x = _chain_in_uniform_field(2000, overflow=True)
    logo = Oracle(spec)
    logo.residual(x)
    sites = spec.itvar_sites()
    # uniform field: the restricted chains spread evenly, theta / n per site
    np.testing.assert_allclose(logo.phi(0)[sites], 2.0 / 20, rtol=1e-12)
    assert logo.lngn(0) == pytest.approx(2000 * 1.0 + np.log(20), rel=1e-14)


def test_flat_1d_lngn_drops_the_layer_adjustment():
    lat = Lattice(1, [12, 0, 0], [BOUND_SURFACE, 0, 0], [BOUND_MIRROR1, 0, 0], lam=0.25, layer_adjustment=0.7)
    segs = [Segment("S", 1, np.r_[1.0, np.zeros(13)]), Segment("A"), Segment("W")]
    chi = np.zeros((3, 3))
    chi[0, 1] = chi[1, 0] = -1.0
    mols = [Molecule("p", [(1, 7)], MOL_FREE, phibulk=0.02), Molecule("w", [(2, 1)], MOL_SOLVENT)]
    spec = SystemSpec(lat, segs, chi, mols, overflow_protection=True)
    o = Oracle(spec)
    g = np.random.default_rng(3).uniform(-2.0, 1.0, o.M)
    g[0] = g[-1] = -np.finfo(float).max / 2
    want = np.log(np.exp(g[1:-1]).sum())      # every interior layer with weight 1
    assert o.lat_lngn(g) == pytest.approx(want, rel=1e-14)
    spec.overflow_protection = False
    lin = Oracle(spec).lat_lngn(np.exp(g))    # the plain path weighs layer 1 by 0.7, layer n by 1.3
    w = np.ones(12)
    w[0], w[-1] = 0.7, 1.3
    assert lin == pytest.approx(np.log((w * np.exp(g[1:-1])).sum()), rel=1e-14)


@pytest.mark.parametrize("cyl", [False, True])
def test_2d_lngn_mirror2_weights(cyl):
    """The 2D ComputeLnGN with mirror2 on every side: interior 1 (L(x) on the
    cylinder), half of the rows x = 1, nx and of the columns y = 1 and
    y = ny - 1 (0-based, the reference's MY-2), corners added back with 1/4
    (flat) or 4 L(x) (cylinder)."""
    from field_b200.desc import GEOM_CYLINDRICAL, GEOM_FLAT
    nx, ny = 6, 7
    lat = Lattice(2, [nx, ny, 0], [BOUND_MIRROR2, BOUND_MIRROR2, 0], [BOUND_MIRROR2, BOUND_MIRROR2, 0],
                  geometry=GEOM_CYLINDRICAL if cyl else GEOM_FLAT, lam=1 / 6)
    segs = [Segment("A"), Segment("W")]
    mols = [Molecule("p", [(0, 5)], MOL_FREE, phibulk=0.05), Molecule("w", [(1, 1)], MOL_SOLVENT)]
    spec = SystemSpec(lat, segs, np.zeros((2, 2)), mols, overflow_protection=True)
    o = Oracle(spec)
    g = np.random.default_rng(9).uniform(-1.0, 1.0, o.M)
    Lx = np.array([np.pi * ((x) ** 2 - (x - 1) ** 2) for x in range(nx + 2)]) if cyl else np.ones(nx + 2)
    w = np.zeros((nx + 2, ny + 2))
    for x in range(1, nx + 1):
        w[x, 1:ny + 1] = Lx[x]
    w[1, 1:ny + 1] -= 0.5 * Lx[1]
    w[nx, 1:ny + 1] -= 0.5 * Lx[nx]
    for x in range(1, nx + 1):
        w[x, 1] -= 0.5 * Lx[x]
        w[x, ny - 1] -= 0.5 * Lx[x]
    for (x, y) in [(1, 1), (1, ny - 1), (nx, 1), (nx, ny - 1)]:
        w[x, y] += (4 * Lx[x]) if cyl else 0.25
    want = np.log((w.reshape(-1) * np.exp(g)).sum())
    assert o.lat_lngn(g) == pytest.approx(want, rel=1e-13)
