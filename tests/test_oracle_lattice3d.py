"""The 3D lattice types of the oracle (FCC, HEX, stencils) against a
restatement of the reference's own array arithmetic (no GPU).

SFbox computes these steps on the flat site vector with shifted array
operations: ``times(a, b, c, n)`` sets a[i] = b[i] c[i], ``addTimes`` adds it,
``set(P, Q, l, n)`` sets P[i] = Q[i] l and ``addset`` adds it, each over a
sub-range given by the shift, after SetBoundaries has copied the boundary
planes one axis after the other.  The tables below list those operations in
the reference's order as (output shift, input shift, range shortening):
Lat3DFCC1stO.cpp:79-91, Lat3DHEX1stO.cpp:79-91 for the steps and
Lat3D.cpp:1733-1778 for the contact averages (Sides).  The oracle computes
the same sums site by site with per-axis boundary mapping, so the interior
values must agree bit for bit.
"""
import numpy as np
import pytest

from field_b200.desc import (BOUND_MIRROR1, BOUND_MIRROR2, BOUND_PERIODIC, LATTICE_FCC, LATTICE_HEX,
                             LATTICE_STANDARD, LATTICE_STENCILS, Lattice, Molecule, MOL_FREE, MOL_SOLVENT, Segment,
                             SystemSpec)
from field_b200.sfinput import build_system, parse_input
from oracle.oracle import Oracle

SHAPE_N = [6, 5, 7]
LO = [BOUND_MIRROR1, BOUND_MIRROR2, BOUND_PERIODIC]
HI = [BOUND_MIRROR2, BOUND_MIRROR1, BOUND_PERIODIC]


def _spec(ltype, lam3=(0.0, 0.0, 0.0, 0.0), n=SHAPE_N, lo=LO, hi=HI):
    lat = Lattice(3, list(n), list(lo), list(hi), lattice_type=ltype, lambda_3d=lam3)
    segs = [Segment("A"), Segment("W")]
    chi = np.array([[0.0, 0.5], [0.5, 0.0]])
    mols = [Molecule("p", [(0, 6)], MOL_FREE, phibulk=0.05), Molecule("w", [(1, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, chi, mols)


def _copy_layer(bc, n, lower):
    if bc == BOUND_PERIODIC:
        return n if lower else 1
    k = 1 if bc == BOUND_MIRROR1 else 2
    return k if lower else n + 1 - k


def _set_planes(P, shape, lo, hi, axes):
    """SetBx1, SetBxm, ... on whole boundary planes, in the given axis order."""
    P = P.reshape(shape).copy()
    for ax in axes:
        n = shape[ax] - 2
        for lower in (True, False):
            dst = 0 if lower else n + 1
            src = _copy_layer((lo if lower else hi)[ax], n, lower)
            idx_d = [slice(None)] * 3
            idx_s = [slice(None)] * 3
            idx_d[ax], idx_s[ax] = dst, src
            P[tuple(idx_d)] = P[tuple(idx_s)]
    return P.reshape(-1)


def _strides(shape):
    return shape[1] * shape[2], shape[2], 1


def _step_table(kind, shape):
    jx, jy, jz = _strides(shape)
    if kind == LATTICE_FCC:
        return [(jx + jy, 0, jx + jy), (0, jx + jy, jx + jy), (jx, jy, jx + jy), (jy, jx, jx + jy),
                (jy + jz, 0, jy + jz), (0, jy + jz, jy + jz), (jy, jz, jy + jz), (jz, jy, jy + jz),
                (jx + jz, 0, jx + jz), (0, jx + jz, jx + jz), (jx, jz, jx + jz), (jz, jx, jx + jz)]
    return [(jx, 0, jx), (0, jx, jx), (jx, jy, jx + jy), (0, jy, jy), (jy, 0, jy), (jy, jx, jy + jx),
            (jz, jy, jy + jz), (jz, 0, jz), (jz, jx, jx + jz), (jx, jz, jx + jz), (0, jz, jz), (jy, jz, jy + jz)]


def _step_shifts(gin, g, shape, kind):
    """One PropagateG(Gi, G, Gout) of the twelve-neighbour lattices."""
    M = gin.size
    gs_1 = _set_planes(gin, shape, LO, HI, (0, 1, 2))
    gs = np.zeros(M)
    for i, (a, b, sub) in enumerate(_step_table(kind, shape)):
        n = M - sub
        prod = gs_1[b:b + n] * g[a:a + n]
        if i == 0:
            gs[a:a + n] = prod
        else:
            gs[a:a + n] += prod
    return gs * (1.0 / 12.0)


def _sides_table(kind, shape, l):
    jx, jy, _ = _strides(shape)
    if kind == LATTICE_HEX:
        w = 1.0 / 12.0
        return [(0, jx, jx, w), (jx, 0, jx, w), (jy, jx, jx + jy, w), (jy, 0, jy, w), (0, jy, jy, w),
                (jx, jy, jx + jy, w), (jy, 1, jy + 1, w), (0, 1, 1, w), (jx, 1, jx + 1, w), (1, jx, jx + 1, w),
                (1, 0, 1, w), (1, jy, jy + 1, w)]
    l0, l1, l2, l3 = l
    t = [(0, 0, 0, l0), (0, jx, jx, l1), (jx, 0, jx, l1), (0, jy, jy, l1), (jy, 0, jy, l1), (0, 1, 1, l1),
         (1, 0, 1, l1)]
    t += [(0, jx + jy, jx + jy, l2), (0, jx - jy, jx - jy, l2), (jx - jy, 0, jx - jy, l2),
          (jx + jy, 0, jx + jy, l2), (0, jx + 1, jx + 1, l2), (0, jx - 1, jx - 1, l2), (jx - 1, 0, jx - 1, l2),
          (jx + 1, 0, jx + 1, l2), (0, jy + 1, jy + 1, l2), (0, jy - 1, jy - 1, l2), (jy - 1, 0, jy - 1, l2),
          (jy + 1, 0, jy + 1, l2)]
    t += [(0, jx + jy + 1, jx + jy + 1, l3), (0, jx + jy - 1, jx + jy - 1, l3), (0, jx - jy + 1, jx - jy + 1, l3),
          (0, jx - jy - 1, jx - jy - 1, l3), (jx - jy - 1, 0, jx - jy - 1, l3), (jx - jy + 1, 0, jx - jy + 1, l3),
          (jx + jy - 1, 0, jx + jy - 1, l3), (jx + jy + 1, 0, jx + jy + 1, l3)]
    return t


def _sides_shifts(q, shape, kind, l):
    """Lat3D::Sides(P, Q): SetBoundaries(Q) (z, y, then x planes), then the
    set / addset sequence."""
    M = q.size
    Q = _set_planes(q, shape, LO, HI, (2, 1, 0))
    P = np.zeros(M)
    for i, (a, b, sub, w) in enumerate(_sides_table(kind, shape, l)):
        n = M - sub
        if i == 0:
            P[a:a + n] = Q[b:b + n] * w
        else:
            P[a:a + n] += Q[b:b + n] * w
    return P


def _interior(shape):
    m = np.zeros(shape, bool)
    m[1:-1, 1:-1, 1:-1] = True
    return m.reshape(-1)


@pytest.mark.parametrize("kind", [LATTICE_FCC, LATTICE_HEX])
def test_twelve_neighbour_step_matches_shift_sequence(kind):
    spec = _spec(kind)
    o = Oracle(spec)
    shape = spec.lattice.shape
    rng = np.random.default_rng(41)
    gin = rng.uniform(0.1, 2.0, o.M)
    g = rng.uniform(0.2, 1.5, o.M)
    want = _step_shifts(gin, g, shape, kind)
    got = o.propagate(gin, g)
    inner = _interior(shape)
    assert np.array_equal(got[inner], want[inner])


@pytest.mark.parametrize("kind,lam", [(LATTICE_STANDARD, (0.0, 1 / 6, 0.0, 0.0)),
                                      (LATTICE_STENCILS, (0.1, 0.08, 0.02, 0.0225)),
                                      (LATTICE_FCC, (1 / 27,) * 4),
                                      (LATTICE_HEX, None)])
def test_contacts_match_shift_sequence(kind, lam):
    spec = _spec(kind, lam if kind == LATTICE_STENCILS else (0.0, 0.0, 0.0, 0.0))
    o = Oracle(spec)
    shape = spec.lattice.shape
    q = np.random.default_rng(43).uniform(0.0, 1.0, o.M)
    l = lam
    if kind == LATTICE_STENCILS:   # lambda3 recomputed from the other three (Lat3D.cpp:259)
        l = (lam[0], lam[1], lam[2], (1.0 - lam[0] - 6.0 * lam[1] - 12.0 * lam[2]) / 8.0)
    want = _sides_shifts(q, shape, kind, l)
    got = o.side(q)
    inner = _interior(shape)
    if kind == LATTICE_STANDARD:
        # the reference adds the zero-weight edge and corner products too
        np.testing.assert_allclose(got[inner], want[inner], rtol=1e-15, atol=0)
    else:
        assert np.array_equal(got[inner], want[inner])
    assert np.all(got[~inner] == 0.0)


@pytest.mark.parametrize("kind", [LATTICE_FCC, LATTICE_HEX])
def test_twelve_neighbour_step_is_symmetric(kind):
    """On a periodic box with G = 1 the step is a symmetric averaging
    operator: <a, A b> = <A a, b>, and it keeps constants."""
    spec = _spec(kind, n=[5, 6, 4], lo=[BOUND_PERIODIC] * 3, hi=[BOUND_PERIODIC] * 3)
    o = Oracle(spec)
    inner = _interior(spec.lattice.shape)
    rng = np.random.default_rng(5)
    a, b = rng.normal(size=o.M), rng.normal(size=o.M)
    one = np.ones(o.M)
    Aa, Ab = o.propagate(a, one), o.propagate(b, one)
    assert abs(a[inner] @ Ab[inner] - Aa[inner] @ b[inner]) < 1e-12 * np.abs(a[inner] @ Ab[inner]) + 1e-12
    np.testing.assert_allclose(o.propagate(one, one)[inner], 1.0, rtol=1e-15)
    np.testing.assert_allclose(o.side(one)[inner], 1.0, rtol=1e-15)


def test_lattice_type_validation():
    with pytest.raises(ValueError):          # lambdas do not sum to 1
        Oracle(_spec(LATTICE_STENCILS, (0.1, 0.1, 0.02, 0.02)))
    with pytest.raises(ValueError):          # a weight above 0.5
        Oracle(_spec(LATTICE_STENCILS, (0.6, 0.0, 0.0, 0.05)))
    lat2 = Lattice(2, [5, 5, 0], [BOUND_MIRROR1] * 2 + [0], [BOUND_MIRROR1] * 2 + [0], lattice_type=LATTICE_FCC)
    spec2 = SystemSpec(lat2, [Segment("A"), Segment("W")], np.zeros((2, 2)),
                       [Molecule("p", [(0, 4)], MOL_FREE, phibulk=0.1), Molecule("w", [(1, 1)], MOL_SOLVENT)])
    with pytest.raises(ValueError):
        Oracle(spec2)


_INPUT = """\
lat : box : gradients : 3
lat : box : n_layers_x : 5
lat : box : n_layers_y : 5
lat : box : n_layers_z : 5
{extra}mon : A : freedom : free
mon : W : freedom : free
mon : A : chi - W : 0.5
mol : p : composition : (A)6
mol : p : freedom : free
mol : p : phibulk : 0.05
mol : w : composition : (W)1
mol : w : freedom : solvent
start
"""


def test_input_latticetype():
    spec, _ = build_system(parse_input(_INPUT.format(extra="lat : box : latticetype : FCC\n"))[0])
    assert spec.lattice.lattice_type == LATTICE_FCC
    spec, _ = build_system(parse_input(_INPUT.format(extra="lat : box : latticetype : HEX\n"))[0])
    assert spec.lattice.lattice_type == LATTICE_HEX
    spec, _ = build_system(parse_input(_INPUT.format(extra="lat : box : latticetype : stencils\n"))[0])
    assert spec.lattice.lattice_type == LATTICE_STENCILS and spec.lattice.lambda_3d == (1 / 27,) * 4
    lam = "".join(f"lat : box : lambda{k} : {v}\n" for k, v in enumerate((0.1, 0.08, 0.02, 0.0225)))
    spec, _ = build_system(parse_input(_INPUT.format(extra="lat : box : latticetype : stencils\n" + lam))[0])
    assert spec.lattice.lambda_3d == (0.1, 0.08, 0.02, 0.0225)
    with pytest.raises(ValueError):          # lambda and lambda0 do not combine (Lat3D.cpp:221-224)
        build_system(parse_input(_INPUT.format(extra="lat : box : latticetype : stencils\n" + lam +
                                               "lat : box : lambda : 0.2\n"))[0])
    with pytest.raises(ValueError):          # lambda0..3 go together (Lat3D.cpp:225-230)
        build_system(parse_input(_INPUT.format(extra="lat : box : latticetype : stencils\n"
                                               "lat : box : lambda0 : 0.1\n"))[0])
    with pytest.raises(ValueError):
        build_system(parse_input(_INPUT.format(extra="lat : box : latticetype : hex\n"))[0])
