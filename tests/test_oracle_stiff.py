"""The stiff_range copolymers of 3D second-order lattices
(SF_Copol2ndO_stiff_range) in the oracle (no GPU): its steps against a numpy
restatement of the reference's shifted-array operations, the bulk limit and
the mass sum rule.

Lat3D2ndO::PropagateF/B(..., S, stiff) (Lat3D2ndO.cpp:155-247, :680-764)
compute gx_k[i + e] (+)= gz_kp[i] G[i + e] p[i] for the components read from
the lower neighbour and gx_k[i] (+)= gz_kp[i + e] G[i] p[i] for those read
from the upper one, with p = S inside the range and 0.2 outside for kp = k,
(1 - p)/4 otherwise; the isotropic steps (:250-344, :765-850) use G/6 for
every term, the forward -y component reading +z twice and -y never.
"""
import numpy as np
import pytest

from field_b200.desc import (BOUND_MIRROR1, BOUND_PERIODIC, Lattice, Molecule, MOL_FREE, MOL_RESTRICTED,
                             MOL_SOLVENT, Segment, SEG_PINNED, SystemSpec)
from oracle.oracle import Oracle

OPP = [5, 4, 3, 2, 1, 0]


def _spec(n=(5, 6, 4), periodic=True, mask=None, mols=None):
    b = [BOUND_PERIODIC] * 3 if periodic else [BOUND_MIRROR1] * 3
    lat = Lattice(3, list(n), b, b, order=2)
    shape = lat.shape
    if mask is None:
        mask = np.zeros(shape)
        mask[:, :, : shape[2] // 2] = 1.0
    lat.stiff_range = mask.reshape(-1)
    segs = [Segment("A"), Segment("B"), Segment("W")]
    chi = np.zeros((3, 3))
    chi[0, 2] = chi[2, 0] = 0.4
    pf = np.full((3, 3), 0.2)
    pf[0, 1] = pf[1, 0] = 0.5
    pf[0, 0] = 0.35
    mols = mols or [Molecule("AB", [(0, 4), (1, 3), (0, 2)], MOL_FREE, phibulk=0.05),
                    Molecule("W", [(2, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, chi, mols, pf=pf)


def _strides(shape):
    return shape[1] * shape[2], shape[2], 1


def _periodic_planes(P, shape):
    P = P.reshape(shape).copy()
    for ax in range(3):
        n = shape[ax] - 2
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[ax], hi[ax] = 0, n + 1
        src_lo = [slice(None)] * 3
        src_hi = [slice(None)] * 3
        src_lo[ax], src_hi[ax] = n, 1
        P[tuple(lo)] = P[tuple(src_lo)]
        P[tuple(hi)] = P[tuple(src_hi)]
    return P.reshape(-1)


def _ref_step(gin, G, mask, S, shape, backward, iso):
    """The reference's array operations on periodic boundaries."""
    M = G.size
    jx, jy, jz = _strides(shape)
    e = [jx, jy, jz, jz, jy, jx]            # stride of the axis of each component
    up = [True, True, True, False, False, False]   # + components
    gz = [_periodic_planes(gin[k * M:(k + 1) * M], shape) for k in range(6)]
    ps = np.where(mask != 0, S, 0.2)
    pl = (1.0 - ps) / 4.0
    gI = G * (1.0 / 6.0)
    out = [np.zeros(M) for _ in range(6)]
    started = [False] * 6

    def put(k, lo_out, val):
        n = val.size
        sl = slice(lo_out, lo_out + n)
        if started[k]:
            out[k][sl] += val
        else:
            out[k][sl] = val
            started[k] = True

    if not backward:
        for k in range(6):
            terms = ([0, 2, 2, 3, 4, 5] if k == 4 else list(range(6))) if iso else [q for q in range(6) if q != OPP[k]]
            d = e[k]
            n = M - d
            for kp in terms:
                if up[k]:   # gx_k[i + d] from gz_kp[i], G[i + d], p[i]
                    w = gI[d:d + n] if iso else G[d:d + n] * 0 + 1
                    v = gz[kp][:n] * gI[d:d + n] if iso else gz[kp][:n] * G[d:d + n] * (ps if kp == k else pl)[:n]
                    put(k, d, v)
                else:       # gx_k[i] from gz_kp[i + d], G[i], p[i]
                    v = gz[kp][d:d + n] * gI[:n] if iso else gz[kp][d:d + n] * G[:n] * (ps if kp == k else pl)[:n]
                    put(k, 0, v)
    else:
        for kp in [5, 4, 3, 2, 1, 0]:
            d = e[kp]
            n = M - d
            for k in range(6):
                if not iso and k == OPP[kp]:
                    continue
                if not up[kp]:  # gz_kp read at the lower neighbour: gx_k[i + d], gz[i], p[i]
                    v = gz[kp][:n] * gI[d:d + n] if iso else gz[kp][:n] * G[d:d + n] * (ps if kp == k else pl)[:n]
                    put(k, d, v)
                else:           # read at the upper neighbour: gx_k[i], gz[i + d], p[i]
                    v = gz[kp][d:d + n] * gI[:n] if iso else gz[kp][d:d + n] * G[:n] * (ps if kp == k else pl)[:n]
                    put(k, 0, v)
    return np.concatenate(out)


@pytest.mark.parametrize("backward", [False, True])
@pytest.mark.parametrize("iso", [False, True])
def test_stiff_steps_match_array_operations(backward, iso):
    spec = _spec()
    o = Oracle(spec)
    shape = spec.lattice.shape
    rng = np.random.default_rng(12)
    gin = rng.uniform(0.2, 1.5, 6 * o.M)
    G = rng.uniform(0.3, 1.2, o.M)
    mask = spec.lattice.stiff_range
    want = _ref_step(gin, G, mask, 0.45, shape, backward, iso)
    got = o.propagate_stiff(gin, G, 0.45, backward=backward, iso=iso)
    inner = np.zeros(shape, bool)
    inner[1:-1, 1:-1, 1:-1] = True
    inner = np.tile(inner.reshape(-1), 6)
    assert np.array_equal(got[inner], want[inner])


def test_backward_stiff_step_does_not_keep_constants_at_the_range_edge():
    """Backward, the weights of one output component come from the target
    site (+ components) and from the source site (- components), so where the
    range ends inside the box they need not sum to 1 -- as the reference
    computes them.  Forward (one site per component) and inside a uniform
    range they do."""
    spec = _spec(periodic=False)
    o = Oracle(spec)
    shape = spec.lattice.shape
    one = np.ones(6 * o.M)
    g = np.ones(o.M)
    inner = (slice(None), slice(1, -1), slice(1, -1), slice(1, -1))
    fwd = o.propagate_stiff(one, g, 0.45).reshape(6, *shape)[inner]
    bwd = o.propagate_stiff(one, g, 0.45, backward=True).reshape(6, *shape)[inner]
    np.testing.assert_allclose(fwd, 1.0, rtol=1e-15)
    assert np.max(np.abs(bwd - 1.0)) > 0.05


def test_stiff_copolymer_bulk_and_mass():
    """With the whole box in the range every step keeps G = 1 (the isotropic
    steps' -y quirk included: six terms of 1/6), so u = 0 gives the bulk
    profiles.  A restricted copolymer keeps its mass only to ~1e-4 in a
    field: forward step s takes Pf(s-1, s+1), backward step s Pf(s, s+2),
    and the isotropic end steps differ, so the forward and backward
    operators are not each other's transposes (SF_Copol2ndO_stiff_range.cpp:
    211-234)."""
    spec = _spec(periodic=False, mask=np.ones((7, 8, 6)))
    o = Oracle(spec)
    o.residual(np.zeros(spec.n_itvar()))
    sites = spec.itvar_sites()
    np.testing.assert_allclose(o.phi(0)[sites], 0.05 * 6 / 9, rtol=1e-12)
    np.testing.assert_allclose(o.phi(1)[sites], 0.05 * 3 / 9, rtol=1e-12)
    mols = [Molecule("AB", [(0, 4), (1, 3), (0, 2)], MOL_RESTRICTED, theta=3.0),
            Molecule("W", [(2, 1)], MOL_SOLVENT)]
    spec_r = _spec(periodic=False, mols=mols)   # mass is kept with a partial range too
    o_r = Oracle(spec_r)
    o_r.residual(np.random.default_rng(3).normal(0, 0.3, spec_r.n_itvar()))
    w = o_r.site_weights()
    mass = sum((o_r.mol_phi(0, s) * w).sum() for s in (0, 1))
    assert 1e-7 < abs(mass - 3.0) < 1e-3


def test_stiff_range_refuses_homopolymers():
    mols = [Molecule("A9", [(0, 9)], MOL_FREE, phibulk=0.05), Molecule("W", [(2, 1)], MOL_SOLVENT)]
    with pytest.raises(ValueError):
        Oracle(_spec(mols=mols))
