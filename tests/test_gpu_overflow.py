"""Overflow protection on the GPU against the oracle: log-space steps and
lnGN at the lattice level, full residual evaluations, a converged solve,
and a chain whose weights overflow a double."""
import numpy as np
import pytest
import torch

from cases import CASES, random_x
from field_b200.desc import (BOUND_MIRROR2, BOUND_SURFACE, GEOM_CYLINDRICAL, GEOM_FLAT, Lattice, Molecule,
                             MOL_FREE, MOL_SOLVENT, Segment, SystemSpec)
from field_b200.system import System
from oracle.oracle import Oracle
from test_oracle_overflow import LOG_CASES, _chain_in_uniform_field

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def _lattice2d(cyl, lo=BOUND_MIRROR2, hi=BOUND_MIRROR2):
    lat = Lattice(2, [9, 8, 0], [lo, BOUND_MIRROR2, 0], [hi, BOUND_MIRROR2, 0],
                  geometry=GEOM_CYLINDRICAL if cyl else GEOM_FLAT, lam=0.2)
    segs = [Segment("A"), Segment("W")]
    chi = np.array([[0.0, 0.6], [0.6, 0.0]])
    mols = [Molecule("p", [(0, 6)], MOL_FREE, phibulk=0.05), Molecule("w", [(1, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, chi, mols, overflow_protection=True)


@pytest.mark.parametrize("cyl", [False, True])
@pytest.mark.parametrize("lo", [BOUND_MIRROR2, BOUND_SURFACE])
def test_log_step_and_lngn(gpu_lib, cyl, lo):
    spec = _lattice2d(cyl, lo=lo)
    s = System(spec)
    o = Oracle(spec)
    rng = np.random.default_rng(5)
    LZ = -np.finfo(float).max / 2
    gin = rng.uniform(-3.0, 2.0, o.M)
    g = rng.uniform(-1.0, 1.0, o.M)
    g[rng.random(o.M) < 0.1] = LZ          # some sites where G = 0
    gin[rng.random(o.M) < 0.1] = LZ
    want = o.propagate(gin, g)
    got = s.propagate(torch.tensor(gin, device="cuda"), torch.tensor(g, device="cuda")).cpu().numpy()
    inner = np.zeros(spec.lattice.shape, bool)
    inner[1:-1, 1:-1] = True
    inner = inner.ravel()
    assert np.array_equal(got[inner] == LZ, want[inner] == LZ)
    ok = inner & (want > LZ)
    assert np.max(np.abs(got[ok] - want[ok])) < 1e-13 * max(1.0, np.max(np.abs(want[ok])))
    assert s.lngn(torch.tensor(gin, device="cuda")) == pytest.approx(o.lat_lngn(gin), rel=1e-13, abs=1e-13)


@pytest.mark.parametrize("case", LOG_CASES)
def test_log_space_residual_parity(gpu_lib, case):
    spec = CASES[case]()
    spec.overflow_protection = True
    s = System(spec)
    o = Oracle(spec)
    x = random_x(spec, seed=19, scale=0.25)
    fg, fc = s.residual(x), o.residual(x)
    assert rel(fg, fc) <= 1e-11
    for i in range(len(spec.segments)):
        assert rel(s.phi(i), o.phi(i)) <= 1e-11
    for m in range(len(spec.molecules)):
        assert abs(s.mol_scalars(m)["lngn"] - o.lngn(m)) <= 1e-11 * max(1.0, abs(o.lngn(m)))
    Fg, Og, _, _ = s.thermo()
    Fc, Oc, _, _ = o.thermo()
    assert abs(Fg - Fc) <= 1e-10 * max(1.0, abs(Fc)) and abs(Og - Oc) <= 1e-10 * max(1.0, abs(Oc), abs(Fc))


@pytest.mark.parametrize("case", ["1d_surface", "2d_flat_surface"])
def test_log_space_converged_parity(gpu_lib, case):
    spec = CASES[case]()
    spec.overflow_protection = True
    s = System(spec)
    o = Oracle(spec)
    x0 = np.zeros(spec.n_itvar())
    rg = s.solve(x0, tol=1e-10, maxit=4000, m=8, eta=0.3)
    xc, rc, it, err = o.solve_diis(x0, tol=1e-10, maxit=4000, m=8, eta=0.3)
    assert rg.converged and rc == 0
    s.residual(rg.x)
    o.residual(xc)
    for i in range(len(spec.segments)):
        np.testing.assert_allclose(s.phi(i), o.phi(i), rtol=1e-9, atol=1e-12)


def test_long_chain_stays_finite(gpu_lib):
    """2000 segments in u = -1: e^2000 overflows a double; in logarithms the
    restricted chains spread evenly, theta / n per site."""
    spec, x = _chain_in_uniform_field(2000, overflow=True)
    s = System(spec)
    s.residual(x)
    sites = spec.itvar_sites()
    np.testing.assert_allclose(s.phi(0)[sites], 2.0 / 20, rtol=1e-11)
    assert s.mol_scalars(0)["lngn"] == pytest.approx(2000.0 + np.log(20), rel=1e-13)


def test_overflow_protection_outside_batch_and_derivatives(gpu_lib):
    from field_b200._native import SfgpuError
    from field_b200.batch import BatchSolver
    spec = CASES["1d_surface"]()
    spec.overflow_protection = True
    s = System(spec)
    x = random_x(spec)
    for call in (lambda: s.jvp(x, x), lambda: s.vjp(x, x)):
        with pytest.raises(SfgpuError) as e:
            call()
        assert e.value.code == 7
    with pytest.raises(SfgpuError) as e:
        BatchSolver([spec], m=5, eta=0.1)
    assert e.value.code == 7
    spec3 = CASES["3d_mirror_mix"]()
    spec3.overflow_protection = True
    with pytest.raises(SfgpuError) as e:
        System(spec3)
    assert e.value.code == 7
