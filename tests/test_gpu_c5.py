"""The second-order configuration at its stated size: Lat3D2ndO 96^3, a brush
of (X)1(A)199 grafted at z = 0 at seeded random sites (density 0.05), bending
penalty (Pf A-A 0.5), good solvent chi 0.3.

* checkpointed chain storage for residual evaluations
  (sfgpu_system_create_checkpointed): bit-identical residuals and profiles
  against full storage, on every full-storage chain family and on the 96^3
  brush itself;
* 32 grafting-density variants (0.01 .. 0.1) solved together, one stream and
  host thread each (sfgpu_solve_diis_many): every variant's iterates equal
  those of the same variant solved alone; on a smaller brush the batch
  converges and matches the single solves;
* the adjoint gradient at 96^3 with respect to u (64 random sites) and chi
  against central finite differences.
"""
import numpy as np
import pytest

from cases import CASES, random_x
from field_b200 import configs
from field_b200.system import System, solve_diis_many

pytestmark = pytest.mark.gpu

STRIDE = 14   # ~sqrt(200)


@pytest.mark.parametrize("case,stride", [("2d_cylinder", 3), ("3d_periodic_melt", 4), ("3d_2nd_brush", 4),
                                         ("3d_2nd_brush", 7), ("2d_2nd_lumped", 3), ("1d_2nd_lumped", 5),
                                         ("3d_mirror_mix", 2), ("1d_periodic_restricted", 6)])
def test_checkpointed_chain_storage_is_bit_identical(gpu_lib, case, stride):
    spec = CASES[case]()
    x = random_x(spec, seed=5, scale=0.2)
    full, ck = System(spec), System(spec, checkpoint_stride=stride)
    f1, f2 = full.residual(x), ck.residual(x)
    assert np.array_equal(f1, f2)
    for i in range(len(spec.segments)):
        assert np.array_equal(full.phi(i), ck.phi(i))
    for m in range(len(spec.molecules)):
        assert full.mol_scalars(m)["lngn"] == ck.mol_scalars(m)["lngn"]


def _brush(sigma=0.05, n=96):
    spec, x0 = configs.brush3d(n=n, N=200, sigma=sigma, chi=0.3, S=0.5)
    return spec, x0


def test_c5_brush_96_checkpointed_equals_full_storage(gpu_lib):
    spec, x0 = _brush()
    x = np.random.default_rng(96).normal(0.0, 0.05, spec.n_itvar())
    ck = System(spec, checkpoint_stride=STRIDE)
    f2 = ck.residual(x)
    phi2 = [ck.phi(i) for i in range(len(spec.segments))]
    del ck
    full = System(spec)
    f1 = full.residual(x)
    assert np.array_equal(f1, f2)
    for i in range(len(spec.segments)):
        assert np.array_equal(full.phi(i), phi2[i])


def test_c5_32_density_variants_batched_equal_single_solves(gpu_lib):
    sigmas = np.linspace(0.01, 0.1, 32)
    specs = [_brush(sigma=float(sg))[0] for sg in sigmas]
    systems = [System(sp, checkpoint_stride=STRIDE) for sp in specs]
    x0s = [np.zeros(sp.n_itvar()) for sp in specs]
    many = solve_diis_many(systems, x0s, tol=1e-12, maxit=3, m=5, eta=0.1)
    for i in (0, 13, 31):
        one = systems[i].solve(x0s[i], tol=1e-12, maxit=3, m=5, eta=0.1)
        assert many[i].iterations == one.iterations == 3
        assert np.array_equal(many[i].x, one.x), i


def test_brush_density_variants_batched_converge(gpu_lib):
    sigmas = np.linspace(0.05, 0.2, 8)
    specs = [configs.brush3d(n=12, N=24, sigma=float(sg), chi=0.3, S=0.5)[0] for sg in sigmas]
    systems = [System(sp, checkpoint_stride=5) for sp in specs]
    x0s = [np.zeros(sp.n_itvar()) for sp in specs]
    many = solve_diis_many(systems, x0s, tol=1e-9, maxit=4000, m=8, eta=0.1)
    for i, sp in enumerate(specs):
        assert many[i].converged, (i, many[i].status, many[i].error)
        one = System(sp).solve(x0s[i], tol=1e-9, maxit=4000, m=8, eta=0.1)
        assert one.converged and one.iterations == many[i].iterations
        np.testing.assert_array_equal(one.x, many[i].x)


def test_c5_adjoint_gradient_against_differences_96(gpu_lib):
    """d(|f|^2/2)/du at 64 random sites from the reverse sweep (checkpoints
    every 14 positions) and d(w.f)/dchi_AW against central differences."""
    spec, _ = _brush()
    s = System(spec, checkpoint_stride=STRIDE)
    s.set_checkpoint(STRIDE)
    x = np.random.default_rng(97).normal(0.0, 0.05, s.nvar)
    f = s.residual(x)
    _, g = s.vjp(x, f)
    rng = np.random.default_rng(98)
    idx = rng.choice(s.nvar, size=64, replace=False)
    h = 1e-6
    gscale = np.max(np.abs(g))
    for i in idx:
        e = np.zeros(s.nvar)
        e[i] = 1.0
        fd = (0.5 * np.sum(s.residual(x + h * e) ** 2) - 0.5 * np.sum(s.residual(x - h * e) ** 2)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * gscale, (i, fd, g[i])
    # chi: f is linear in chi at fixed x, so the central difference is exact
    # up to rounding
    w = rng.normal(size=s.nvar)
    dchi = s.vjp_chi(x, w)
    a, b = 1, 2   # A - W
    hc = 1e-3
    vals = []
    for sgn in (1, -1):
        sp, _ = _brush()
        sp.chi = np.array(spec.chi, dtype=float).copy()
        sp.chi[a, b] += sgn * hc
        sp.chi[b, a] += sgn * hc
        vals.append(float(w @ System(sp, checkpoint_stride=STRIDE).residual(x)))
    fd = (vals[0] - vals[1]) / (2 * hc)
    got = dchi[a, b] + dchi[b, a]
    assert abs(fd - got) <= 1e-8 * max(1.0, abs(fd)), (fd, got)


@pytest.mark.parametrize("xc", [1, 3, 8, 32])
@pytest.mark.parametrize("form", [1, 2])
def test_pipelined_3d_step_bit_identical(gpu_lib, xc, form):
    """The software-pipelined 3D first-order step (form 1; form 2 with two y
    rows per thread in the forward steps) gives the plain x-marching step's
    results bit for bit, for chunk depths that do and do not divide the
    lattice and y extents that do and do not fill the last tile
    (composition-free forward steps and composing backward steps both run
    inside a residual)."""
    for case in ("3d_periodic_melt", "3d_mirror_mix", "3d_2nd_brush"):
        spec = CASES[case]()
        x = random_x(spec, seed=9, scale=0.2)
        a, b = System(spec), System(spec)
        a.set_tile(xc)
        b.set_tile(xc)
        a.set_tile_pipelined(form)
        b.set_tile_pipelined(0)
        assert np.array_equal(a.residual(x), b.residual(x)), case
        for i in range(len(spec.segments)):
            assert np.array_equal(a.phi(i), b.phi(i)), (case, i)
    for n in (40, 21):
        spec, x0 = configs.melt3d(n=n, nA=10, nB=10)
        a, b = System(spec), System(spec)
        a.set_tile(xc)
        b.set_tile(xc)
        a.set_tile_pipelined(form)
        b.set_tile_pipelined(0)
        assert np.array_equal(a.residual(x0), b.residual(x0)), n
