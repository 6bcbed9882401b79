"""Exact Jacobian-vector products (forward-mode tangent of the residual) and
the Newton-Krylov iteration built on them.

J*v is checked against central finite differences of the residual (h = 1e-5,
truncation error ~h^2, tolerance 1e-6 relative to max|J v|), the primal f of
the tangent sweep against sfgpu_residual bit for bit, the residual wrapped
as a torch.autograd.Function (forward mode, test harness only) against
torch.func.jvp, and derivatives at 64 random sites of a 3D melt against
finite differences.
"""
import numpy as np
import pytest
import torch

from cases import CASES, DIFFERENTIABLE, random_x
from field_b200 import configs
from field_b200.system import System
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

H = 1e-5
TOL_FD = 1e-6


def fd_jv(sys_, x, v, h=H):
    return (sys_.residual(x + h * v) - sys_.residual(x - h * v)) / (2 * h)


@pytest.mark.parametrize("case", DIFFERENTIABLE)
def test_jvp_matches_central_differences(gpu_lib, case):
    spec = CASES[case]()
    s = System(spec)
    x = random_x(spec, seed=21, scale=0.2)
    v = np.random.default_rng(22).normal(0.0, 1.0, s.nvar)
    f, jv = s.jvp(x, v)
    if "dendrimer" in case:
        # the derivatives run a dendrimer as its bond tree: the same molecule
        # through the tree recursion, equal to the generation walk up to rounding
        np.testing.assert_allclose(f, s.residual(x), rtol=0, atol=1e-12 * np.max(np.abs(f)))
    else:
        assert np.array_equal(f, s.residual(x)), "primal of the tangent sweep differs from the residual"
    ref = fd_jv(s, x, v)
    err = np.max(np.abs(jv - ref)) / max(np.max(np.abs(ref)), 1e-300)
    assert err < TOL_FD, err


def test_jvp_is_linear_in_v(gpu_lib):
    spec, x0 = configs.cyl_micelle(nx=24, ny=20, nA=7, nB=6, radius=4)
    s = System(spec)
    rng = np.random.default_rng(3)
    v1, v2 = rng.normal(size=s.nvar), rng.normal(size=s.nvar)
    _, a = s.jvp(x0, v1)
    _, b = s.jvp(x0, v2)
    _, c = s.jvp(x0, 2.0 * v1 - 0.5 * v2)
    np.testing.assert_allclose(c, 2.0 * a - 0.5 * b, rtol=1e-10, atol=1e-12 * np.max(np.abs(c)))


class Residual(torch.autograd.Function):
    """f(x) of one system, with its forward-mode derivative from sfgpu_jvp
    (test harness only)."""

    @staticmethod
    def forward(x, sys_):
        return torch.from_numpy(sys_.residual(x.detach().cpu().numpy()))

    @staticmethod
    def setup_context(ctx, inputs, output):
        ctx.x, ctx.sys_ = inputs[0].detach().cpu().numpy(), inputs[1]

    @staticmethod
    def jvp(ctx, dx, _):
        _, jv = ctx.sys_.jvp(ctx.x, dx.detach().cpu().numpy())
        return torch.from_numpy(jv)


def test_autograd_function_forward_mode(gpu_lib):
    spec, x0 = configs.flat_adsorption(n=40, N=30)
    s = System(spec)
    x = torch.tensor(random_x(spec, seed=5, scale=0.2))
    v = torch.tensor(np.random.default_rng(6).normal(size=s.nvar))
    with torch.autograd.forward_ad.dual_level():
        out = Residual.apply(torch.autograd.forward_ad.make_dual(x, v), s)
        tangent = torch.autograd.forward_ad.unpack_dual(out).tangent
    ref = fd_jv(s, x.numpy(), v.numpy())
    assert np.max(np.abs(tangent.numpy() - ref)) / np.max(np.abs(ref)) < TOL_FD


def test_derivatives_at_64_random_sites_3d(gpu_lib):
    """Config C3 shape (3D periodic A_nA B_nB melt): d f / d u at 64 random
    sites (unit directions) against central finite differences."""
    spec, x0 = configs.melt3d(n=32, nA=20, nB=20)
    s = System(spec)
    rng = np.random.default_rng(64)
    idx = rng.choice(s.nvar, size=64, replace=False)
    for i in idx:
        e = np.zeros(s.nvar)
        e[i] = 1.0
        _, jv = s.jvp(x0, e)
        ref = fd_jv(s, x0, e)
        assert np.max(np.abs(jv - ref)) <= TOL_FD * max(np.max(np.abs(ref)), 1e-12), i


def test_newton_krylov_c1(gpu_lib):
    spec, x0 = configs.flat_adsorption()
    s = System(spec)
    r = s.solve_nk(x0, tol=1e-10, maxit=40, krylov=40)
    assert r.converged, (r.status, r.error, r.iterations)
    o = Oracle(spec)
    assert np.linalg.norm(o.residual(r.x)) < 1e-9
    xd, rc, it, err = o.solve_diis(x0, tol=1e-10, maxit=5000, m=10, eta=0.5)
    o.residual(xd)
    phi_d = o.phi(1)
    o.residual(r.x)
    np.testing.assert_allclose(o.phi(1), phi_d, rtol=1e-7, atol=1e-12)


def test_newton_krylov_agrees_with_pure_diis_on_sweep(gpu_lib):
    """Newton-Krylov (exact J*v, GMRES) reaches the same fixed point as the
    oracle's Pure_DIIS on every 1D sweep instance where Pure_DIIS (m=5,
    eta=0.1) converges.  The poor-solvent instances (chi_AW >= 0.74) where
    Pure_DIIS stalls are skipped: there the homogeneous start sits near the
    spinodal and neither method is expected to find a unique solution."""
    insts = configs.sweep1d(count=24, N_range=(20, 200))
    checked = 0
    for i, (spec, x0) in enumerate(insts):
        o = Oracle(spec)
        xd, rc, _, _ = o.solve_diis(x0, tol=1e-10, maxit=3000, m=5, eta=0.1)
        if rc != 0:
            continue
        r = System(spec).solve_nk(x0, tol=1e-10, maxit=120, krylov=40)
        assert r.converged, (i, r.status, r.error, r.iterations)
        assert np.linalg.norm(o.residual(r.x)) < 1e-8, i
        phi_nk = [o.phi(k).copy() for k in range(len(spec.segments))]
        o.residual(xd)
        for k in range(len(spec.segments)):
            np.testing.assert_allclose(phi_nk[k], o.phi(k), rtol=1e-6, atol=1e-10 * np.max(o.phi(k)))
        checked += 1
    assert checked >= 15


@pytest.mark.parametrize("case,stride", [("3d_2nd_brush", 4), ("2d_cylinder", 3), ("1d_2nd_lumped", 5)])
def test_jvp_on_checkpointed_system(gpu_lib, case, stride):
    """A system created with checkpointed chain storage keeps every slice of
    the tangent sweeps in a buffer of their own: J.v equals the full-storage
    system's bit for bit."""
    spec = CASES[case]()
    x = random_x(spec, seed=21, scale=0.2)
    v = np.random.default_rng(22).normal(size=spec.n_itvar())
    f1, jv1 = System(spec).jvp(x, v)
    f2, jv2 = System(spec, checkpoint_stride=stride).jvp(x, v)
    assert np.array_equal(f1, f2) and np.array_equal(jv1, jv2)
