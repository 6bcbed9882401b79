"""Reverse-mode derivative of the residual (J(x)^T w from the adjoint sweep)
and the L-BFGS iteration that uses it as the gradient of |f|^2 / 2.

First- and second-order lattices.  The adjoint is checked by the dot-product identity <w, J v> = <J^T w, v>
against the forward-mode tangent (itself pinned to finite differences in
test_gpu_tangent.py), relative tolerance 1e-10 of |w| |J v|; directional
derivatives of |f|^2/2 against central differences; and the primal f of the
adjoint sweep against sfgpu_residual (1e-12 of max|f|: the sweep propagates
full chains where the residual may use the half-chain trick for symmetric
homopolymers).
"""
import numpy as np
import torch
import pytest

from cases import CASES, DIFFERENTIABLE, REVERSE_EXCLUDED, random_x
from field_b200 import configs
from field_b200.system import System
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

FIRST_ORDER = sorted(k for k in DIFFERENTIABLE if not any(t in k for t in REVERSE_EXCLUDED))


@pytest.mark.parametrize("case", FIRST_ORDER)
def test_dot_product_identity(gpu_lib, case):
    spec = CASES[case]()
    s = System(spec)
    x = random_x(spec, seed=31, scale=0.2)
    rng = np.random.default_rng(32)
    v = rng.normal(size=s.nvar)
    w = rng.normal(size=s.nvar)
    f, jv = s.jvp(x, v)
    f2, jtw = s.vjp(x, w)
    np.testing.assert_allclose(f2, f, rtol=0, atol=1e-12 * np.max(np.abs(f)))
    lhs, rhs = float(w @ jv), float(jtw @ v)
    scale = np.linalg.norm(w) * np.linalg.norm(jv)
    assert abs(lhs - rhs) <= 1e-10 * scale, (lhs, rhs)


@pytest.mark.parametrize("case", ["1d_surface", "2d_cylinder", "3d_periodic_melt", "3d_fcc_colloid",
                                  "3d_hex_colloid", "3d_stencils_melt", "1d_branched", "2d_branched",
                                  "3d_branched", "1d_comb_branched", "1d_ring", "1d_dendrimer",
                                  "2d_dendrimer"])
def test_gradient_of_half_squared_norm(gpu_lib, case):
    spec = CASES[case]()
    s = System(spec)
    x = random_x(spec, seed=41, scale=0.2)
    f, g = s.vjp(x, s.residual(x))
    rng = np.random.default_rng(42)
    h = 1e-5
    for _ in range(4):
        d = rng.normal(size=s.nvar)
        phi_p = 0.5 * np.sum(s.residual(x + h * d) ** 2)
        phi_m = 0.5 * np.sum(s.residual(x - h * d) ** 2)
        fd = (phi_p - phi_m) / (2 * h)
        assert abs(fd - g @ d) <= 1e-7 * np.linalg.norm(g) * np.linalg.norm(d), (fd, g @ d)


@pytest.mark.parametrize("case", ["3d_2nd_brush", "3d_2nd_fcc_brush", "1d_2nd_lumped", "2d_2nd_lumped",
                                  "2d_2nd_lumped_periodic", "1d_cyl_2nd_lumped", "1d_sphere_2nd_lumped",
                                  "2d_cyl_2nd_lumped", "3d_2nd_stiff_copol"])
def test_second_order_dot_product_and_gradient(gpu_lib, case):
    """Second-order (six-direction) reverse sweep on the pinned 3D brush (and
    on the FCC lattice type, whose contact averages span the 27-site cube):
    <w, J v> = <J^T w, v> against the forward-mode tangent, and the gradient
    of |f|^2/2 against central differences."""
    spec = CASES[case]()
    s = System(spec)
    x = random_x(spec, seed=71, scale=0.2)
    rng = np.random.default_rng(72)
    v, w = rng.normal(size=s.nvar), rng.normal(size=s.nvar)
    f, jv = s.jvp(x, v)
    f2, jtw = s.vjp(x, w)
    np.testing.assert_allclose(f2, f, rtol=0, atol=1e-12 * np.max(np.abs(f)))
    assert abs(float(w @ jv) - float(jtw @ v)) <= 1e-10 * np.linalg.norm(w) * np.linalg.norm(jv)
    _, g = s.vjp(x, f)
    h = 1e-5
    for _ in range(3):
        d = rng.normal(size=s.nvar)
        fd = (0.5 * np.sum(s.residual(x + h * d) ** 2) - 0.5 * np.sum(s.residual(x - h * d) ** 2)) / (2 * h)
        assert abs(fd - g @ d) <= 1e-7 * np.linalg.norm(g) * np.linalg.norm(d), (fd, g @ d)
    s.set_checkpoint(4)
    f3, jtw3 = s.vjp(x, w)
    assert np.array_equal(f3, f2)
    np.testing.assert_allclose(jtw3, jtw, rtol=0, atol=1e-12 * np.max(np.abs(jtw)))


def test_lbfgs_c1(gpu_lib):
    spec, x0 = configs.flat_adsorption()
    s = System(spec)
    r = s.solve_lbfgs(x0, tol=1e-9, maxit=4000, m=20)
    assert r.converged, (r.status, r.error, r.iterations)
    o = Oracle(spec)
    assert np.linalg.norm(o.residual(r.x)) < 1e-8
    xd, rc, _, _ = o.solve_diis(x0, tol=1e-10, maxit=5000, m=10, eta=0.5)
    phi_l = o.phi(1).copy()
    o.residual(xd)
    np.testing.assert_allclose(phi_l, o.phi(1), rtol=1e-6, atol=1e-12)


@pytest.mark.parametrize("case", ["1d_surface", "1d_periodic_restricted", "2d_flat_surface", "3d_mirror_mix"])
def test_checkpointed_reverse_sweep(gpu_lib, case):
    """Checkpoints every k positions with segments recomputed on demand give
    the stored-slice result: f bit for bit (same kernels, same order), J^T w
    to the last bits (the transposed stencil scatters with FP64 atomics,
    whose order varies between runs)."""
    spec = CASES[case]()
    s = System(spec)
    x = random_x(spec, seed=51, scale=0.2)
    w = np.random.default_rng(52).normal(size=s.nvar)
    f0, g0 = s.vjp(x, w)
    tol = 1e-12 * np.max(np.abs(g0))
    for k in (1, 2, 3, 5, 1000):
        s.set_checkpoint(k)
        f, g = s.vjp(x, w)
        assert np.array_equal(f, f0), k
        np.testing.assert_allclose(g, g0, rtol=0, atol=tol, err_msg=str(k))
    s.set_checkpoint(0)
    f, g = s.vjp(x, w)
    np.testing.assert_allclose(g, g0, rtol=0, atol=tol)


def test_lbfgs_with_checkpoints_c1(gpu_lib):
    spec, x0 = configs.flat_adsorption()
    s = System(spec)
    s.set_checkpoint(10)
    r = s.solve_lbfgs(x0, tol=1e-9, maxit=4000, m=20)
    assert r.converged, (r.status, r.error, r.iterations)
    assert np.linalg.norm(Oracle(spec).residual(r.x)) < 1e-8


@pytest.mark.parametrize("case", ["1d_surface", "2d_cylinder", "3d_mirror_mix", "3d_2nd_brush", "3d_hex_colloid",
                                  "3d_stencils_colloid"])
def test_chi_gradient_against_differences(gpu_lib, case):
    """d(w.f)/d chi at fixed x against central differences of w.f with chi
    changed symmetrically (chi(a,b) = chi(b,a) += h).  f is linear in chi at
    fixed x, so the difference quotient is exact up to rounding; pairs whose
    change would merge or split classes of equal chi rows are skipped."""
    spec = CASES[case]()
    s = System(spec)
    x = random_x(spec, seed=61, scale=0.2)
    w = np.random.default_rng(62).normal(size=s.nvar)
    d = s.vjp_chi(x, w)
    ns = len(spec.segments)
    h = 1e-3
    checked = 0
    for a in range(ns):
        for b in range(a + 1, ns):
            vals = []
            for sgn in (1, -1):
                sp = CASES[case]()
                sp.chi = np.array(spec.chi, dtype=float).copy()
                sp.chi[a, b] += sgn * h
                sp.chi[b, a] += sgn * h
                s2 = System(sp)
                if s2.nclass != s.nclass:
                    break
                vals.append(float(w @ s2.residual(x)))
            if len(vals) < 2:
                continue
            fd = (vals[0] - vals[1]) / (2 * h)
            got = d[a, b] + d[b, a]
            assert abs(fd - got) <= 1e-8 * max(1.0, abs(fd)), (a, b, fd, got)
            checked += 1
    assert checked >= 2


class ResidualRev(torch.autograd.Function):
    """f(x) of one system with its reverse-mode derivative from sfgpu_vjp
    (test harness only): backward(grad_f) returns J(x)^T grad_f."""

    @staticmethod
    def forward(ctx, x, sys_):
        xn = x.detach().cpu().numpy()
        ctx.x, ctx.sys_ = xn, sys_
        return torch.from_numpy(sys_.residual(xn))

    @staticmethod
    def backward(ctx, grad_f):
        _, xbar = ctx.sys_.vjp(ctx.x, grad_f.detach().cpu().numpy())
        return torch.from_numpy(xbar), None


@pytest.mark.parametrize("case", ["1d_lambda_chi", "2d_cylinder", "3d_2nd_brush"])
def test_autograd_function_reverse_mode(gpu_lib, case):
    """torch.autograd.gradcheck (central differences, eps 1e-6) of the
    residual with its adjoint as backward, on a random subspace of x so
    that the check stays small."""
    spec = CASES[case]()
    s = System(spec)
    x0 = random_x(spec, seed=81, scale=0.2)
    rng = np.random.default_rng(82)
    B = torch.tensor(rng.normal(size=(s.nvar, 3)) / np.sqrt(s.nvar))
    base = torch.tensor(x0)

    def f_of(a):
        return ResidualRev.apply(base + B @ a, s)

    a = torch.zeros(3, dtype=torch.float64, requires_grad=True)
    # the transposed stencil scatters with FP64 atomics: repeated backward
    # calls agree to rounding, not bit for bit
    assert torch.autograd.gradcheck(f_of, (a,), eps=1e-6, atol=1e-6, rtol=1e-5, fast_mode=False, nondet_tol=1e-12)


def test_auto_checkpoint_stride(gpu_lib):
    spec = CASES["1d_surface"]()
    s = System(spec)
    x = random_x(spec, seed=91, scale=0.2)
    w = np.random.default_rng(92).normal(size=s.nvar)
    _, g0 = s.vjp(x, w)
    s.set_checkpoint(-1)
    _, g = s.vjp(x, w)
    np.testing.assert_allclose(g, g0, rtol=0, atol=1e-12 * np.max(np.abs(g0)))


@pytest.mark.parametrize("case", ["1d_surface", "1d_lambda_chi", "1d_periodic_restricted", "2d_cylinder",
                                  "2d_flat_surface", "3d_mirror_mix", "3d_2nd_brush", "3d_fcc_colloid",
                                  "3d_hex_mirror", "3d_stencils_colloid", "1d_branched", "3d_branched",
                                  "1d_comb_branched", "1d_ring", "1d_dendrimer"])
def test_free_energy_gradient(gpu_lib, case):
    """dF/dx from the reverse sweep against central differences of F
    (h = 1e-5) along random directions; F itself equals sfgpu_free_energy
    after a residual at the same x."""
    spec = CASES[case]()
    s = System(spec)
    x = random_x(spec, seed=101, scale=0.2)
    F, g = s.free_energy_grad(x)
    s.residual(x)
    assert F == pytest.approx(s.free_energy(), rel=1e-13, abs=1e-13)

    def F_at(y):
        s.residual(y)
        return s.free_energy()

    rng = np.random.default_rng(102)
    h = 1e-5
    for _ in range(4):
        d = rng.normal(size=s.nvar)
        fd = (F_at(x + h * d) - F_at(x - h * d)) / (2 * h)
        assert abs(fd - g @ d) <= 1e-7 * np.linalg.norm(g) * np.linalg.norm(d) + 1e-9 * abs(F), (fd, g @ d)


def test_phi_sensitivity_to_chi(gpu_lib):
    """dL/dchi for L = omega . phi_A at a converged C1-shaped solution,
    through the solution's dependence on chi (adjoint GMRES on J^T), against
    central differences of L between solutions re-converged (Newton-Krylov,
    |f| < 1e-12) with chi(a,b) = chi(b,a) changed by +-1e-4."""
    def build(dchi=None):
        spec, x0 = configs.flat_adsorption(n=40, N=20)
        if dchi is not None:
            a, b, h = dchi
            spec.chi = np.array(spec.chi, dtype=float).copy()
            spec.chi[a, b] += h
            spec.chi[b, a] += h
        return spec, x0

    spec, x0 = build()
    s = System(spec)
    r = s.solve_nk(x0, tol=1e-12, maxit=100, krylov=40)
    assert r.converged
    iA = spec.segment_index("A")
    omega = np.zeros((len(spec.segments), s.M))
    omega[iA] = np.random.default_rng(111).normal(size=s.M)
    d, relres = s.phi_sensitivity_chi(r.x, omega, rtol=1e-11)
    assert relres < 1e-10
    h = 1e-4
    for other in ("W", "S"):
        j = spec.segment_index(other)
        vals = []
        for sgn in (1, -1):
            sp, _ = build((iA, j, sgn * h))
            s2 = System(sp)
            r2 = s2.solve_nk(r.x, tol=1e-12, maxit=100, krylov=40)
            assert r2.converged
            vals.append(float(np.sum(omega[iA] * s2.phi(iA))))
        fd = (vals[0] - vals[1]) / (2 * h)
        got = d[iA, j] + d[j, iA]
        assert abs(fd - got) <= 1e-5 * max(abs(fd), 1e-8), (other, fd, got)


def test_c3_full_size_gradient_at_64_sites(gpu_lib):
    """The differentiation configuration at its stated size: Lat3D1stO 128^3
    periodic, (A)50(B)50 melt at chi_AB 0.2, seeded uniform start in
    [-0.05, 0.05].  The gradient of |f|^2/2 from the adjoint sweep with sqrt(N)
    checkpoints (stride 10) and the forward-mode J*e_i, at 64 random sites,
    against central finite differences with h = 1e-6; the checkpointed sweep
    equals the stored one."""
    spec, x0 = configs.melt3d()
    s = System(spec)
    s.set_checkpoint(10)
    f = s.residual(x0)
    _, g = s.vjp(x0, f)
    s.set_checkpoint(0)
    _, g_stored = s.vjp(x0, f)
    np.testing.assert_allclose(g, g_stored, rtol=0, atol=1e-12 * np.max(np.abs(g_stored)))
    rng = np.random.default_rng(64)
    idx = rng.choice(s.nvar, size=64, replace=False)
    h = 1e-6
    gscale = np.max(np.abs(g))
    for i in idx:
        e = np.zeros(s.nvar)
        e[i] = 1.0
        fp, fm = s.residual(x0 + h * e), s.residual(x0 - h * e)
        fd_grad = (0.5 * np.sum(fp ** 2) - 0.5 * np.sum(fm ** 2)) / (2 * h)
        assert abs(fd_grad - g[i]) <= 1e-6 * gscale, (i, fd_grad, g[i])
        _, jv = s.jvp(x0, e)
        fd_jv = (fp - fm) / (2 * h)
        assert np.max(np.abs(jv - fd_jv)) <= 1e-6 * max(np.max(np.abs(fd_jv)), 1e-12), i


def test_checkpoint_stride_by_measurement(gpu_lib):
    """The measured checkpoint stride (sfgpu_system_autotune_checkpoint)
    respects the memory bound it is given and leaves J^T w unchanged."""
    spec = CASES["1d_surface"]()
    s = System(spec)
    x = random_x(spec, seed=61, scale=0.2)
    w = np.random.default_rng(62).normal(size=s.nvar)
    f0, g0 = s.vjp(x, w)
    k, ms = s.autotune_checkpoint(x, reps=2)
    assert k >= 0 and ms > 0
    f1, g1 = s.vjp(x, w)
    assert np.array_equal(f0, f1)
    np.testing.assert_allclose(g1, g0, rtol=0, atol=1e-12 * np.max(np.abs(g0)))
    # a bound below full storage (2N slices) forces checkpoints
    N = max(m.N for m in spec.molecules)
    slice_bytes = 8.0 * spec.M
    bound = 0.75 * 2 * N * slice_bytes
    k2, _ = s.autotune_checkpoint(x, reps=1, max_bytes=bound)
    assert k2 > 0
    nq = -(-N // k2)
    assert (2 * nq + 2 * k2 + 1) * slice_bytes <= bound
    f2, g2 = s.vjp(x, w)
    np.testing.assert_allclose(g2, g0, rtol=0, atol=1e-12 * np.max(np.abs(g0)))
