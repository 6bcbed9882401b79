"""Reverse-mode derivative of the residual (J(x)^T w from the adjoint sweep)
and the L-BFGS iteration that uses it as the gradient of |f|^2 / 2.

The adjoint is checked by the dot-product identity <w, J v> = <J^T w, v>
against the forward-mode tangent (itself pinned to finite differences in
test_gpu_tangent.py), relative tolerance 1e-10 of |w| |J v|; directional
derivatives of |f|^2/2 against central differences; and the primal f of the
adjoint sweep against sfgpu_residual (1e-12 of max|f|: the sweep propagates
full chains where the residual may use the half-chain trick for symmetric
homopolymers).
"""
import numpy as np
import pytest

from cases import CASES, random_x
from field_b200 import configs
from field_b200._native import SfgpuError
from field_b200.system import System
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

FIRST_ORDER = sorted(k for k in CASES if "2nd" not in k)


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


@pytest.mark.parametrize("case", ["1d_surface", "2d_cylinder", "3d_periodic_melt"])
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


def test_second_order_is_rejected(gpu_lib):
    spec = CASES["3d_2nd_brush"]()
    s = System(spec)
    x = np.zeros(s.nvar)
    with pytest.raises(SfgpuError) as e:
        s.vjp(x, x)
    assert e.value.code == 7


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
