"""Batched persistent solver: every instance matches the single-system
Pure_DIIS path and the oracle (same algorithm, same iterates up to the order
of floating-point reductions)."""
import numpy as np
import pytest

from field_b200 import configs
from field_b200.batch import BatchSolver
from field_b200.system import System
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def test_batch_uneven_sweep_matches_oracle(gpu_lib):
    """Uneven 1D instances (config C4 shapes, smaller N) in one launch."""
    insts = configs.sweep1d(count=24, N_range=(20, 200))
    specs = [s for s, _ in insts]
    bs = BatchSolver(specs, m=5, eta=0.1)
    x0 = np.concatenate([x for _, x in insts])
    res = bs.solve(x0, tol=1e-9, maxit=3000)
    assert res.converged.all(), (res.status, res.errors)
    for i, (spec, x) in enumerate(insts):
        o = Oracle(spec)
        xi = bs.split(res.x)[i]
        f = o.residual(xi)
        assert np.linalg.norm(f) < 1e-8
        for seg in range(len(spec.segments)):
            np.testing.assert_allclose(bs.phi(i, seg), o.phi(seg), rtol=1e-9, atol=1e-13)


def test_batch_equals_single_system(gpu_lib):
    """C2-shaped instances (small cylinder): batched and plain forms follow
    the same Pure_DIIS iterates."""
    insts = [configs.cyl_micelle(nx=30, ny=24, nA=8, nB=8, radius=4, seed=100 + i) for i in range(6)]
    bs = BatchSolver([s for s, _ in insts], m=10, eta=0.1)
    res = bs.solve(np.concatenate([x for _, x in insts]), tol=1e-8, maxit=2000)
    assert res.converged.all()
    for i, (spec, x0) in enumerate(insts):
        r = System(spec).solve(x0, tol=1e-8, maxit=2000, m=10, eta=0.1)
        assert r.converged
        assert abs(r.iterations - res.iterations[i]) <= 2
        np.testing.assert_allclose(bs.split(res.x)[i], r.x, rtol=0, atol=1e-7)


def test_batch_reports_nonconvergence(gpu_lib):
    insts = [configs.flat_adsorption(n=20, N=10)] * 1 + [configs.flat_adsorption(n=30, N=50, phib=0.05)]
    bs = BatchSolver([configs.flat_adsorption(n=20, N=10)[0], configs.flat_adsorption(n=30, N=50, phib=0.05)[0]],
                     m=5, eta=0.1)
    x0 = np.zeros(bs.total)
    res = bs.solve(x0, tol=1e-12, maxit=3)
    assert (res.status == 5).all() and (res.iterations == 3).all()
