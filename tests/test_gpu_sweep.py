"""var : sweeps solved as batched instances (field_b200.sweep) on the GPU."""
import numpy as np
import pytest

from field_b200 import configs
from field_b200.sfinput import parse_input
from field_b200.sweep import solve_sweep
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

SWEEP = (configs.C1_INPUT.format(n=40, N=20, phib=0.01, chi_aw=0.0, chi_as=-1.0)
         + "var : mon : A : chi - W\nvar : mon : step : 0.1\nvar : mon : end_value : 0.8\nvar : mon : type : real\n"
         + "newton : isaac : tolerance : 1e-9\n")


def test_sweep_schedules_agree(gpu_lib):
    """The 9 points of a chi sweep solved in one batch from zero, in three
    waves, and as SFbox's chain (each point from its predecessor): every point
    converges, satisfies the oracle's equations, and the three schedules reach
    the same solutions.  (At chi = 1 Pure_DIIS from zero fails on the oracle
    too, so the sweep stops at 0.8.  Pure_DIIS's first step replaces the
    guess by -eta g(guess), sfnewton.cpp:578-584, so a warm start changes
    only that first gradient and need not save iterations.)"""
    calc = parse_input(SWEEP)[-1]
    cold = solve_sweep(calc, waves=1, m=5)
    three = solve_sweep(calc, waves=3, m=5)
    chain = solve_sweep(calc, waves=100, m=5)
    assert len(cold.x) == 9 and (chain.wave == np.arange(9)).all()
    for res in (cold, three, chain):
        assert res.converged.all(), res.status
    for i, spec in enumerate(cold.specs):
        assert spec.chi[1, 2] == pytest.approx(0.1 * i)
        o = Oracle(spec)
        for res in (cold, three, chain):
            assert np.linalg.norm(o.residual(res.x[i])) < 1e-8
        np.testing.assert_allclose(three.x[i], cold.x[i], rtol=0, atol=1e-6)
        np.testing.assert_allclose(chain.x[i], cold.x[i], rtol=0, atol=1e-6)
    assert (three.wave == np.arange(9) % 3).all()
