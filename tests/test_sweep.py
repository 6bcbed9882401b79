"""var : sweeps (Vary.cpp): the sequence of values and the calculations a
sweep expands into (host logic, no GPU)."""
import numpy as np
import pytest

from field_b200 import configs
from field_b200.sfinput import build_system, parse_input
from field_b200.sweep import expand_variation, sweep_calculations

BASE = configs.C1_INPUT.format(n=20, N=10, phib=0.01, chi_aw=0.5, chi_as=-1.0)


def _calc(extra):
    # the base text ends its calculation with 'start'; the var statements
    # open the next one, which inherits everything before them
    return parse_input(BASE + extra)[-1]


def test_no_var_is_one_calculation():
    var, calcs = sweep_calculations(_calc(""))
    assert var is None and len(calcs) == 1


def test_linear_real_clamps_last_step_to_end_value():
    """0.5 -> 1.0 in steps of 0.15: 0.5, 0.65, 0.8, 0.95, then the step
    overshoots and the last value is clamped to 1.0 (Vary.cpp:154-158)."""
    v = expand_variation(_calc("var : mon : A : chi - W\nvar : mon : step : 0.15\n"
                               "var : mon : end_value : 1.0\nvar : mon : type : real\n"))
    assert v.parameter == "chi - W"
    np.testing.assert_allclose(v.values, [0.5, 0.65, 0.8, 0.95, 1.0], rtol=0, atol=1e-15)


def test_decreasing_sweep():
    """A negative step runs downwards; a step pointing away from end_value
    gives at most one calculation and is rejected (Vary.cpp:71-79)."""
    v = expand_variation(_calc("var : mol : pol : phibulk\nvar : mol : step : -0.002\n"
                               "var : mol : end_value : 0.004\nvar : mol : type : real\n"))
    np.testing.assert_allclose(v.values, [0.01, 0.008, 0.006, 0.004], rtol=1e-12)


def test_exponential_steps_per_decade():
    """scale exponential: step = points per decade, value *= 10^(1/step)."""
    v = expand_variation(_calc("var : mol : pol : phibulk\nvar : mol : step : 2\nvar : mol : scale : exponential\n"
                               "var : mol : end_value : 1e-4\nvar : mol : type : real\n"))
    want = [0.01, 0.01 / 10 ** 0.5, 0.001, 0.001 / 10 ** 0.5, 1e-4]
    np.testing.assert_allclose(v.values, want, rtol=1e-12)


def test_integer_type_steps_until_the_integer_changes():
    """type integer: fractional steps advance until int() changes
    (Vary.cpp:147-151), and the sweep stops at end_value."""
    v = expand_variation(_calc("var : lat : flat : n_layers\nvar : lat : step : 2.5\n"
                               "var : lat : end_value : 30\nvar : lat : type : integer\n"))
    assert v.values == [20, 22, 25, 27, 30]


def test_sweep_calculations_set_the_parameter():
    var, calcs = sweep_calculations(_calc("var : mon : A : chi - W\nvar : mon : step : 0.25\n"
                                          "var : mon : end_value : 1.0\nvar : mon : type : real\n"))
    specs = [build_system(c)[0] for c in calcs]
    assert [s.chi[1, 2] for s in specs] == [0.5, 0.75, 1.0]
    assert all(("var", "mon", "step") not in c for c in calcs)


@pytest.mark.parametrize("extra", ["var : mon : A : chi - S\nvar : mon : step : 0.1\nvar : mon : type : real\n",
                                   "var : mon : A : chi - X\nvar : mon : step : 0.1\nvar : mon : end_value : 1\n"
                                   "var : mon : type : real\n",
                                   "var : mon : A : chi - W\nvar : mon : step : -0.1\nvar : mon : end_value : 0.5\n"
                                   "var : mon : type : real\n"])
def test_invalid_variations_are_rejected(extra):
    with pytest.raises(ValueError):
        expand_variation(_calc(extra))


def test_batchable_routes_special_systems_to_the_single_system_path():
    import sys, os
    sys.path.insert(0, os.path.dirname(__file__))
    from cases import CASES
    from field_b200.sweep import batchable
    for k in ("1d_surface", "1d_force", "3d_fcc_colloid", "3d_hex_colloid", "3d_stencils_melt"):
        assert batchable(CASES[k]()), k   # the wide kernel takes the lattice types and the force
    for k in ("1d_dendrimer", "3d_2nd_brush", "2d_2nd_lumped"):
        assert not batchable(CASES[k]()), k
    spec = CASES["1d_surface"]()
    spec.overflow_protection = True
    assert not batchable(spec)
