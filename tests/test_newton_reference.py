"""SFbox's Newton iteration (the plain Newton form) against SFbox itself.

The library's restatement of SFNewton::iterate (field_b200/csrc/sfgpu_newton.h)
runs on the CPU over the oracle's residual (a test harness compiled here) and
on the GPU over the device residual (sfgpu_solve_newton).  Both must reach
SFbox's own Newton solution (tests/golden/reference_cases.npz, written by the
reference's sources) from x = 0 with tolerance 1e-12, for the default
'pseudohessian' method and for 'hessian': phi within 1e-10 and F within 1e-9
relative.  Over the oracle the iterations are SFbox's own (same count, x to
1e-12); over the device residual the count may differ by two (the residuals
agree to rounding, not bit for bit).
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(HERE, "golden"))

from make_reference_golden import NEWTON_CASES, NEWTON_METHODS, newton_input  # noqa: E402
from reference_inputs import INPUTS  # noqa: E402
from field_b200.desc import NewtonSettings  # noqa: E402
from field_b200.sfinput import build_system, parse_input  # noqa: E402

with np.load(os.path.join(HERE, "golden", "reference_cases.npz")) as _z:
    DATA = {k: _z[k] for k in _z.files if "/newton_" in k}

PARAMS = [(c, m) for c in NEWTON_CASES for m in NEWTON_METHODS]


def _settings(method):
    st = NewtonSettings()
    st.tolerance, st.iterationlimit, st.pseudohessian = 1e-12, 5000, int(method == "pseudohessian")
    st.deltamax, st.deltamin, st.linesearchlimit = 0.5, 0.0, 20
    st.small_alpha, st.max_n_small_alpha = 1e-5, 50
    st.reset_hessian_criterion, st.max_accuracy_for_hessian_scaling = 1e3, 0.1
    st.ignore_newton_direction = 0
    return st


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    from oracle import oracle as orc
    orc.build()
    so = str(tmp_path_factory.mktemp("newton") / "libnewton_on_oracle.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", so,
                    os.path.join(HERE, "newton", "newton_on_oracle.cpp"),
                    os.path.join(ROOT, "oracle", "liboracle.so"), f"-Wl,-rpath,{os.path.join(ROOT, 'oracle')}"],
                   check=True)
    lib = C.CDLL(so)
    lib.newton_on_oracle.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_void_p,
                                     C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)]
    return lib


def _check(spec, case, method, it, phi_of, F, it_slack=2):
    inner = spec.lattice.interior_mask()
    want = DATA[f"{case}/newton_{method}_phi"]
    for i in range(len(spec.segments)):
        w = want[i][inner]
        if np.max(np.abs(w)) > 0:
            assert np.max(np.abs(phi_of(i)[inner] - w)) <= 1e-10 * np.max(np.abs(w)), (case, method, i)
    Fw = DATA[f"{case}/newton_{method}_F"][0]
    assert abs(F - Fw) <= 1e-9 * max(1.0, abs(Fw)), (case, method, F, Fw)
    assert abs(it - DATA[f"{case}/newton_{method}_iterations"][0]) <= it_slack, (case, method, it)


@pytest.mark.parametrize("case,method", PARAMS)
def test_newton_on_oracle_reaches_sfbox_newton(harness, case, method):
    from oracle.oracle import Oracle
    spec, _ = build_system(parse_input(newton_input(INPUTS[case], method))[0])
    o = Oracle(spec)
    x = np.zeros(o.nvar)
    st = _settings(method)
    it, nf, acc = C.c_int(), C.c_int(), C.c_double()
    rc = harness.newton_on_oracle(o.h, o.nvar, x.ctypes.data_as(C.POINTER(C.c_double)), C.byref(st),
                                  C.byref(it), C.byref(nf), C.byref(acc))
    assert rc == 0 and acc.value <= 1e-12, (rc, acc.value, it.value)
    # the oracle's residual follows SFbox's to rounding: the same iterations
    np.testing.assert_allclose(x, DATA[f"{case}/newton_{method}_x"], rtol=0, atol=1e-12)
    o.residual(x)
    _check(spec, case, method, it.value, o.phi, o.free_energy(), it_slack=0)


@pytest.mark.gpu
@pytest.mark.parametrize("case,method", PARAMS)
def test_gpu_newton_reaches_sfbox_newton(gpu_lib, case, method):
    from field_b200.system import System
    spec, _ = build_system(parse_input(newton_input(INPUTS[case], method))[0])
    s = System(spec)
    r = s.solve_newton(np.zeros(s.nvar), tol=1e-12, maxit=5000, pseudohessian=(method == "pseudohessian"))
    assert r.converged, (r.status, r.iterations, r.error)
    s.residual(r.x)
    _check(spec, case, method, r.iterations, s.phi, s.free_energy())
