"""The committed fixtures of tests/golden (made by tests/golden/make_golden.py
from the oracle): the oracle must still produce them exactly, and the CUDA
path must meet them within the parity tolerances."""
import os

import numpy as np
import pytest

from cases import CASES

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "oracle_cases.npz")


def _load():
    with np.load(GOLDEN) as z:
        data = {k: z[k] for k in z.files}
    cases = sorted({k.split("/")[0] for k in data})
    return data, cases


DATA, GOLDEN_CASES = _load()


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_oracle_reproduces_golden(case):
    from oracle.oracle import Oracle
    spec = CASES[case]()
    o = Oracle(spec)
    x = DATA[f"{case}/x"]
    np.testing.assert_array_equal(o.residual(x), DATA[f"{case}/f"])
    phi = np.stack([o.phi(i) for i in range(len(spec.segments))])
    np.testing.assert_array_equal(phi, DATA[f"{case}/phi"])
    np.testing.assert_array_equal([o.lngn(m) for m in range(len(spec.molecules))], DATA[f"{case}/lngn"])
    assert o.free_energy() == DATA[f"{case}/F"][0]


@pytest.mark.gpu
@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_gpu_meets_golden(gpu_lib, case):
    from field_b200.system import System
    spec = CASES[case]()
    s = System(spec)
    x = DATA[f"{case}/x"]
    f = s.residual(x)
    want = DATA[f"{case}/f"]
    assert np.max(np.abs(f - want)) <= 1e-11 * max(1.0, np.max(np.abs(want)))
    phi = DATA[f"{case}/phi"]
    for i in range(len(spec.segments)):
        assert np.max(np.abs(s.phi(i) - phi[i])) <= 1e-11 * max(np.max(np.abs(phi[i])), 1e-300)
    for m, v in enumerate(DATA[f"{case}/lngn"]):
        assert abs(s.mol_scalars(m)["lngn"] - v) <= 1e-12 * max(1.0, abs(v))
    F = DATA[f"{case}/F"][0]
    assert abs(s.free_energy() - F) <= 1e-11 * max(1.0, abs(F))
