"""The lattice-level C ABI as a drop-in for SFbox's Matrix1 loop.

A caller that keeps its own chain loop (SF_Copol1stO::Matrix1,
SF_Copol1stO.cpp:1187-1281; SF_Copol2ndO::Matrix1, SF_Copol2ndO.cpp:250-356)
calls sfgpu_lat_propagate per chain position and then sfgpu_lat_connect,
sfgpu_lat_correct_double_count and sfgpu_lat_norm_phi_free / _restr.  Run
that loop here on device tensors and compare the molecule's profiles with the
ones the library's own molecule driver computes inside sfgpu_residual.
"""
import os
import sys

import numpy as np
import pytest
import torch

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from reference_inputs import INPUTS  # noqa: E402
from field_b200.desc import MOL_FREE, MOL_RESTRICTED  # noqa: E402
from field_b200.sfinput import build_system, parse_input  # noqa: E402

pytestmark = pytest.mark.gpu

# (input case, molecule index): free and restricted chains, first order on
# 1D/2D/3D lattices, second order in 3D (K = 6) and lumped in 2D (K = 5)
LOOPS = [("1d_flat_surface", 0), ("1d_flat_mirror2", 0), ("1d_flat_mirror2", 1), ("2d_cylinder_core", 0),
         ("3d_mirror_colloid", 0), ("3d_2nd_palindrome", 0), ("2d_2nd_lumped", 0), ("2d_2nd_lumped", 1)]


def _chain(mol):
    return [b[0] for b in mol.blocks for _ in range(b[1])]


@pytest.mark.parametrize("case,mi", LOOPS)
def test_matrix1_loop_through_the_lattice_calls(gpu_lib, case, mi):
    from field_b200.system import System
    spec, _ = build_system(parse_input(INPUTS[case])[0])
    s = System(spec)
    x = np.random.default_rng(11).normal(0.0, 0.3, s.nvar)
    s.residual(x)
    mol = spec.molecules[mi]
    assert mol.freedom in (MOL_FREE, MOL_RESTRICTED)
    K = spec.lattice.components
    M = spec.M
    seg = _chain(mol)
    N = len(seg)
    pf = spec.pf if spec.pf is not None else np.full((len(spec.segments),) * 2, 0.2)
    G = {i: torch.tensor(s.swf(i), device="cuda") for i in set(seg)}
    GK = {i: G[i].repeat(K) for i in G}
    # forward: Gi[.,1] = G(seg 1), Gi[.,s] = step(Gi[.,s-1]) with S = Pf(s-1, s)
    gf = [GK[seg[0]].clone()]
    for t in range(1, N):
        gf.append(s.propagate(gf[-1], G[seg[t]], S=pf[seg[t - 1], seg[t]], backward=False))
    # backward with composition, then CorrectDoubleCountG and the norm
    phi = {i: torch.zeros(M, device="cuda", dtype=torch.float64) for i in set(seg)}
    gb = GK[seg[N - 1]].clone()
    s.connect(gb, gf[N - 1], phi[seg[N - 1]])
    for t in range(N - 2, -1, -1):
        gb = s.propagate(gb, G[seg[t]], S=pf[seg[t], seg[t + 1]], backward=True)
        s.connect(gb, gf[t], phi[seg[t]])
    for i in phi:
        s.correct_double_count(phi[i], G[i])
    lngn = s.lngn(gb)
    assert abs(lngn - s.mol_scalars(mi)["lngn"]) <= 1e-12 * max(1.0, abs(lngn))
    for i in phi:
        if mol.freedom == MOL_FREE:
            s.norm_phi_free(phi[i], mol.phibulk / (N * (6.0 if K > 1 else 1.0)))
        else:
            s.norm_phi_restr(phi[i], gb, mol.theta / N)
    inner = spec.lattice.interior_mask()
    for i in phi:
        got = phi[i].cpu().numpy()[inner]
        want = s.mol_phi(mi, i)[inner]
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-15 * np.max(np.abs(want)))


def test_log_space_lattices_refuse_the_lattice_calls(gpu_lib):
    from field_b200.system import System
    spec, _ = build_system(parse_input(INPUTS["1d_flat_overflow"])[0])
    s = System(spec)
    p = torch.zeros(spec.M, device="cuda", dtype=torch.float64)
    rc = s.lib.sfgpu_lat_norm_phi_free(s.h, __import__("ctypes").c_void_p(p.data_ptr()), 1.0)
    assert rc == 7   # SFGPU_ERR_UNSUPPORTED
