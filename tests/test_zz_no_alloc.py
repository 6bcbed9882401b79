"""The allocation-free chain entry point (sfgpu_chain_phi_noalloc) against
the system path, through the C ABI.

It serves callers that cannot allocate device memory; its output must equal
what the ordinary path computes for the same chain: the molecule profile of
sfgpu_residual divided by the free normalisation phibulk/N, and the same
lnGN.  Two calls in a row check that the shared scratch array carries no
state from one call to the next.  Kept in a file of its own that pytest
collects last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from field_b200 import _native, configs
from field_b200.desc import MOL_FREE
from field_b200.system import System

from cases import CASES

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _run_noalloc(lib, spec, mol, G_dev, phi_dev, lngn_dev, stream):
    segs = np.array([b[0] for b in mol.blocks for _ in range(b[1])], dtype=np.int32)
    ns = len(spec.segments)
    g_ptrs = (C.c_void_p * ns)(*[C.c_void_p(t.data_ptr()) if t is not None else None for t in G_dev])
    p_ptrs = (C.c_void_p * ns)(*[C.c_void_p(t.data_ptr()) if t is not None else None for t in phi_dev])
    lat = spec.lattice.to_c()
    return lib.sfgpu_chain_phi_noalloc(C.byref(lat), len(segs), segs.ctypes.data_as(C.POINTER(C.c_int)), ns,
                                       g_ptrs, p_ptrs, C.c_void_p(lngn_dev.data_ptr()), C.c_void_p(stream))


def _flat1d_layer_adjustment():
    spec, _ = configs.flat_adsorption(n=30, N=21, phib=0.02, chi_aw=0.6, chi_as=-1.2)
    spec.lattice.layer_adjustment = 0.8
    return spec


# one case per family of lattice tables the call builds: the 2D cylinder
# (radial lambda tables), the 1D flat lattice with a surface and a layer
# adjustment in the lnGN weights, the 1D sphere around a colloid (curved
# tables with an offset), a 3D FCC box (twelve-neighbour step)
NOALLOC_CASES = {
    "2d_cylinder": lambda: configs.cyl_micelle(nx=40, ny=36, nA=12, nB=9, radius=5)[0],
    "1d_flat_layer_adjustment": _flat1d_layer_adjustment,
    "1d_sphere_colloid": lambda: CASES["1d_sphere_colloid"](),
    "3d_fcc_colloid": lambda: CASES["3d_fcc_colloid"](),
}


@pytest.mark.parametrize("name", sorted(NOALLOC_CASES))
def test_noalloc_chain_matches_system_path(gpu_lib, name):
    lib = _native.load()
    spec = NOALLOC_CASES[name]()
    mol_index = 0
    mol = spec.molecules[mol_index]
    assert mol.freedom == MOL_FREE
    rng = np.random.default_rng(2024)
    x = rng.normal(0.0, 0.3, spec.n_itvar())
    ref = System(spec)
    ref.residual(x)
    want_lngn = ref.mol_scalars(mol_index)["lngn"]
    norm = mol.phibulk / mol.N
    used = sorted({b[0] for b in mol.blocks})
    G_dev = [None] * len(spec.segments)
    for i in used:
        G_dev[i] = torch.tensor(ref.swf(i), device="cuda")
    want = {i: ref.mol_phi(mol_index, i) for i in used}
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        phi_dev = [None] * len(spec.segments)
        for i in used:
            # stale values in the outputs must not leak into the result
            phi_dev[i] = torch.full((spec.M,), 7.0 + call, device="cuda", dtype=torch.float64)
        lngn_dev = torch.zeros(1, device="cuda", dtype=torch.float64)
        torch.cuda.synchronize()
        rc = _run_noalloc(lib, spec, mol, G_dev, phi_dev, lngn_dev, stream)
        assert rc == 0, _native.last_error()
        torch.cuda.synchronize()
        assert abs(lngn_dev.item() - want_lngn) <= 1e-12 * max(1.0, abs(want_lngn))
        for i in used:
            got = phi_dev[i].cpu().numpy() * norm
            np.testing.assert_allclose(got, want[i], rtol=RTOL, atol=1e-300)


def test_noalloc_rejects_chains_beyond_the_scratch_limit(gpu_lib):
    lib = _native.load()
    spec, _ = configs.cyl_micelle(nx=128, ny=128, nA=100, nB=100)   # 200 x 16900 values > 2M doubles
    mol = spec.molecules[0]
    dummy = torch.zeros(spec.M, device="cuda", dtype=torch.float64)
    G_dev = [dummy, dummy, None]
    phi_dev = [dummy.clone(), dummy.clone(), None]
    lngn_dev = torch.zeros(1, device="cuda", dtype=torch.float64)
    rc = _run_noalloc(lib, spec, mol, G_dev, phi_dev, lngn_dev, torch.cuda.current_stream().cuda_stream)
    assert rc == 1   # SFGPU_ERR_INVALID, nothing queued
    assert torch.count_nonzero(phi_dev[0]).item() == 0
