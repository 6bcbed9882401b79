"""CUDA path vs the CPU oracle on identical seeded inputs, through the C ABI.

Tolerances (FP64 throughout): single propagator steps and contact averages
agree to 1e-14 relative (the library is built without FMA contraction and
keeps SFbox's operation order); whole residual evaluations to 1e-11
relative (reductions and exp/log differ in the last bits); converged
profiles to 1e-10 in phi and 1e-9 in the free energy.
"""
import numpy as np
import pytest
import torch

from cases import CASES, random_x
from field_b200.system import System
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

TOL_STEP = 1e-14
TOL_EVAL = 1e-11


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("case", sorted(CASES))
def test_propagator_step(gpu_lib, case):
    spec = CASES[case]()
    sys_ = System(spec)
    o = Oracle(spec)
    rng = np.random.default_rng(3)
    K = sys_.K
    gin = o.set_boundaries(rng.uniform(0.2, 2.0, o.M)) if K == 1 else rng.uniform(0.2, 2.0, K * o.M)
    g = o.set_boundaries(rng.uniform(0.1, 1.5, o.M))
    for backward in ([0] if K == 1 else [0, 1]):
        want = o.propagate(gin, g, S=0.35, backward=backward)
        gin_t = torch.tensor(gin, device="cuda")
        if K > 1:
            sys_.set_boundaries(gin_t)
        got = sys_.propagate(gin_t, torch.tensor(g, device="cuda"), S=0.35, backward=bool(backward)).cpu().numpy()
        if K in (3, 5):
            # the lumped steps write interior entries only
            inner = np.zeros(spec.lattice.shape, bool)
            inner[(slice(1, -1),) * spec.lattice.gradients] = True
            inner = np.tile(inner.ravel(), K)
            got, want = got[inner], want[inner]
        assert rel(got, want) <= TOL_STEP, (case, backward, rel(got, want))


@pytest.mark.parametrize("case", sorted(CASES))
def test_side_fraction(gpu_lib, case):
    spec = CASES[case]()
    sys_ = System(spec)
    o = Oracle(spec)
    rng = np.random.default_rng(4)
    phi = o.set_boundaries(rng.uniform(0.0, 1.0, o.M))
    want = o.side(phi)
    got = sys_.side_fraction(torch.tensor(phi, device="cuda")).cpu().numpy()
    assert rel(got, want) <= TOL_STEP


@pytest.mark.parametrize("case", sorted(CASES))
def test_residual_and_profiles(gpu_lib, case):
    spec = CASES[case]()
    sys_ = System(spec)
    o = Oracle(spec)
    assert sys_.nvar == o.nvar and sys_.M == o.M
    x = random_x(spec)
    f_gpu = sys_.residual(x)
    f_cpu = o.residual(x)
    assert np.all(np.isfinite(f_gpu))
    assert rel(f_gpu, f_cpu) <= TOL_EVAL, rel(f_gpu, f_cpu)
    for i, seg in enumerate(spec.segments):
        assert rel(sys_.phi(i), o.phi(i)) <= TOL_EVAL, (seg.name, rel(sys_.phi(i), o.phi(i)))
    for m in range(len(spec.molecules)):
        sc = sys_.mol_scalars(m)
        assert abs(sc["lngn"] - o.lngn(m)) <= 1e-12 * max(1.0, abs(o.lngn(m)))
        assert abs(sc["phibulk"] - o.phibulk(m)) <= 1e-12 * max(1e-300, abs(o.phibulk(m))) + 1e-300


@pytest.mark.parametrize("case", sorted(CASES))
def test_free_energy(gpu_lib, case):
    spec = CASES[case]()
    sys_ = System(spec)
    o = Oracle(spec)
    x = random_x(spec, seed=11, scale=0.2)
    sys_.residual(x)
    o.residual(x)
    Fg, Fc = sys_.free_energy(), o.free_energy()
    assert abs(Fg - Fc) <= 1e-11 * max(1.0, abs(Fc)), (Fg, Fc)


def test_edge_single_layer_and_short_chains(gpu_lib):
    """Smallest lattices and chains: one interior layer, N = 1, 2, 3."""
    from field_b200 import configs
    for n, N in [(1, 2), (2, 3), (3, 1), (5, 2)]:
        spec, _ = configs.flat_adsorption(n=n, N=N)
        sys_ = System(spec)
        o = Oracle(spec)
        x = random_x(spec, seed=n * 10 + N)
        assert rel(sys_.residual(x), o.residual(x)) <= TOL_EVAL


def test_solve_c1_converged_parity(gpu_lib):
    """Config C1 converged by the device Pure_DIIS and by the oracle's: same
    algorithm, so the profiles agree to 1e-10 and the free energy to 1e-9."""
    from field_b200 import configs
    spec, x0 = configs.flat_adsorption()
    sys_ = System(spec)
    o = Oracle(spec)
    rg = sys_.solve(x0, tol=1e-10, maxit=5000, m=10, eta=0.5)
    xc, rc, it, err = o.solve_diis(x0, tol=1e-10, maxit=5000, m=10, eta=0.5)
    assert rg.converged and rc == 0
    sys_.residual(rg.x)
    o.residual(xc)
    for i in range(3):
        np.testing.assert_allclose(sys_.phi(i), o.phi(i), rtol=1e-10, atol=1e-12)
    assert abs(sys_.free_energy() - o.free_energy()) <= 1e-9
    # the converged residual of the GPU iterate is below tolerance on the oracle too
    assert np.linalg.norm(o.residual(rg.x)) < 1e-9


def test_full_size_c2_residual(gpu_lib):
    """Config C2 (Lat2DCyl1stO 128x128, A20B20, seeded micelle) at full size."""
    from field_b200 import configs
    spec, x0 = configs.cyl_micelle()
    sys_ = System(spec)
    o = Oracle(spec)
    f_gpu, f_cpu = sys_.residual(x0), o.residual(x0)
    assert rel(f_gpu, f_cpu) <= TOL_EVAL
    assert abs(sys_.free_energy() - o.free_energy()) <= 1e-10 * max(1.0, abs(o.free_energy()))


def test_full_size_c3_residual(gpu_lib):
    """Config C3 (Lat3D1stO 128^3 periodic, A50B50 melt) at full size: one
    residual against the oracle plus the sum rule sum_z phi = phibulk * GN."""
    from field_b200 import configs
    spec, x0 = configs.melt3d()
    sys_ = System(spec)
    o = Oracle(spec)
    f_gpu, f_cpu = sys_.residual(x0), o.residual(x0)
    assert rel(f_gpu, f_cpu) <= TOL_EVAL
    sites = spec.itvar_sites()
    tot = (sys_.phi(0) + sys_.phi(1))[sites].sum()
    gn = np.exp(sys_.mol_scalars(0)["lngn"])
    assert abs(tot - gn) < 1e-10 * gn


def test_brush_2nd_order_residual_48(gpu_lib):
    """Config C5 shape (Lat3D2ndO, grafted (X)1(A)199 brush, mirror walls,
    bending S=0.5) on a 48^3 lattice: residual, profiles and lnGN."""
    from field_b200 import configs
    spec, _ = configs.brush3d(n=48, N=200, sigma=0.05, S=0.5)
    rng = np.random.default_rng(77)
    x = rng.normal(0.0, 0.05, spec.n_itvar())
    sys_ = System(spec)
    o = Oracle(spec)
    f_gpu, f_cpu = sys_.residual(x), o.residual(x)
    assert rel(f_gpu, f_cpu) <= TOL_EVAL
    for i in range(len(spec.segments)):
        assert rel(sys_.phi(i), o.phi(i)) <= TOL_EVAL
    assert abs(sys_.mol_scalars(0)["lngn"] - o.lngn(0)) <= 1e-12 * abs(o.lngn(0))


def test_autotuned_tile_keeps_results(gpu_lib):
    """The 3D tile depth changes the launch shape only, not the numbers."""
    from field_b200 import configs
    spec, x0 = configs.melt3d(n=20, nA=6, nB=5)
    s = System(spec)
    f_ref = s.residual(x0)
    for xc in (1, 3, 7, 32):
        s.set_tile(xc)
        assert np.array_equal(s.residual(x0), f_ref)
    s.autotune(reps=3)
    assert np.array_equal(s.residual(x0), f_ref)


@pytest.mark.parametrize("case", ["1d_2nd_lumped", "2d_2nd_lumped", "1d_sphere_2nd_lumped", "2d_cyl_2nd_lumped"])
def test_lumped_second_order_converged_parity(gpu_lib, case):
    """Lat1D2ndO / Lat2D2ndO converged by the device Pure_DIIS and by the
    oracle's: profiles to 1e-10, free energy to 1e-9."""
    spec = CASES[case]()
    sys_ = System(spec)
    o = Oracle(spec)
    x0 = np.zeros(spec.n_itvar())
    rg = sys_.solve(x0, tol=1e-10, maxit=4000, m=8, eta=0.3)
    xc, rc, it, err = o.solve_diis(x0, tol=1e-10, maxit=4000, m=8, eta=0.3)
    assert rg.converged and rc == 0, (rg.converged, rc, err)
    sys_.residual(rg.x)
    o.residual(xc)
    for i in range(len(spec.segments)):
        np.testing.assert_allclose(sys_.phi(i), o.phi(i), rtol=1e-10, atol=1e-12)
    assert abs(sys_.free_energy() - o.free_energy()) <= 1e-9 * max(1.0, abs(o.free_energy()))


@pytest.mark.parametrize("case", ["3d_2nd_brush", "1d_2nd_lumped", "2d_2nd_lumped", "2d_2nd_lumped_periodic",
                                  "1d_cyl_2nd_lumped", "2d_cyl_2nd_lumped"])
def test_bond_orientation(gpu_lib, case):
    """Bond-orientation profiles of the second-order lattices against the
    oracle, per molecule and axis."""
    spec = CASES[case]()
    sys_ = System(spec)
    o = Oracle(spec)
    x = random_x(spec, seed=21)
    sys_.set_bond_orientation(True)
    sys_.residual(x)
    o.residual(x)
    na = 2 if sys_.K == 3 else 3
    for m in range(len(spec.molecules)):
        for a in range(na):
            want = o.bond_orientation(m, a)
            got = sys_.bond_orientation(m, a)
            assert np.max(np.abs(got - want)) <= TOL_EVAL * max(np.max(np.abs(want)), 1e-300), (m, a)
    from field_b200._native import SfgpuError
    with pytest.raises(SfgpuError):
        sys_.bond_orientation(0, na)


def test_bond_orientation_errors(gpu_lib):
    """First-order lattices have no bond orientation; a second-order system
    reports it only once enabled."""
    from field_b200._native import SfgpuError
    s1 = System(CASES["1d_surface"]())
    with pytest.raises(SfgpuError) as e:
        s1.set_bond_orientation(True)
    assert e.value.code == 7
    s2 = System(CASES["3d_2nd_brush"]())
    with pytest.raises(SfgpuError):
        s2.bond_orientation(0, 0)


@pytest.mark.parametrize("case", sorted(CASES))
def test_thermo(gpu_lib, case):
    """F, the grand potential and both densities against the oracle."""
    spec = CASES[case]()
    sys_ = System(spec)
    o = Oracle(spec)
    x = random_x(spec, seed=13, scale=0.2)
    sys_.residual(x)
    o.residual(x)
    Fg, Og, feg, gpg = sys_.thermo()
    Fc, Oc, fec, gpc = o.thermo()
    assert abs(Fg - Fc) <= 1e-11 * max(1.0, abs(Fc))
    assert abs(Og - Oc) <= 1e-11 * max(1.0, abs(Oc), abs(Fc))
    assert Fg == pytest.approx(sys_.free_energy(), rel=1e-14, abs=1e-14)
    assert rel(feg, fec) <= TOL_EVAL and rel(gpg, gpc) <= TOL_EVAL


@pytest.mark.parametrize("case", ["3d_fcc_colloid", "3d_hex_colloid", "3d_hex_mirror", "3d_stencils_colloid",
                                  "3d_2nd_fcc_brush", "3d_2nd_stiff_copol"])
def test_lattice_types_converged_parity(gpu_lib, case):
    """FCC, HEX and stencils 3D lattices (and a second-order lattice with FCC
    contacts) converged by the device Pure_DIIS and by the oracle's."""
    spec = CASES[case]()
    sys_ = System(spec)
    o = Oracle(spec)
    x0 = np.zeros(spec.n_itvar())
    rg = sys_.solve(x0, tol=1e-10, maxit=3000, m=8, eta=0.3)
    xc, rc, it, err = o.solve_diis(x0, tol=1e-10, maxit=3000, m=8, eta=0.3)
    assert rg.converged and rc == 0, (rg.converged, rc, err)
    assert rg.iterations > 5
    sys_.residual(rg.x)
    o.residual(xc)
    for i in range(len(spec.segments)):
        np.testing.assert_allclose(sys_.phi(i), o.phi(i), rtol=1e-9, atol=1e-12)
    assert abs(sys_.free_energy() - o.free_energy()) <= 1e-9 * max(1.0, abs(o.free_energy()))


@pytest.mark.parametrize("case", ["1d_dendrimer", "2d_dendrimer", "3d_dendrimer", "1d_force", "2d_cyl_force",
                                  "3d_force"])
def test_dendrimer_converged_parity(gpu_lib, case):
    """Symmetric dendrimers (SF_Dend1stO) and force-ensemble copolymers
    converged by the device Pure_DIIS and by the oracle's; for dendrimers the
    batched kernel reports SFGPU_ERR_UNSUPPORTED."""
    from field_b200._native import SfgpuError
    from field_b200.batch import BatchSolver
    spec = CASES[case]()
    sys_ = System(spec)
    o = Oracle(spec)
    x0 = np.zeros(spec.n_itvar())
    rg = sys_.solve(x0, tol=1e-10, maxit=4000, m=8, eta=0.3)
    xc, rc, it, err = o.solve_diis(x0, tol=1e-10, maxit=4000, m=8, eta=0.3)
    assert rg.converged and rc == 0, (rg.converged, rc, err)
    sys_.residual(rg.x)
    o.residual(xc)
    for i in range(len(spec.segments)):
        np.testing.assert_allclose(sys_.phi(i), o.phi(i), rtol=1e-9, atol=1e-12)
    assert abs(sys_.free_energy() - o.free_energy()) <= 1e-9 * max(1.0, abs(o.free_energy()))
    if "dendrimer" in case:
        with pytest.raises(SfgpuError) as e:
            BatchSolver([spec], m=5, eta=0.1)
        assert e.value.code == 7


def test_stiff_range_refusals(gpu_lib):
    """A stiff range takes copolymers only (SF_MolList2ndO.cpp:39-47); bond
    orientation is not built for it."""
    from field_b200._native import SfgpuError
    from field_b200.desc import Molecule, MOL_FREE
    spec = CASES["3d_2nd_stiff_copol"]()
    s = System(spec)
    with pytest.raises(SfgpuError) as e:
        s.set_bond_orientation(True)
    assert e.value.code == 7
    spec.molecules[0] = Molecule("A9", [(1, 9)], MOL_FREE, phibulk=0.03)
    with pytest.raises(SfgpuError) as e:
        System(spec)
    assert e.value.code == 7
