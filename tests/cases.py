"""Small seeded systems covering every lattice, boundary and molecule type of
the hot path; shared by the parity tests."""
import numpy as np

from field_b200 import configs
from field_b200.desc import (BOUND_MIRROR1, BOUND_MIRROR2, BOUND_PERIODIC, BOUND_SURFACE, GEOM_FLAT, Lattice,
                             Molecule, MOL_FREE, MOL_RESTRICTED, MOL_SOLVENT, Segment, SEG_FROZEN, SystemSpec)


def _flat2d_surface():
    lat = Lattice(2, [14, 11, 0], [BOUND_SURFACE, BOUND_MIRROR2, 0], [BOUND_MIRROR1, BOUND_MIRROR1, 0],
                  geometry=GEOM_FLAT, lam=1 / 6)
    MX, MY = lat.shape
    surf = np.zeros((MX, MY))
    surf[0, :] = 1.0
    segs = [Segment("S", SEG_FROZEN, surf.reshape(-1)), Segment("A"), Segment("B"), Segment("W")]
    chi = np.zeros((4, 4))
    chi[0, 1] = chi[1, 0] = -0.8
    chi[1, 3] = chi[3, 1] = 0.9
    chi[2, 3] = chi[3, 2] = 0.2
    mols = [Molecule("AB", [(1, 5), (2, 4), (1, 2)], MOL_FREE, phibulk=0.02),
            Molecule("h", [(2, 7)], MOL_RESTRICTED, theta=3.0),
            Molecule("W", [(3, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, chi, mols)


def _melt_mirror():
    lat = Lattice(3, [7, 6, 5], [BOUND_MIRROR1, BOUND_MIRROR2, BOUND_PERIODIC],
                  [BOUND_MIRROR2, BOUND_MIRROR1, BOUND_PERIODIC])
    segs = [Segment("A"), Segment("B"), Segment("W")]
    chi = np.array([[0, 0.4, 1.0], [0.4, 0, 0.1], [1.0, 0.1, 0]])
    mols = [Molecule("AB", [(0, 6), (1, 5)], MOL_FREE, phibulk=0.1), Molecule("A8", [(0, 8)], MOL_FREE, phibulk=0.05),
            Molecule("W", [(2, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, chi, mols)


def _flat1d_periodic():
    lat = Lattice(1, [33, 0, 0], [BOUND_PERIODIC, 0, 0], [BOUND_PERIODIC, 0, 0], lam=0.25)
    segs = [Segment("A"), Segment("B"), Segment("W")]
    chi = np.array([[0, 0.5, 1.2], [0.5, 0, -0.2], [1.2, -0.2, 0]])
    mols = [Molecule("ABA", [(0, 4), (1, 9), (0, 4)], MOL_RESTRICTED, theta=6.0),
            Molecule("W", [(2, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, chi, mols)


def _flat1d_mirror2_layeradj():
    spec, _ = configs.flat_adsorption(n=25, N=9, phib=0.03, chi_aw=0.7, chi_as=-1.5)
    spec.lattice.lambda_chi = 0.2
    return spec


CASES = {
    "1d_surface": lambda: configs.flat_adsorption(n=40, N=21)[0],
    "1d_surface_even": lambda: configs.flat_adsorption(n=17, N=30, phib=0.002, chi_aw=0.2, chi_as=-2.0)[0],
    "1d_lambda_chi": _flat1d_mirror2_layeradj,
    "1d_periodic_restricted": _flat1d_periodic,
    "2d_cylinder": lambda: configs.cyl_micelle(nx=20, ny=16, nA=6, nB=5, radius=4)[0],
    "2d_flat_surface": _flat2d_surface,
    "3d_periodic_melt": lambda: configs.melt3d(n=9, nA=7, nB=6)[0],
    "3d_mirror_mix": _melt_mirror,
    "3d_2nd_brush": lambda: configs.brush3d(n=6, N=15, sigma=0.2, S=0.5)[0],
}


def random_x(spec, seed=7, scale=0.3):
    rng = np.random.default_rng(seed)
    return rng.normal(0.0, scale, spec.n_itvar())
