"""Small seeded systems covering every lattice, boundary and molecule type of
the hot path; shared by the parity tests."""
import numpy as np

from field_b200 import configs
from field_b200.desc import (BOUND_MIRROR1, BOUND_MIRROR2, BOUND_PERIODIC, BOUND_SURFACE, GEOM_CYLINDRICAL,
                             GEOM_FLAT, GEOM_SPHERICAL, LATTICE_FCC, LATTICE_HEX, LATTICE_STENCILS, Lattice,
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


def _typed(spec, ltype, lambda_3d=(0.0, 0.0, 0.0, 0.0)):
    """The same system on another 3D lattice type (lat : latticetype)."""
    spec.lattice.lattice_type = ltype
    spec.lattice.lambda_3d = tuple(lambda_3d)
    return spec


def _colloid3d(periodic=False):
    """Frozen block of sites (a particle) in a mirror/periodic (or fully
    periodic) 3D box with an adsorbing diblock and a solvent: converges to a
    non-uniform solution."""
    if periodic:
        lat = Lattice(3, [8, 7, 6], [BOUND_PERIODIC] * 3, [BOUND_PERIODIC] * 3)
    else:
        lat = Lattice(3, [8, 7, 6], [BOUND_MIRROR1, BOUND_MIRROR2, BOUND_PERIODIC],
                      [BOUND_MIRROR2, BOUND_MIRROR1, BOUND_PERIODIC])
    mask = np.zeros(lat.shape)
    mask[1:3, 1:3, 2:5] = 1.0
    segs = [Segment("S", SEG_FROZEN, mask.reshape(-1)), Segment("A"), Segment("B"), Segment("W")]
    chi = np.zeros((4, 4))
    chi[0, 1] = chi[1, 0] = -1.5
    chi[1, 3] = chi[3, 1] = 0.7
    chi[2, 3] = chi[3, 2] = 0.2
    mols = [Molecule("AB", [(1, 5), (2, 4)], MOL_FREE, phibulk=0.02), Molecule("W", [(3, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, chi, mols)


def _dendrimer(gradients):
    """A two-generation dendrimer @dend(2, (A)3, 3, (B)2(A)1, 2) (N = 22)
    adsorbing on a surface (1D, 2D) or free in a periodic/mirror box (3D),
    with a free linear chain and a solvent."""
    if gradients == 1:
        lat = Lattice(1, [24, 0, 0], [BOUND_SURFACE, 0, 0], [BOUND_MIRROR1, 0, 0], lam=1 / 6)
    elif gradients == 2:
        lat = Lattice(2, [12, 9, 0], [BOUND_SURFACE, BOUND_MIRROR1, 0], [BOUND_MIRROR2, BOUND_MIRROR1, 0], lam=0.2)
    else:
        lat = Lattice(3, [6, 5, 7], [BOUND_MIRROR1, BOUND_PERIODIC, BOUND_MIRROR2],
                      [BOUND_MIRROR2, BOUND_PERIODIC, BOUND_MIRROR1])
    mask = np.zeros(lat.shape)
    if gradients < 3:
        mask[0] = 1.0
    else:
        mask[2:4, 2:4, 3:5] = 1.0
    segs = [Segment("S", SEG_FROZEN, mask.reshape(-1)), Segment("A"), Segment("B"), Segment("W")]
    chi = np.zeros((4, 4))
    chi[0, 1] = chi[1, 0] = -1.2
    chi[1, 3] = chi[3, 1] = 0.5
    chi[2, 3] = chi[3, 2] = -0.3
    d = Molecule("dend", [(1, 3), (2, 2), (1, 1)], MOL_RESTRICTED if gradients != 3 else MOL_FREE,
                 theta=1.5, phibulk=0.01, generations=[(1, 3), (2, 2)])
    return SystemSpec(lat, segs, chi, [d, Molecule("B6", [(2, 6)], MOL_FREE, phibulk=0.02),
                                       Molecule("W", [(3, 1)], MOL_SOLVENT)])


def _stiff_copolymer():
    """A 3D second-order lattice with 'lat : stiff_range' over the lower half
    in z (SF_Copol2ndO_stiff_range), a triblock with its own persistence
    factors, a frozen particle and a solvent."""
    lat = Lattice(3, [6, 5, 7], [BOUND_MIRROR1, BOUND_PERIODIC, BOUND_MIRROR2],
                  [BOUND_MIRROR2, BOUND_PERIODIC, BOUND_MIRROR1], order=2)
    mask = np.zeros(lat.shape)
    mask[:, :, :4] = 1.0
    lat.stiff_range = mask.reshape(-1)
    part = np.zeros(lat.shape)
    part[3:5, 2:4, 5:7] = 1.0
    segs = [Segment("S", SEG_FROZEN, part.reshape(-1)), Segment("A"), Segment("B"), Segment("W")]
    chi = np.zeros((4, 4))
    chi[0, 1] = chi[1, 0] = -1.0
    chi[1, 3] = chi[3, 1] = 0.6
    pf = np.full((4, 4), 0.2)
    pf[1, 2] = pf[2, 1] = 0.5
    pf[1, 1] = 0.4
    mols = [Molecule("ABA", [(1, 4), (2, 3), (1, 3)], MOL_FREE, phibulk=0.03), Molecule("W", [(3, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, chi, mols, pf=pf)


def _force_copolymer(gradients):
    """A diblock pulled with mol : force (+0.8 forward, -0.8 backward) next to
    a surface (1D), in a cylinder with a core (2D) or around a particle (3D)."""
    if gradients == 1:
        lat = Lattice(1, [20, 0, 0], [BOUND_SURFACE, 0, 0], [BOUND_MIRROR1, 0, 0], lam=1 / 6)
    elif gradients == 2:
        lat = Lattice(2, [10, 9, 0], [BOUND_MIRROR1, BOUND_MIRROR2, 0], [BOUND_MIRROR1, BOUND_MIRROR1, 0],
                      geometry=GEOM_CYLINDRICAL, lam=0.2)
    else:
        lat = Lattice(3, [5, 6, 7], [BOUND_MIRROR1, BOUND_PERIODIC, BOUND_MIRROR2],
                      [BOUND_MIRROR2, BOUND_PERIODIC, BOUND_MIRROR1])
    mask = np.zeros(lat.shape)
    if gradients == 1:
        mask[0] = 1.0
    elif gradients == 2:
        mask[1:3, 1:4] = 1.0
    else:
        mask[2:4, 2:4, 3:5] = 1.0
    segs = [Segment("S", SEG_FROZEN, mask.reshape(-1)), Segment("A"), Segment("B"), Segment("W")]
    chi = np.zeros((4, 4))
    chi[0, 1] = chi[1, 0] = -1.3
    chi[2, 3] = chi[3, 2] = 0.5
    mols = [Molecule("AB", [(1, 5), (2, 7)], MOL_FREE, phibulk=0.02, force=0.8),
            Molecule("W", [(3, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, chi, mols)


# stencils contact weights: centre, face, edge, corner (0.1 + 6*0.08 + 12*0.02 + 8*0.0225 = 1)
STENCILS = (0.1, 0.08, 0.02, 0.0225)


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


def _cyl1d_micelle():
    """Lat1DCyl1stO around the axis (no offset), mirror1 both sides with a
    layer adjustment of the first and last layer, lambda_chi != lambda, an
    AB diblock, a restricted homopolymer and solvent."""
    lat = Lattice(1, [22, 0, 0], [BOUND_MIRROR1, 0, 0], [BOUND_MIRROR1, 0, 0], geometry=GEOM_CYLINDRICAL,
                  lam=1 / 6, lambda_chi=0.2, layer_adjustment=0.8)
    segs = [Segment("A"), Segment("B"), Segment("W")]
    chi = np.array([[0, 0.3, 1.4], [0.3, 0, -0.1], [1.4, -0.1, 0]])
    mols = [Molecule("AB", [(0, 7), (1, 6)], MOL_FREE, phibulk=0.02),
            Molecule("h", [(0, 9)], MOL_RESTRICTED, theta=5.0),
            Molecule("W", [(2, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, chi, mols)


def _sphere1d_colloid():
    """Lat1DSphere1stO: a colloid of radius 3 (offset_first_layer) whose
    surface layer adsorbs a homopolymer, mirror2 at the outer edge."""
    lat = Lattice(1, [18, 0, 0], [BOUND_SURFACE, 0, 0], [BOUND_MIRROR2, 0, 0], geometry=GEOM_SPHERICAL,
                  lam=1 / 6, offset_first_layer=3.0)
    surf = np.zeros(lat.M)
    surf[0] = 1.0
    segs = [Segment("S", SEG_FROZEN, surf), Segment("A"), Segment("W")]
    chi = np.zeros((3, 3))
    chi[0, 1] = chi[1, 0] = -1.4
    chi[1, 2] = chi[2, 1] = 0.6
    mols = [Molecule("A", [(1, 16)], MOL_FREE, phibulk=0.01), Molecule("W", [(2, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, chi, mols)


def _flat1d_2nd():
    """Lat1D2ndO: surface with an adsorbing frozen layer below, mirror2 above
    (the upper side swaps the +x/-x components there, the lower side does not
    for mirror2), stiff A chains (S = 0.5) in solvent."""
    lat = Lattice(1, [24, 0, 0], [BOUND_SURFACE, 0, 0], [BOUND_MIRROR2, 0, 0], order=2, lam=1 / 6)
    M = lat.M
    surf = np.zeros(M)
    surf[0] = 1.0
    segs = [Segment("S", SEG_FROZEN, surf), Segment("A"), Segment("W")]
    chi = np.zeros((3, 3))
    chi[0, 1] = chi[1, 0] = -1.2
    chi[1, 2] = chi[2, 1] = 0.6
    pf = np.full((3, 3), 0.2)
    pf[1, 1] = 0.5
    mols = [Molecule("A", [(1, 15)], MOL_FREE, phibulk=0.02), Molecule("W", [(2, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, chi, mols, pf=pf)


def _flat2d_2nd():
    """Lat2D2ndO: mirror2 below in x (no swap) and mirror1 above, surface and
    mirror2 in y; an AB copolymer with stiffness across the junction, a
    restricted homopolymer and solvent."""
    lat = Lattice(2, [11, 9, 0], [BOUND_MIRROR2, BOUND_SURFACE, 0], [BOUND_MIRROR1, BOUND_MIRROR2, 0], order=2,
                  lam=1 / 6)
    segs = [Segment("A"), Segment("B"), Segment("W")]
    chi = np.array([[0, 0.4, 1.0], [0.4, 0, 0.1], [1.0, 0.1, 0]])
    pf = np.full((3, 3), 0.2)
    pf[0, 0], pf[0, 1], pf[1, 0] = 0.45, 0.3, 0.3
    mols = [Molecule("AB", [(0, 6), (1, 5)], MOL_FREE, phibulk=0.05),
            Molecule("h", [(1, 7)], MOL_RESTRICTED, theta=4.0),
            Molecule("W", [(2, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, chi, mols, pf=pf)


def _flat2d_2nd_periodic():
    """Lat2D2ndO with periodic x (no swaps) and surface/mirror1 y."""
    lat = Lattice(2, [8, 7, 0], [BOUND_PERIODIC, BOUND_SURFACE, 0], [BOUND_PERIODIC, BOUND_MIRROR1, 0], order=2,
                  lam=1 / 6)
    segs = [Segment("A"), Segment("W")]
    chi = np.array([[0, 0.8], [0.8, 0]])
    pf = np.full((2, 2), 0.3)
    mols = [Molecule("A", [(0, 9)], MOL_FREE, phibulk=0.04), Molecule("W", [(1, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, chi, mols, pf=pf)


def _cyl1d_2nd():
    """Lat1DCyl2ndO around the axis, mirror1 both sides: a stiff AB diblock
    (S = 0.5 inside A, 0.3 across the junction) and solvent."""
    lat = Lattice(1, [20, 0, 0], [BOUND_MIRROR1, 0, 0], [BOUND_MIRROR1, 0, 0], geometry=GEOM_CYLINDRICAL,
                  order=2, lam=1 / 6)
    segs = [Segment("A"), Segment("B"), Segment("W")]
    chi = np.array([[0, 0.3, 1.3], [0.3, 0, -0.1], [1.3, -0.1, 0]])
    pf = np.full((3, 3), 0.2)
    pf[0, 0], pf[0, 1], pf[1, 0] = 0.5, 0.3, 0.3
    mols = [Molecule("AB", [(0, 8), (1, 6)], MOL_FREE, phibulk=0.03), Molecule("W", [(2, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, chi, mols, pf=pf)


def _sphere1d_2nd():
    """Lat1DSphere2ndO: a colloid of radius 4 with an adsorbing surface
    layer, mirror2 outside; stiff free chains and a restricted one."""
    lat = Lattice(1, [16, 0, 0], [BOUND_SURFACE, 0, 0], [BOUND_MIRROR2, 0, 0], geometry=GEOM_SPHERICAL,
                  order=2, lam=1 / 6, offset_first_layer=4.0)
    surf = np.zeros(lat.M)
    surf[0] = 1.0
    segs = [Segment("S", SEG_FROZEN, surf), Segment("A"), Segment("W")]
    chi = np.zeros((3, 3))
    chi[0, 1] = chi[1, 0] = -1.2
    chi[1, 2] = chi[2, 1] = 0.5
    pf = np.full((3, 3), 0.2)
    pf[1, 1] = 0.45
    mols = [Molecule("A", [(1, 12)], MOL_FREE, phibulk=0.01), Molecule("r", [(1, 7)], MOL_RESTRICTED, theta=20.0),
            Molecule("W", [(2, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, chi, mols, pf=pf)


def _cyl2d_2nd():
    """Lat2DCyl2ndO: radius x with a core of radius 2 behind a surface,
    mirror1 outside; y from a surface to mirror2; an AB diblock and solvent."""
    lat = Lattice(2, [10, 8, 0], [BOUND_SURFACE, BOUND_SURFACE, 0], [BOUND_MIRROR1, BOUND_MIRROR2, 0],
                  geometry=GEOM_CYLINDRICAL, order=2, lam=1 / 6, offset_first_layer=2.0)
    segs = [Segment("A"), Segment("B"), Segment("W")]
    chi = np.array([[0, 0.5, 1.1], [0.5, 0, 0.2], [1.1, 0.2, 0]])
    pf = np.full((3, 3), 0.2)
    pf[0, 0] = 0.4
    mols = [Molecule("AB", [(0, 5), (1, 6)], MOL_FREE, phibulk=0.04), Molecule("W", [(2, 1)], MOL_SOLVENT)]
    return SystemSpec(lat, segs, chi, mols, pf=pf)


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
    "3d_fcc_colloid": lambda: _typed(_colloid3d(), LATTICE_FCC),
    # HEX neighbours are not mirror symmetric: on mirror boundaries its step
    # is not detailed-balanced, so the periodic box is the physical case
    "3d_hex_colloid": lambda: _typed(_colloid3d(periodic=True), LATTICE_HEX),
    "3d_hex_mirror": lambda: _typed(_colloid3d(), LATTICE_HEX),
    "3d_stencils_colloid": lambda: _typed(_colloid3d(), LATTICE_STENCILS, STENCILS),
    "3d_stencils_melt": lambda: _typed(configs.melt3d(n=7, nA=5, nB=6)[0], LATTICE_STENCILS, STENCILS),
    "1d_dendrimer": lambda: _dendrimer(1),
    "2d_dendrimer": lambda: _dendrimer(2),
    "3d_dendrimer": lambda: _dendrimer(3),
    "3d_2nd_stiff_copol": _stiff_copolymer,
    "1d_force": lambda: _force_copolymer(1),
    "2d_cyl_force": lambda: _force_copolymer(2),
    "3d_force": lambda: _force_copolymer(3),
    "3d_2nd_fcc_brush": lambda: _typed(configs.brush3d(n=6, N=15, sigma=0.2, S=0.5)[0], LATTICE_FCC),
    "1d_cylinder": _cyl1d_micelle,
    "1d_sphere_colloid": _sphere1d_colloid,
    "1d_2nd_lumped": _flat1d_2nd,
    "2d_2nd_lumped": _flat2d_2nd,
    "2d_2nd_lumped_periodic": _flat2d_2nd_periodic,
    "1d_cyl_2nd_lumped": _cyl1d_2nd,
    "1d_sphere_2nd_lumped": _sphere1d_2nd,
    "2d_cyl_2nd_lumped": _cyl2d_2nd,
}

def _from_input(name):
    """A system of the SFbox fixture inputs (tests/golden/reference_inputs.py)."""
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from reference_inputs import INPUTS
    from field_b200.sfinput import build_system, parse_input
    return build_system(parse_input(INPUTS[name])[0])[0]


CASES.update({
    "1d_branched": lambda: _from_input("1d_branched"),
    "2d_branched": lambda: _from_input("2d_branched"),
    "3d_branched": lambda: _from_input("3d_branched"),
    "1d_comb_branched": lambda: _from_input("1d_comb_branched_side"),
    "1d_ring": lambda: _from_input("1d_ring"),
})

# cases with forward-mode derivatives (all); the reverse mode leaves out the
# second-order lumped lattices and stiff ranges (the adjoint tests list "2nd"
# cases by name)
DIFFERENTIABLE = sorted(CASES)


def random_x(spec, seed=7, scale=0.3):
    rng = np.random.default_rng(seed)
    return rng.normal(0.0, scale, spec.n_itvar())

REVERSE_EXCLUDED = ("2nd",)
