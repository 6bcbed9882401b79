"""Synthetic SFbox systems of the benchmark shapes (all seeded).

There is no public data set for this path; these generators build the
systems the SCF hot path is measured on, with their sizes, compositions and
initial-guess distributions:

* ``flat_adsorption``  Lat1DFlat1stO, homopolymer A_N in monomeric solvent W
  next to a frozen surface S (config C1 at n=100, N=100).
* ``cyl_micelle``      Lat2DCyl1stO, diblock A_nA B_nB in solvent W with a
  seeded spherical micelle plus Gaussian noise (config C2 at 128x128, A20B20).
* ``melt3d``           Lat3D1stO periodic A_nA B_nB melt (config C3 at 128^3).
* ``sweep1d``          uneven Lat1DFlat1stO instances (config C4).
* ``brush3d``          Lat3D2ndO grafted brush of (X)1(A)_{N-1} (config C5).
"""
from __future__ import annotations

import numpy as np

from .desc import (BOUND_MIRROR1, BOUND_PERIODIC, BOUND_SURFACE, GEOM_CYLINDRICAL, Lattice, Molecule,
                   MOL_FREE, MOL_RESTRICTED, MOL_SOLVENT, Segment, SEG_FREE, SEG_FROZEN, SEG_PINNED,
                   SystemSpec)

BASE_SEED = 20261203

C1_INPUT = """\
lat : flat : gradients : 1
lat : flat : n_layers : {n}
lat : flat : geometry : flat
lat : flat : lambda : 0.16666666666666667
lat : flat : lowerbound : surface
lat : flat : upperbound : mirror1
mon : S : freedom : frozen
mon : S : frozen_range : lowerbound
mon : A : freedom : free
mon : W : freedom : free
mon : A : chi - W : {chi_aw}
mon : A : chi - S : {chi_as}
mol : pol : composition : (A){N}
mol : pol : freedom : free
mol : pol : phibulk : {phib}
mol : water : composition : (W)1
mol : water : freedom : solvent
newton : isaac : method : Pure_DIIS
newton : isaac : tolerance : 1e-7
start
"""


def flat_adsorption(n=100, N=100, phib=0.01, chi_aw=0.5, chi_as=-1.0):
    from .sfinput import build_system, parse_input
    text = C1_INPUT.format(n=n, N=N, phib=phib, chi_aw=chi_aw, chi_as=chi_as)
    spec, _ = build_system(parse_input(text)[0])
    return spec, np.zeros(spec.n_itvar())


def _x_from_potentials(spec: SystemSpec, u_by_seg: dict, noise: np.ndarray = None):
    """Pack per-segment potential fields (full lattice arrays) into SFbox's
    iteration-variable layout: site-major, one value per class."""
    cls, nc = spec.class_layout()
    sites = spec.itvar_sites()
    x = np.zeros((len(sites), nc))
    for seg, u in u_by_seg.items():
        c = cls[seg]
        if c >= 0:
            x[:, c] = np.asarray(u).reshape(-1)[sites]
    if noise is not None:
        x += noise.reshape(x.shape)
    return x.reshape(-1)


def cyl_micelle(nx=128, ny=128, nA=20, nB=20, phib=0.005, chi_aw=1.6, chi_bw=0.0, radius=6.0,
                noise=0.1, seed=BASE_SEED + 2):
    lat = Lattice(gradients=2, n_layers=[nx, ny, 0], bound_lo=[BOUND_MIRROR1] * 2 + [0],
                  bound_hi=[BOUND_MIRROR1] * 2 + [0], geometry=GEOM_CYLINDRICAL, lam=1.0 / 6.0)
    segs = [Segment("A"), Segment("B"), Segment("W")]
    chi = np.zeros((3, 3))
    chi[0, 2] = chi[2, 0] = chi_aw
    chi[1, 2] = chi[2, 1] = chi_bw
    mols = [Molecule("AB", [(0, nA), (1, nB)], MOL_FREE, phibulk=phib), Molecule("W", [(2, 1)], MOL_SOLVENT)]
    spec = SystemSpec(lat, segs, chi, mols)
    MX, MY = lat.shape
    xx, yy = np.meshgrid(np.arange(MX) - 0.5, np.arange(MY) - (MY / 2.0), indexing="ij")
    inside = (xx ** 2 + yy ** 2) < radius ** 2
    uA = np.where(inside, -1.0, 0.0)
    uW = np.where(inside, 1.0, 0.0)
    rng = np.random.default_rng(seed)
    nv = spec.n_itvar()
    x = _x_from_potentials(spec, {0: uA, 1: np.zeros_like(uA), 2: uW}, rng.normal(0.0, noise, nv))
    return spec, x


CYL_INPUT = """\
lat : cyl : gradients : 2
lat : cyl : geometry : cylindrical
lat : cyl : n_layers_x : {nx}
lat : cyl : n_layers_y : {ny}
lat : cyl : lambda : 0.16666666666666667
lat : cyl : lowerbound_x : mirror1
lat : cyl : upperbound_x : mirror1
lat : cyl : lowerbound_y : mirror1
lat : cyl : upperbound_y : mirror1
mon : A : freedom : free
mon : B : freedom : free
mon : W : freedom : free
mon : A : chi - W : {chi_aw!r}
mon : B : chi - W : {chi_bw!r}
mol : AB : composition : (A){nA}(B){nB}
mol : AB : freedom : free
mol : AB : phibulk : {phib!r}
mol : water : composition : (W)1
mol : water : freedom : solvent
newton : isaac : method : Pure_DIIS
newton : isaac : m : {m}
newton : isaac : deltamax : {eta!r}
newton : isaac : tolerance : {tol!r}
newton : isaac : iterationlimit : {maxit}
start
"""


def cyl_micelle_input(nx=128, ny=128, nA=20, nB=20, phib=0.005, chi_aw=1.6, chi_bw=0.0, m=10, eta=0.1,
                      tol=1e-7, maxit=2000):
    """The SFbox input file of cyl_micelle's system (the iteration variables'
    initial guess is cyl_micelle's x, passed separately)."""
    return CYL_INPUT.format(nx=nx, ny=ny, nA=nA, nB=nB, phib=phib, chi_aw=chi_aw, chi_bw=chi_bw, m=m, eta=eta,
                            tol=tol, maxit=maxit)


def melt3d(n=128, nA=50, nB=50, chi_ab=0.2, amp=0.05, seed=BASE_SEED + 3):
    lat = Lattice(gradients=3, n_layers=[n, n, n], bound_lo=[BOUND_PERIODIC] * 3, bound_hi=[BOUND_PERIODIC] * 3)
    segs = [Segment("A"), Segment("B")]
    chi = np.array([[0.0, chi_ab], [chi_ab, 0.0]])
    mols = [Molecule("AB", [(0, nA), (1, nB)], MOL_SOLVENT)]
    spec = SystemSpec(lat, segs, chi, mols)
    rng = np.random.default_rng(seed)
    x = rng.uniform(-amp, amp, spec.n_itvar())
    return spec, x


def sweep1d_inputs(count=256, seed=BASE_SEED + 4, n_range=(50, 400), N_range=(20, 1000), tolerance=1e-7):
    """SFbox input files of the uneven 1D instances: layers U{50..400}, N
    log-uniform, chi_AW on a shuffled grid over [0,1], phibulk log-uniform in
    [1e-4,1e-1], chi_AS U[-2,0] (Pure_DIIS at the given tolerance)."""
    rng = np.random.default_rng(seed)
    chis = rng.permutation(np.linspace(0.0, 1.0, count))
    out = []
    for i in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        N = int(round(np.exp(rng.uniform(np.log(N_range[0]), np.log(N_range[1])))))
        phib = float(np.exp(rng.uniform(np.log(1e-4), np.log(1e-1))))
        chi_as = float(rng.uniform(-2.0, 0.0))
        text = C1_INPUT.format(n=n, N=N, phib=phib, chi_aw=float(chis[i]), chi_as=chi_as)
        out.append(text.replace("newton : isaac : tolerance : 1e-7", f"newton : isaac : tolerance : {tolerance!r}"))
    return out


def sweep1d(count=256, seed=BASE_SEED + 4, n_range=(50, 400), N_range=(20, 1000)):
    """The uneven 1D instances of sweep1d_inputs as (spec, x0 = 0)."""
    from .sfinput import build_system, parse_input
    out = []
    for text in sweep1d_inputs(count, seed, n_range, N_range):
        spec, _ = build_system(parse_input(text)[0])
        out.append((spec, np.zeros(spec.n_itvar())))
    return out


def brush3d(n=96, N=200, sigma=0.05, chi=0.3, S=0.2, seed=BASE_SEED + 5, nz=None):
    """Grafted brush (X)1(A)_{N-1} on the first z layer of a mirror-bounded
    2nd-order 3D lattice; round(sigma*n^2) seeded grafting sites."""
    nz = n if nz is None else nz
    lat = Lattice(gradients=3, n_layers=[n, n, nz], bound_lo=[BOUND_MIRROR1] * 3, bound_hi=[BOUND_MIRROR1] * 3,
                  order=2)
    MX, MY, MZ = lat.shape
    rng = np.random.default_rng(seed)
    ng = int(round(sigma * n * n))
    flat = rng.choice(n * n, size=ng, replace=False)
    mask = np.zeros((MX, MY, MZ))
    for f in flat:
        mask[1 + f // n, 1 + f % n, 1] = 1.0
    segs = [Segment("X", SEG_PINNED, mask.reshape(-1)), Segment("A"), Segment("W")]
    chim = np.zeros((3, 3))
    chim[1, 2] = chim[2, 1] = chi
    pf = np.full((3, 3), 0.2)
    pf[1, 1] = S
    mols = [Molecule("brush", [(0, 1), (1, N - 1)], MOL_RESTRICTED, theta=float(ng * N)),
            Molecule("W", [(2, 1)], MOL_SOLVENT)]
    spec = SystemSpec(lat, segs, chim, mols, pf=pf)
    x = np.zeros(spec.n_itvar())
    return spec, x
