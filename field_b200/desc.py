"""System descriptions shared by the CUDA library and its checkers.

``SystemSpec`` is the host-side picture of one SFbox calculation restricted to
the SCF hot path: a lattice (``lat``), segment types (``mon``), a chi matrix,
persistence factors (2nd order) and molecules (``mol``).  ``to_c()`` packs it
into the ``sfgpu_system_desc`` C struct declared in ``include/sfgpu.h``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

BOUND_SURFACE, BOUND_MIRROR1, BOUND_MIRROR2, BOUND_PERIODIC = 1, 2, 3, 4
GEOM_FLAT, GEOM_CYLINDRICAL, GEOM_SPHERICAL = 0, 1, 2
LATTICE_STANDARD, LATTICE_STENCILS, LATTICE_FCC, LATTICE_HEX = 0, 1, 2, 3
SEG_FREE, SEG_FROZEN, SEG_PINNED = 0, 1, 2
MOL_FREE, MOL_RESTRICTED, MOL_SOLVENT, MOL_NEUTRALIZER = 0, 1, 2, 3

BOUND_NAMES = {"surface": BOUND_SURFACE, "mirror1": BOUND_MIRROR1,
               "mirror2": BOUND_MIRROR2, "periodic": BOUND_PERIODIC}


class LatticeDesc(C.Structure):
    _fields_ = [("gradients", C.c_int), ("geometry", C.c_int), ("order", C.c_int),
                ("n_layers", C.c_int * 3), ("bound_lo", C.c_int * 3), ("bound_hi", C.c_int * 3),
                ("lam", C.c_double), ("lambda_chi", C.c_double),
                ("layer_adjustment", C.c_double), ("dimensions", C.c_double),
                ("offset_first_layer", C.c_double), ("stiff_range", C.POINTER(C.c_double)),
                ("lattice_type", C.c_int),
                ("lambda_3d", C.c_double * 4), ("bondlength", C.c_double)]


class SegmentDesc(C.Structure):
    _fields_ = [("freedom", C.c_int), ("range", C.POINTER(C.c_double)), ("valence", C.c_double),
                ("epsilon", C.c_double)]


class MoleculeDesc(C.Structure):
    _fields_ = [("n_blocks", C.c_int), ("block_segment", C.POINTER(C.c_int)),
                ("block_length", C.POINTER(C.c_int)), ("freedom", C.c_int),
                ("phibulk", C.c_double), ("theta", C.c_double), ("n_generations", C.c_int),
                ("generation_blocks", C.POINTER(C.c_int)), ("generation_repeat", C.POINTER(C.c_int)),
                ("force", C.c_double), ("bond_parent", C.POINTER(C.c_int)), ("ring", C.c_int)]


class SystemDesc(C.Structure):
    _fields_ = [("lattice", LatticeDesc), ("n_segments", C.c_int),
                ("segments", C.POINTER(SegmentDesc)), ("chi", C.POINTER(C.c_double)),
                ("pf", C.POINTER(C.c_double)), ("n_molecules", C.c_int),
                ("molecules", C.POINTER(MoleculeDesc)), ("overflow_protection", C.c_int),
                ("temperature", C.c_double)]


class NewtonSettings(C.Structure):
    """sfgpu_newton_settings: SFbox's Newton iteration parameters."""
    _fields_ = [("tolerance", C.c_double), ("iterationlimit", C.c_int), ("pseudohessian", C.c_int),
                ("deltamax", C.c_double), ("deltamin", C.c_double), ("linesearchlimit", C.c_int),
                ("small_alpha", C.c_double), ("max_n_small_alpha", C.c_int),
                ("reset_hessian_criterion", C.c_double), ("max_accuracy_for_hessian_scaling", C.c_double),
                ("ignore_newton_direction", C.c_int)]


def dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def iptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


@dataclass
class Lattice:
    gradients: int
    n_layers: Sequence[int]
    bound_lo: Sequence[int]
    bound_hi: Sequence[int]
    geometry: int = GEOM_FLAT
    order: int = 1
    lam: float = 1.0 / 6.0
    lambda_chi: float = -1.0
    layer_adjustment: float = 1.0
    dimensions: float = 3.0
    offset_first_layer: float = 0.0
    lattice_type: int = LATTICE_STANDARD
    lambda_3d: Sequence[float] = (0.0, 0.0, 0.0, 0.0)
    stiff_range: Optional[np.ndarray] = None     # M values, 1 inside 'lat : stiff_range'
    bondlength: float = 3e-10                    # lat : bondlength (m), charged systems

    @property
    def shape(self):
        return tuple(int(n) + 2 for n in self.n_layers[: self.gradients])

    @property
    def M(self) -> int:
        return int(np.prod(self.shape))

    def interior_mask(self) -> np.ndarray:
        """M booleans, True on sites with no coordinate in a boundary layer."""
        mask = np.ones(self.shape, dtype=bool)
        for k, n in enumerate(self.shape):
            idx = [slice(None)] * len(self.shape)
            idx[k] = 0
            mask[tuple(idx)] = False
            idx[k] = n - 1
            mask[tuple(idx)] = False
        return mask.reshape(-1)

    @property
    def components(self) -> int:
        """Direction components of a propagator: 1 (first order); second order
        6 in 3D, and 3 (1D) / 5 (2D), which lump the bond directions along the
        homogeneous gradients (Lat1D2ndO, Lat2D2ndO)."""
        if self.order != 2:
            return 1
        return {1: 3, 2: 5, 3: 6}[self.gradients]

    def to_c(self) -> LatticeDesc:
        d = LatticeDesc()
        d.gradients, d.geometry, d.order = self.gradients, self.geometry, self.order
        for k in range(3):
            d.n_layers[k] = int(self.n_layers[k]) if k < self.gradients else 0
            d.bound_lo[k] = int(self.bound_lo[k]) if k < self.gradients else 0
            d.bound_hi[k] = int(self.bound_hi[k]) if k < self.gradients else 0
        d.lam, d.lambda_chi = self.lam, self.lambda_chi
        d.layer_adjustment, d.dimensions = self.layer_adjustment, self.dimensions
        d.offset_first_layer = self.offset_first_layer
        d.lattice_type = int(self.lattice_type)
        for k in range(4):
            d.lambda_3d[k] = float(self.lambda_3d[k])
        d.bondlength = float(self.bondlength)
        if self.stiff_range is not None:
            self._stiff = np.ascontiguousarray(self.stiff_range, dtype=np.float64).reshape(-1)
            if self._stiff.size != self.M:
                raise ValueError(f"stiff_range has {self._stiff.size} values, lattice has {self.M}")
            d.stiff_range = dptr(self._stiff)
        else:
            d.stiff_range = C.POINTER(C.c_double)()
        return d


@dataclass
class Segment:
    name: str
    freedom: int = SEG_FREE
    range: Optional[np.ndarray] = None      # M range values (frozen/pinned)
    valence: float = 0.0                    # mon : valence (elementary charges)
    epsilon: float = 80.0                   # mon : epsilon (relative dielectric constant)


@dataclass
class Molecule:
    name: str
    blocks: List[tuple]                     # [(segment index, length), ...]
    freedom: int = MOL_FREE
    phibulk: float = 0.0
    theta: float = 0.0
    # symmetric dendrimer: per generation (number of its blocks in `blocks`,
    # functionality f); None for a linear chain
    generations: Optional[List[tuple]] = None
    force: float = 0.0                      # mol : force (constant-force ensemble)
    # branched molecule: the segment each segment is bonded to on its way to
    # segment 0 (-1 for segment 0), in the order of `blocks`; None if linear
    bond_parent: Optional[List[int]] = None
    ring: bool = False                      # mol : ring (homopolymer ring)

    def generation_blocks(self) -> List[List[tuple]]:
        out, b = [], 0
        for nb, _f in self.generations or []:
            out.append(self.blocks[b:b + nb])
            b += nb
        return out

    @property
    def N(self) -> int:
        """Chain length; a dendrimer's generation blocks share their first
        segment among f copies (SF_MolStructure::SetMolLength,
        SF_MolStructure.cpp:847-877)."""
        if not self.generations:
            return int(sum(n for _, n in self.blocks))
        L = 0
        for blocks, (_nb, f) in reversed(list(zip(self.generation_blocks(), self.generations))):
            L = (L + sum(n for _, n in blocks) - 1) * f + 1
        return int(L)

    def count(self, seg: int) -> int:
        """Segments of type seg in one molecule (GetAvNumSegments,
        SF_MolStructure.cpp:552-595)."""
        if not self.generations:
            return int(sum(n for s, n in self.blocks if s == seg))
        num = 0
        for blocks, (_nb, f) in reversed(list(zip(self.generation_blocks(), self.generations))):
            n = sum(k for s, k in blocks if s == seg)
            num = (num + n - 1) * f + 1 if blocks[0][0] == seg else (num + n) * f
        return int(num)

    def segment_types(self) -> List[int]:
        return sorted({s for s, _ in self.blocks})


@dataclass
class SystemSpec:
    lattice: Lattice
    segments: List[Segment]
    chi: np.ndarray
    molecules: List[Molecule]
    pf: Optional[np.ndarray] = None
    overflow_protection: bool = False
    temperature: float = 298.15             # sys : temperature (K), electrostatic terms
    _keep: list = field(default_factory=list, repr=False)

    @property
    def M(self) -> int:
        return self.lattice.M

    def segment_index(self, name: str) -> int:
        for i, s in enumerate(self.segments):
            if s.name == name:
                return i
        raise KeyError(name)

    def to_c(self) -> SystemDesc:
        keep = []
        ns = len(self.segments)
        segs = (SegmentDesc * ns)()
        for i, s in enumerate(self.segments):
            segs[i].freedom = s.freedom
            segs[i].valence, segs[i].epsilon = float(s.valence), float(s.epsilon)
            if s.range is not None:
                r = np.ascontiguousarray(s.range, dtype=np.float64)
                if r.size != self.M:
                    raise ValueError(f"range of segment {s.name} has {r.size} values, lattice has {self.M}")
                keep.append(r)
                segs[i].range = dptr(r)
            else:
                segs[i].range = C.POINTER(C.c_double)()
        chi = np.ascontiguousarray(self.chi, dtype=np.float64).reshape(ns, ns)
        keep.append(chi)
        mols = (MoleculeDesc * len(self.molecules))()
        for m, mol in enumerate(self.molecules):
            bs = np.array([b[0] for b in mol.blocks], dtype=np.int32)
            bl = np.array([b[1] for b in mol.blocks], dtype=np.int32)
            keep += [bs, bl]
            mols[m].n_blocks = len(mol.blocks)
            mols[m].block_segment, mols[m].block_length = iptr(bs), iptr(bl)
            mols[m].freedom, mols[m].phibulk, mols[m].theta = mol.freedom, mol.phibulk, mol.theta
            mols[m].force = float(mol.force)
            mols[m].ring = int(bool(mol.ring))
            if mol.bond_parent is not None:
                bp = np.ascontiguousarray(mol.bond_parent, dtype=np.int32)
                if bp.size != mol.N:
                    raise ValueError(f"bond_parent of molecule {mol.name} has {bp.size} entries, chain has {mol.N}")
                keep.append(bp)
                mols[m].bond_parent = iptr(bp)
            else:
                mols[m].bond_parent = C.POINTER(C.c_int)()
            if mol.generations:
                gb = np.array([g[0] for g in mol.generations], dtype=np.int32)
                gr = np.array([g[1] for g in mol.generations], dtype=np.int32)
                keep += [gb, gr]
                mols[m].n_generations = len(mol.generations)
                mols[m].generation_blocks, mols[m].generation_repeat = iptr(gb), iptr(gr)
            else:
                mols[m].n_generations = 0
                mols[m].generation_blocks = C.POINTER(C.c_int)()
                mols[m].generation_repeat = C.POINTER(C.c_int)()
        d = SystemDesc()
        d.lattice = self.lattice.to_c()
        d.n_segments = ns
        d.segments = C.cast(segs, C.POINTER(SegmentDesc))
        d.chi = dptr(chi)
        if self.pf is not None:
            pf = np.ascontiguousarray(self.pf, dtype=np.float64).reshape(ns, ns)
            keep.append(pf)
            d.pf = dptr(pf)
        else:
            d.pf = C.POINTER(C.c_double)()
        d.n_molecules = len(self.molecules)
        d.molecules = C.cast(mols, C.POINTER(MoleculeDesc))
        d.overflow_protection = int(bool(self.overflow_protection))
        d.temperature = float(self.temperature)
        keep += [segs, mols]
        self._keep = keep
        return d

    # ---- helpers on the iteration-variable packing -----------------------
    def class_layout(self):
        """Classes of liquid segments with equal chi rows, in SFbox's order
        (SF_Solve.cpp:53-86).  Returns (class_of_segment, n_classes)."""
        ns = len(self.segments)
        chi = np.asarray(self.chi, dtype=np.float64).reshape(ns, ns)
        q = [i for i, s in enumerate(self.segments) if s.freedom != SEG_FROZEN]
        n = len(q)
        i = 0
        while i < n:
            s1 = q[i]
            j = i + 1
            while j < n:
                if np.array_equal(chi[:, s1], chi[:, q[j]]):
                    if j != i + 1:
                        q[i + 1], q[j] = q[j], q[i + 1]
                    i += 1
                j += 1
            i += 1
        cls = [-1] * ns
        nc = 0
        i = 0
        while i < n:
            s1 = q[i]
            cls[s1] = nc
            j = i + 1
            while j < n:
                if np.array_equal(chi[:, s1], chi[:, q[j]]):
                    i += 1
                    cls[q[i]] = nc
                j += 1
            nc += 1
            i += 1
        return cls, nc

    def itvar_sites(self) -> np.ndarray:
        """Sites carrying iteration variables (SF_Solve.cpp:129-150)."""
        shape = self.lattice.shape
        interior = np.ones(shape, dtype=bool)
        for d in range(len(shape)):
            sl = [slice(None)] * len(shape)
            sl[d] = 0
            interior[tuple(sl)] = False
            sl[d] = shape[d] - 1
            interior[tuple(sl)] = False
        ok = interior.reshape(-1).copy()
        for s in self.segments:
            if s.freedom == SEG_FROZEN and s.range is not None:
                ok &= ~(np.asarray(s.range).reshape(-1) > 0.999)
        return np.nonzero(ok)[0].astype(np.int64)

    @property
    def charged(self) -> bool:
        return any(s.valence != 0 for s in self.segments)

    def potential_sites(self) -> np.ndarray:
        """Sites whose electrostatic potential is an iteration variable in a
        charged system (SF_Solve::PotItVar, SF_Solve.cpp:1761-1776): every
        interior site and every site of a frozen segment's range."""
        if not self.charged:
            return np.zeros(0, dtype=np.int64)
        ok = self.lattice.interior_mask().copy()
        for s in self.segments:
            if s.freedom == SEG_FROZEN and s.range is not None:
                ok |= np.asarray(s.range).reshape(-1) > 0
        return np.nonzero(ok)[0].astype(np.int64)

    def n_itvar(self) -> int:
        return len(self.itvar_sites()) * self.class_layout()[1] + len(self.potential_sites())
