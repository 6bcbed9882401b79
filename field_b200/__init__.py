"""field_b200 -- B200-native (sm_100a, FP64) SF-SCF hot path of SFbox.

The compute path is libsfgpu.so (hand-written CUDA behind the C ABI in
include/sfgpu.h); this package holds the host-side mirror of SFbox's input
format and solver-facing API on top of it.
"""
from .desc import (BOUND_MIRROR1, BOUND_MIRROR2, BOUND_PERIODIC, BOUND_SURFACE, GEOM_CYLINDRICAL,
                   GEOM_FLAT, Lattice, Molecule, MOL_FREE, MOL_RESTRICTED, MOL_SOLVENT, Segment,
                   SEG_FREE, SEG_FROZEN, SEG_PINNED, SystemSpec)
from .sfinput import build_system, parse_input

__all__ = ["Lattice", "Molecule", "Segment", "SystemSpec", "parse_input", "build_system",
           "BOUND_SURFACE", "BOUND_MIRROR1", "BOUND_MIRROR2", "BOUND_PERIODIC", "GEOM_FLAT",
           "GEOM_CYLINDRICAL", "SEG_FREE", "SEG_FROZEN", "SEG_PINNED", "MOL_FREE", "MOL_RESTRICTED",
           "MOL_SOLVENT", "System"]


def __getattr__(name):
    if name == "System":
        from .system import System
        return System
    raise AttributeError(name)
