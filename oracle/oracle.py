"""ctypes wrapper of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
the checker; the product (field_b200) never imports it.  The oracle restates
SFbox's equations (see sfbox_oracle.c) and is pinned against SFbox itself:
build_reference() compiles the reference's own sources (oracle/refbuild) and
tests/golden/reference_cases.npz holds that build's outputs.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    src = os.path.join(_HERE, "sfbox_oracle.c")
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])
    return _LIB


REFBUILD = os.path.join(_HERE, "refbuild")
REFERENCE_SRC = "/root/reference"


def build_reference() -> bool:
    """Build SFbox from the reference's own sources into oracle/_ref (sfbox and
    the sfref driver) when the sources are present; False otherwise."""
    if not os.path.isdir(REFERENCE_SRC):
        return False
    subprocess.check_call(["make", "-s", "-j8", "-C", REFBUILD, f"REF={REFERENCE_SRC}"])
    return True


def lib():
    global _lib
    if _lib is None:
        build()
        l = C.CDLL(_LIB)
        vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
        l.orc_create.argtypes = [vp, C.POINTER(vp)]
        l.orc_destroy.argtypes = [vp]
        for n in ("orc_num_sites", "orc_num_itvar", "orc_num_classes"):
            getattr(l, n).argtypes = [vp]
        l.orc_itvar_sites.argtypes = [vp, ip]
        l.orc_class_of_segment.argtypes = [vp, C.c_int]
        l.orc_residual.argtypes = [vp, dp, dp]
        l.orc_get_phi.argtypes = [vp, C.c_int, dp]
        l.orc_get_mol_phi.argtypes = [vp, C.c_int, C.c_int, dp]
        l.orc_get_lngn.argtypes = [vp, C.c_int]
        l.orc_get_lngn.restype = C.c_double
        l.orc_get_phibulk.argtypes = [vp, C.c_int]
        l.orc_get_phibulk.restype = C.c_double
        l.orc_get_swf.argtypes = [vp, C.c_int, dp]
        l.orc_bond_orientation.argtypes = [vp, C.c_int, C.c_int, dp]
        l.orc_thermo.argtypes = [vp, dp, dp, dp, dp]
        l.orc_free_energy.argtypes = [vp]
        l.orc_free_energy.restype = C.c_double
        l.orc_propagate.argtypes = [vp, dp, dp, dp, C.c_double, C.c_int]
        l.orc_side.argtypes = [vp, dp, dp]
        l.orc_lat_lngn.argtypes = [vp, dp, dp]
        l.orc_propagate_stiff.argtypes = [vp, dp, dp, dp, C.c_double, C.c_int, C.c_int]
        l.orc_site_weights.argtypes = [vp, dp]
        l.orc_set_boundaries.argtypes = [vp, dp]
        l.orc_solve_diis.argtypes = [vp, dp, C.c_double, C.c_int, C.c_int, C.c_double, ip, dp]
        _lib = l
    return _lib


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """One SFbox system evaluated on the CPU by the restated equations."""

    def __init__(self, spec):
        self.spec = spec
        self._desc = spec.to_c()
        h = C.c_void_p()
        rc = lib().orc_create(C.byref(self._desc), C.byref(h))
        if rc != 0:
            raise ValueError(f"oracle rejected the system (status {rc})")
        self.h = h
        self.M = lib().orc_num_sites(h)
        self.nvar = lib().orc_num_itvar(h)
        self.nclass = lib().orc_num_classes(h)
        self.K = spec.lattice.components

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def residual(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        f = np.empty(self.nvar)
        lib().orc_residual(self.h, _d(x), _d(f))
        return f

    def phi(self, seg):
        out = np.empty(self.M)
        lib().orc_get_phi(self.h, seg, _d(out))
        return out

    def mol_phi(self, mol, seg):
        out = np.empty(self.M)
        lib().orc_get_mol_phi(self.h, mol, seg, _d(out))
        return out

    def lngn(self, mol):
        return lib().orc_get_lngn(self.h, mol)

    def bond_orientation(self, mol, axis):
        out = np.empty(self.M)
        rc = lib().orc_bond_orientation(self.h, mol, axis, _d(out))
        if rc:
            raise ValueError(f"orc_bond_orientation failed with status {rc}")
        return out

    def thermo(self):
        """(F, Omega, free-energy density, grand-potential density) of the
        last evaluation."""
        F, Om = C.c_double(), C.c_double()
        fe, gp = np.empty(self.M), np.empty(self.M)
        rc = lib().orc_thermo(self.h, C.byref(F), C.byref(Om), _d(fe), _d(gp))
        if rc:
            raise ValueError(f"orc_thermo failed with status {rc}")
        return F.value, Om.value, fe, gp

    def phibulk(self, mol):
        return lib().orc_get_phibulk(self.h, mol)

    def swf(self, seg):
        out = np.empty(self.M)
        lib().orc_get_swf(self.h, seg, _d(out))
        return out

    def free_energy(self):
        return lib().orc_free_energy(self.h)

    def propagate(self, gin, g, S=0.2, backward=False):
        gin = np.ascontiguousarray(gin, dtype=np.float64)
        g = np.ascontiguousarray(g, dtype=np.float64)
        out = np.zeros(self.K * self.M)
        lib().orc_propagate(self.h, _d(gin), _d(g), _d(out), S, int(backward))
        return out

    def propagate_stiff(self, gin, g, S, backward=False, iso=False):
        """One stiff_range (or isotropic) 3D second-order step."""
        gin = np.ascontiguousarray(gin, dtype=np.float64)
        g = np.ascontiguousarray(g, dtype=np.float64)
        out = np.zeros(6 * self.M)
        rc = lib().orc_propagate_stiff(self.h, _d(gin), _d(g), _d(out), S, int(backward), int(iso))
        if rc:
            raise ValueError(f"orc_propagate_stiff failed with status {rc}")
        return out

    def lat_lngn(self, g):
        """ComputeLnGN of one propagator (logarithms with overflow protection)."""
        g = np.ascontiguousarray(g, dtype=np.float64)
        out = C.c_double()
        lib().orc_lat_lngn(self.h, _d(g), C.byref(out))
        return out.value

    def side(self, phi):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        out = np.empty(self.M)
        lib().orc_side(self.h, _d(phi), _d(out))
        return out

    def site_weights(self):
        out = np.empty(self.M)
        lib().orc_site_weights(self.h, _d(out))
        return out

    def set_boundaries(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64).copy()
        lib().orc_set_boundaries(self.h, _d(p))
        return p

    def solve_diis(self, x0, tol=1e-7, maxit=5000, m=5, eta=0.1):
        x = np.ascontiguousarray(x0, dtype=np.float64).copy()
        it = C.c_int()
        err = C.c_double()
        rc = lib().orc_solve_diis(self.h, _d(x), tol, maxit, m, eta, C.byref(it), C.byref(err))
        return x, rc, it.value, err.value
