"""ctypes binding of libsfgpu.so (the C ABI declared in include/sfgpu.h).

There is no CPU fallback: importing the product path without the built
library, or calling it without a CUDA device, raises immediately.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsfgpu.so")

vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
i32, f64 = C.c_int, C.c_double

# name -> (restype, argtypes); every entry point declared in include/sfgpu.h
PROTOTYPES = {
    "sfgpu_last_error": (C.c_char_p, []),
    "sfgpu_device_count": (i32, [ip]),
    "sfgpu_system_create": (i32, [vp, C.POINTER(vp)]),
    "sfgpu_system_create_checkpointed": (i32, [vp, i32, C.POINTER(vp)]),
    "sfgpu_system_destroy": (i32, [vp]),
    "sfgpu_system_info": (i32, [vp, ip, ip, ip, ip]),
    "sfgpu_system_stream": (i32, [vp, C.POINTER(vp)]),
    "sfgpu_system_set_stream": (i32, [vp, vp]),
    "sfgpu_synchronize": (i32, [vp]),
    "sfgpu_residual": (i32, [vp, vp, vp]),
    "sfgpu_residual_host": (i32, [vp, dp, dp]),
    "sfgpu_get_phi": (i32, [vp, i32, dp]),
    "sfgpu_get_mol_phi": (i32, [vp, i32, i32, dp]),
    "sfgpu_get_mol_scalars": (i32, [vp, i32, dp, dp, dp]),
    "sfgpu_system_set_bond_orientation": (i32, [vp, i32]),
    "sfgpu_thermo": (i32, [vp, dp, dp, dp, dp]),
    "sfgpu_lattice_weights": (i32, [vp, dp, dp]),
    "sfgpu_get_bond_orientation": (i32, [vp, i32, i32, dp]),
    "sfgpu_get_swf": (i32, [vp, i32, dp]),
    "sfgpu_free_energy": (i32, [vp, dp]),
    "sfgpu_lat_propagate": (i32, [vp, vp, vp, vp, f64, i32]),
    "sfgpu_lat_set_boundaries": (i32, [vp, vp, i32]),
    "sfgpu_lat_side_fraction": (i32, [vp, vp, vp]),
    "sfgpu_lat_lngn": (i32, [vp, vp, i32, dp]),
    "sfgpu_lat_connect": (i32, [vp, vp, vp, vp, i32]),
    "sfgpu_lat_correct_double_count": (i32, [vp, vp, vp]),
    "sfgpu_lat_norm_phi_free": (i32, [vp, vp, f64]),
    "sfgpu_lat_norm_phi_restr": (i32, [vp, vp, vp, i32, f64]),
    "sfgpu_solve_diis": (i32, [vp, dp, f64, i32, i32, f64, ip, dp]),
    "sfgpu_solve_diis_many": (i32, [i32, C.POINTER(vp), C.POINTER(dp), f64, i32, i32, f64, i32, ip, ip, dp]),
    "sfgpu_newton_default_settings": (i32, [vp]),
    "sfgpu_solve_newton": (i32, [vp, dp, vp, ip, ip, dp]),
    "sfgpu_profile_propagator": (i32, [vp, i32, dp, dp, dp, dp]),
    "sfgpu_system_set_tile": (i32, [vp, i32]),
    "sfgpu_system_set_tile_pipelined": (i32, [vp, i32]),
    "sfgpu_jvp": (i32, [vp, vp, vp, vp, vp]),
    "sfgpu_jvp_host": (i32, [vp, dp, dp, dp, dp]),
    "sfgpu_solve_nk": (i32, [vp, dp, f64, i32, i32, ip, ip, dp]),
    "sfgpu_vjp": (i32, [vp, vp, vp, vp, vp]),
    "sfgpu_vjp_host": (i32, [vp, dp, dp, dp, dp]),
    "sfgpu_system_set_checkpoint": (i32, [vp, i32]),
    "sfgpu_system_autotune_checkpoint": (i32, [vp, dp, i32, C.c_double, ip, dp]),
    "sfgpu_vjp_chi": (i32, [vp, dp, dp, dp]),
    "sfgpu_free_energy_grad": (i32, [vp, dp, dp, dp]),
    "sfgpu_phi_sensitivity_chi": (i32, [vp, dp, dp, dp, f64, i32, i32, dp]),
    "sfgpu_solve_lbfgs": (i32, [vp, dp, f64, i32, i32, ip, ip, dp]),
    "sfgpu_system_autotune": (i32, [vp, i32, ip, dp]),
    "sfgpu_batch_create": (i32, [i32, vp, i32, C.POINTER(vp)]),
    "sfgpu_batch_destroy": (i32, [vp]),
    "sfgpu_batch_info": (i32, [vp, ip, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "sfgpu_batch_set_stream": (i32, [vp, vp]),
    "sfgpu_batch_set_launch": (i32, [vp, i32, i32]),
    "sfgpu_batch_solve": (i32, [vp, dp, dp, f64, i32, f64, ip, ip, dp]),
    "sfgpu_batch_get_phi": (i32, [vp, i32, i32, dp]),
    "sfgpu_batch_load": (i32, [vp, dp]),
    "sfgpu_batch_solve_resident": (i32, [vp, f64, i32, f64]),
    "sfgpu_batch_results": (i32, [vp, dp, ip, ip, dp]),
    "sfgpu_batch_kernel_ms": (i32, [vp, dp]),
    "sfgpu_chain_phi_noalloc": (i32, [vp, i32, ip, i32, C.POINTER(vp), C.POINTER(vp), vp, vp]),
}

_lib = None


class SfgpuError(RuntimeError):
    def __init__(self, code, what):
        super().__init__(f"{what} failed with status {code}: {last_error()}")
        self.code = code


def load():
    """Load the in-tree library, failing loudly when it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libsfgpu.so not built at {LIB_PATH}; run field_b200.build.build()")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in PROTOTYPES.items():
        if not hasattr(lib, name):
            continue
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    _lib = lib
    return lib


def last_error() -> str:
    if _lib is None:
        return ""
    v = _lib.sfgpu_last_error()
    return v.decode() if v else ""


def check(code, what):
    if code != 0:
        raise SfgpuError(code, what)
