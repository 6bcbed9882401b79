"""Host-side mirror of SFbox's solver-facing API over the C ABI.

``System`` owns one SF-SCF system on the GPU (``sfgpu_system``).  Its methods
map onto the reference interfaces: ``residual`` is ``SF_Solve::residuals``
(SF_Solve.cpp:647), ``phi``/``mol_phi`` read ``SF_State::GetPhi`` /
``SF_Molecule::GetPhi`` results, ``free_energy`` is
``SF_MolList1stO::GetFreeEnergy`` (SF_MolList1stO.cpp:606) and ``solve`` runs
``SFNewton::PlainLBFGSDIIS`` (sfnewton.cpp:566) on the device.  The
Lattice-level methods (``propagate``, ``side_fraction``, ``lngn``) take torch
CUDA tensors and mirror ``Lat1stO::PropagateG`` / ``Lat2ndO::PropagateF/B``,
``Lattice::SideFraction`` and ``Lat1stO::ComputeLnGN``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as nat
from .desc import SystemSpec


def _d(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


@dataclass
class SolveResult:
    x: np.ndarray
    status: int
    iterations: int
    error: float

    @property
    def converged(self) -> bool:
        return self.status == 0


class System:
    def __init__(self, spec: SystemSpec, checkpoint_stride: int = 0):
        """checkpoint_stride k > 0: residual evaluations keep every k-th
        forward slice of a copolymer or second-order chain and recompute the
        rest (sfgpu_system_create_checkpointed)."""
        self.lib = nat.load()
        self.spec = spec
        self._desc = spec.to_c()
        h = C.c_void_p()
        if checkpoint_stride:
            nat.check(self.lib.sfgpu_system_create_checkpointed(C.byref(self._desc), int(checkpoint_stride),
                                                                 C.byref(h)), "sfgpu_system_create_checkpointed")
        else:
            nat.check(self.lib.sfgpu_system_create(C.byref(self._desc), C.byref(h)), "sfgpu_system_create")
        self.h = h
        M, nv, nc, ns = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        nat.check(self.lib.sfgpu_system_info(h, C.byref(M), C.byref(nv), C.byref(nc), C.byref(ns)), "info")
        self.M, self.nvar, self.nclass, self.nsites = M.value, nv.value, nc.value, ns.value
        self.K = spec.lattice.components

    def close(self):
        if getattr(self, "h", None):
            self.lib.sfgpu_system_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- SF_Solve-level ----------------------------------------------------
    def residual(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.size != self.nvar:
            raise ValueError(f"x has {x.size} values, system has {self.nvar} iteration variables")
        f = np.empty(self.nvar)
        nat.check(self.lib.sfgpu_residual_host(self.h, _d(x), _d(f)), "sfgpu_residual_host")
        return f

    def residual_device(self, x_ptr: int, f_ptr: int):
        """x -> f on device pointers, asynchronous on the system's stream."""
        nat.check(self.lib.sfgpu_residual(self.h, C.c_void_p(x_ptr), C.c_void_p(f_ptr)), "sfgpu_residual")

    def use_stream(self, stream_handle: int):
        """Launch on a caller-owned CUDA stream (e.g. torch's current stream)."""
        nat.check(self.lib.sfgpu_system_set_stream(self.h, C.c_void_p(stream_handle)), "set_stream")

    def synchronize(self):
        nat.check(self.lib.sfgpu_synchronize(self.h), "sfgpu_synchronize")

    def phi(self, seg: int) -> np.ndarray:
        out = np.empty(self.M)
        nat.check(self.lib.sfgpu_get_phi(self.h, seg, _d(out)), "sfgpu_get_phi")
        return out

    def mol_phi(self, mol: int, seg: int) -> np.ndarray:
        out = np.empty(self.M)
        nat.check(self.lib.sfgpu_get_mol_phi(self.h, mol, seg, _d(out)), "sfgpu_get_mol_phi")
        return out

    def swf(self, seg: int) -> np.ndarray:
        out = np.empty(self.M)
        nat.check(self.lib.sfgpu_get_swf(self.h, seg, _d(out)), "sfgpu_get_swf")
        return out

    def mol_scalars(self, mol: int):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        nat.check(self.lib.sfgpu_get_mol_scalars(self.h, mol, C.byref(a), C.byref(b), C.byref(c)),
                  "sfgpu_get_mol_scalars")
        return {"lngn": a.value, "phibulk": b.value, "lnc": c.value}

    def lattice_weights(self):
        """(weights of lnGN sums, weights of lattice sums such as F and theta)."""
        a, b = np.empty(self.M), np.empty(self.M)
        nat.check(self.lib.sfgpu_lattice_weights(self.h, _d(a), _d(b)), "sfgpu_lattice_weights")
        return a, b

    def thermo(self):
        """(F, Omega, free-energy density, grand-potential density) of the
        last evaluation (sfgpu_thermo)."""
        F, Om = C.c_double(), C.c_double()
        fe, gp = np.empty(self.M), np.empty(self.M)
        nat.check(self.lib.sfgpu_thermo(self.h, C.byref(F), C.byref(Om), _d(fe), _d(gp)), "sfgpu_thermo")
        return F.value, Om.value, fe, gp

    def set_bond_orientation(self, enable: bool = True):
        """Fill bond-orientation profiles in the following evaluations
        (second-order lattices; Lat2ndO::ConnectG with PHI)."""
        nat.check(self.lib.sfgpu_system_set_bond_orientation(self.h, int(bool(enable))),
                  "sfgpu_system_set_bond_orientation")

    def bond_orientation(self, mol: int, axis: int) -> np.ndarray:
        """Molecule mol's bond-orientation profile along axis 0 (x), 1 (y, yz
        in 1D) or 2 (z), summed over its segment types
        (SF_Copol2ndO::GetBondOrientation)."""
        out = np.empty(self.M)
        nat.check(self.lib.sfgpu_get_bond_orientation(self.h, int(mol), int(axis), _d(out)),
                  "sfgpu_get_bond_orientation")
        return out

    def free_energy(self) -> float:
        F = C.c_double()
        nat.check(self.lib.sfgpu_free_energy(self.h, C.byref(F)), "sfgpu_free_energy")
        return F.value

    def solve(self, x0=None, tol=1e-7, maxit=5000, m=5, eta=0.1) -> SolveResult:
        x = np.zeros(self.nvar) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).copy()
        it, err = C.c_int(), C.c_double()
        rc = self.lib.sfgpu_solve_diis(self.h, _d(x), tol, maxit, m, eta, C.byref(it), C.byref(err))
        if rc not in (0, 5, 4):
            nat.check(rc, "sfgpu_solve_diis")
        return SolveResult(x, rc, it.value, err.value)

    def solve_newton(self, x0=None, tol=1e-7, maxit=5000, pseudohessian=True, deltamax=0.5, **extra) -> SolveResult:
        """SFbox's Newton iteration (SFNewton::iterate, Scheutjens step search)
        over the device residual (sfgpu_solve_newton); extra keys override the
        other sfgpu_newton_settings fields."""
        from .desc import NewtonSettings
        st = NewtonSettings()
        nat.check(self.lib.sfgpu_newton_default_settings(C.byref(st)), "sfgpu_newton_default_settings")
        st.tolerance, st.iterationlimit = float(tol), int(maxit)
        st.pseudohessian, st.deltamax = int(bool(pseudohessian)), float(deltamax)
        for k, v in extra.items():
            setattr(st, k, v)
        x = np.zeros(self.nvar) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).copy()
        it, nf, acc = C.c_int(), C.c_int(), C.c_double()
        rc = self.lib.sfgpu_solve_newton(self.h, _d(x), C.byref(st), C.byref(it), C.byref(nf), C.byref(acc))
        if rc not in (0, 4, 5):
            nat.check(rc, "sfgpu_solve_newton")
        r = SolveResult(x, rc, it.value, acc.value)
        r.evaluations = nf.value
        return r

    def jvp(self, x, v):
        """(f(x), J(x) v) with the exact forward-mode tangent."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        v = np.ascontiguousarray(v, dtype=np.float64)
        f = np.empty(self.nvar)
        jv = np.empty(self.nvar)
        nat.check(self.lib.sfgpu_jvp_host(self.h, _d(x), _d(v), _d(f), _d(jv)), "sfgpu_jvp_host")
        return f, jv

    def vjp(self, x, w):
        """(f(x), J(x)^T w) from the adjoint sweep (first-order lattices and Lat3D2ndO)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        w = np.ascontiguousarray(w, dtype=np.float64)
        f = np.empty(self.nvar)
        xb = np.empty(self.nvar)
        nat.check(self.lib.sfgpu_vjp_host(self.h, _d(x), _d(w), _d(f), _d(xb)), "sfgpu_vjp_host")
        return f, xb

    def vjp_chi(self, x, w) -> np.ndarray:
        """d (w . f(x)) / d chi at fixed x, as an nseg x nseg array (sfgpu_vjp_chi)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        w = np.ascontiguousarray(w, dtype=np.float64)
        ns = len(self.spec.segments)
        out = np.zeros(ns * ns)
        nat.check(self.lib.sfgpu_vjp_chi(self.h, _d(x), _d(w), _d(out)), "sfgpu_vjp_chi")
        return out.reshape(ns, ns)

    def free_energy_grad(self, x):
        """(F(x), dF/dx) with the exact gradient from the reverse sweep (sfgpu_free_energy_grad)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        F = C.c_double()
        g = np.empty(self.nvar)
        nat.check(self.lib.sfgpu_free_energy_grad(self.h, _d(x), C.byref(F), _d(g)), "sfgpu_free_energy_grad")
        return F.value, g

    def phi_sensitivity_chi(self, x, omega, rtol=1e-10, krylov=40, maxcycles=20):
        """dL/d chi at a solution x for L = sum omega . phi (nseg x M weights),
        through the solution's dependence on chi (sfgpu_phi_sensitivity_chi).
        Returns (nseg x nseg array, relative residual of the adjoint solve)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        om = np.ascontiguousarray(omega, dtype=np.float64).reshape(-1)
        ns = len(self.spec.segments)
        if om.size != ns * self.M:
            raise ValueError(f"omega has {om.size} values, expected {ns} x {self.M}")
        out = np.zeros(ns * ns)
        rr = C.c_double()
        nat.check(self.lib.sfgpu_phi_sensitivity_chi(self.h, _d(x), _d(om), _d(out), rtol, krylov, maxcycles,
                                                     C.byref(rr)), "sfgpu_phi_sensitivity_chi")
        return out.reshape(ns, ns), rr.value

    def set_checkpoint(self, stride: int):
        """Reverse-sweep memory: 0 stores every slice, k > 0 keeps checkpoints
        every k positions and recomputes segments (sfgpu_system_set_checkpoint)."""
        nat.check(self.lib.sfgpu_system_set_checkpoint(self.h, int(stride)), "sfgpu_system_set_checkpoint")

    def autotune_checkpoint(self, x, reps: int = 3, max_bytes: float = 0.0):
        """Checkpoint stride of the reverse sweep by timing candidate strides
        at x (sfgpu_system_autotune_checkpoint); returns (stride, ms)."""
        k, ms = C.c_int(), C.c_double()
        x = np.ascontiguousarray(x, dtype=np.float64)
        nat.check(self.lib.sfgpu_system_autotune_checkpoint(self.h, _d(x), int(reps), float(max_bytes), C.byref(k),
                                                             C.byref(ms)), "sfgpu_system_autotune_checkpoint")
        return k.value, ms.value

    def solve_lbfgs(self, x0=None, tol=1e-7, maxit=2000, m=10) -> SolveResult:
        """L-BFGS on |f|^2/2 with the adjoint gradient (sfgpu_solve_lbfgs)."""
        x = np.zeros(self.nvar) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).copy()
        it, ne, err = C.c_int(), C.c_int(), C.c_double()
        rc = self.lib.sfgpu_solve_lbfgs(self.h, _d(x), tol, maxit, m, C.byref(it), C.byref(ne), C.byref(err))
        if rc not in (0, 4, 5):
            nat.check(rc, "sfgpu_solve_lbfgs")
        r = SolveResult(x, rc, it.value, err.value)
        r.evaluations = ne.value
        return r

    def solve_nk(self, x0=None, tol=1e-7, maxit=50, krylov=30) -> SolveResult:
        """Newton-Krylov with exact J*v (sfgpu_solve_nk)."""
        x = np.zeros(self.nvar) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).copy()
        it, nj, err = C.c_int(), C.c_int(), C.c_double()
        rc = self.lib.sfgpu_solve_nk(self.h, _d(x), tol, maxit, krylov, C.byref(it), C.byref(nj), C.byref(err))
        if rc not in (0, 4, 5):
            nat.check(rc, "sfgpu_solve_nk")
        r = SolveResult(x, rc, it.value, err.value)
        r.jvps = nj.value
        return r

    def profile_propagator(self, reps: int = 200):
        a, b, c, d = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        nat.check(self.lib.sfgpu_profile_propagator(self.h, reps, C.byref(a), C.byref(b), C.byref(c), C.byref(d)),
                  "sfgpu_profile_propagator")
        return {"ms_fwd": a.value, "ms_bwd": b.value, "bytes_fwd": c.value, "bytes_bwd": d.value}

    def autotune(self, reps: int = 20):
        x, ms = C.c_int(), C.c_double()
        nat.check(self.lib.sfgpu_system_autotune(self.h, reps, C.byref(x), C.byref(ms)), "sfgpu_system_autotune")
        return {"tile_xc": x.value, "ms_fwd_plus_bwd": ms.value}

    def set_tile_pipelined(self, enable):
        """Form of the 3D first-order step: False/0 plain, True/1 pipelined,
        2 pipelined with two y rows per thread in the forward steps."""
        nat.check(self.lib.sfgpu_system_set_tile_pipelined(self.h, int(enable)), "set_tile_pipelined")

    def set_tile(self, xc: int):
        nat.check(self.lib.sfgpu_system_set_tile(self.h, xc), "sfgpu_system_set_tile")

    # ---- Lattice-level (torch CUDA tensors) -------------------------------
    def _sync_torch(self):
        import torch
        torch.cuda.synchronize()

    def propagate(self, gin, g, S: float = 0.2, backward: bool = False):
        import torch
        # zeroed: the lumped second-order steps write interior entries only,
        # and a surface layer, which later steps read, holds 0 in a propagator
        out = torch.zeros_like(gin)
        self._sync_torch()
        nat.check(self.lib.sfgpu_lat_propagate(self.h, C.c_void_p(gin.data_ptr()), C.c_void_p(g.data_ptr()),
                                               C.c_void_p(out.data_ptr()), float(S), int(backward)),
                  "sfgpu_lat_propagate")
        self.synchronize()
        return out

    def side_fraction(self, phi):
        import torch
        out = torch.empty_like(phi)
        self._sync_torch()
        nat.check(self.lib.sfgpu_lat_side_fraction(self.h, C.c_void_p(phi.data_ptr()), C.c_void_p(out.data_ptr())),
                  "sfgpu_lat_side_fraction")
        self.synchronize()
        return out

    def set_boundaries(self, p):
        self._sync_torch()
        comps = p.numel() // self.M
        nat.check(self.lib.sfgpu_lat_set_boundaries(self.h, C.c_void_p(p.data_ptr()), comps), "set_boundaries")
        self.synchronize()
        return p

    def connect(self, gb, gf, phi):
        """phi += sum_k gb_k gf_k (ConnectG), in place on device tensors."""
        self._sync_torch()
        nat.check(self.lib.sfgpu_lat_connect(self.h, C.c_void_p(gb.data_ptr()), C.c_void_p(gf.data_ptr()),
                                             C.c_void_p(phi.data_ptr()), gb.numel() // self.M),
                  "sfgpu_lat_connect")
        self.synchronize()
        return phi

    def correct_double_count(self, phi, g):
        """phi /= g where g > 0, else 0 (CorrectDoubleCountG), in place."""
        self._sync_torch()
        nat.check(self.lib.sfgpu_lat_correct_double_count(self.h, C.c_void_p(phi.data_ptr()),
                                                          C.c_void_p(g.data_ptr())),
                  "sfgpu_lat_correct_double_count")
        self.synchronize()
        return phi

    def norm_phi_free(self, phi, c: float):
        """phi *= c (NormPhiFree), in place."""
        self._sync_torch()
        nat.check(self.lib.sfgpu_lat_norm_phi_free(self.h, C.c_void_p(phi.data_ptr()), float(c)),
                  "sfgpu_lat_norm_phi_free")
        self.synchronize()
        return phi

    def norm_phi_restr(self, phi, gb, c: float):
        """phi *= c / exp(lnGN(gb)) (second order: c / (6 exp(lnGN))), in place
        (NormPhiRestr)."""
        self._sync_torch()
        nat.check(self.lib.sfgpu_lat_norm_phi_restr(self.h, C.c_void_p(phi.data_ptr()), C.c_void_p(gb.data_ptr()),
                                                    gb.numel() // self.M, float(c)),
                  "sfgpu_lat_norm_phi_restr")
        self.synchronize()
        return phi

    def lngn(self, g) -> float:
        self._sync_torch()
        v = C.c_double()
        nat.check(self.lib.sfgpu_lat_lngn(self.h, C.c_void_p(g.data_ptr()), g.numel() // self.M, C.byref(v)),
                  "sfgpu_lat_lngn")
        return v.value


def solve_diis_many(systems, x0s, tol=1e-7, maxit=5000, m=5, eta=0.1, threads=0):
    """Pure_DIIS on many systems at once, one stream and host thread each
    (sfgpu_solve_diis_many).  Returns a list of SolveResult."""
    lib = nat.load()
    n = len(systems)
    xs = [np.ascontiguousarray(x, dtype=np.float64).copy() for x in x0s]
    hs = (C.c_void_p * n)(*[s.h for s in systems])
    xp = (C.POINTER(C.c_double) * n)(*[_d(x) for x in xs])
    st = (C.c_int * n)()
    it = (C.c_int * n)()
    er = (C.c_double * n)()
    nat.check(lib.sfgpu_solve_diis_many(n, hs, xp, tol, maxit, m, eta, threads, st, it, er), "sfgpu_solve_diis_many")
    return [SolveResult(xs[i], st[i], it[i], er[i]) for i in range(n)]
