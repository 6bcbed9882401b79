"""Batched solving of many SF-SCF instances and the measurement helpers used
by bench.py (roofline figures and launch counts)."""
from __future__ import annotations

import ctypes as C
import json
import os
from dataclasses import dataclass

import numpy as np

from . import _native as nat
from .desc import SystemDesc

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def default_batch() -> int:
    return 296


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def launches_per_residual(spec) -> int:
    """Kernel launches of one single-system residual evaluation
    (sfgpu_system::residual_async): SWF updates, per-molecule propagation,
    state sums, bulk scalars and the residual kernel."""
    K = spec.lattice.components
    n = 0
    for s in spec.segments:
        if s.freedom != 1:
            n += 2  # swf update + state sum
    for mol in spec.molecules:
        N = mol.N
        used = len({b[0] for b in mol.blocks})
        if N == 1:
            n += 3
        elif used == 1 and K == 1:
            half = N // 2
            n += (half - 1) + (N % 2) + (N - (N + 3) // 2 + 1) + 2 + 1
        else:
            n += 1 + (2 if K == 6 else 0) + (N - 1) + 1 + 1 + (N - 1) + 2 + used
    return n + 2


def launch_count(form: str, iterations_total: int, insts, solver=None) -> int:
    if form == "chosen" and solver is not None:
        return solver.launches_in_last_solve_total
    per = launches_per_residual(insts[0][0])
    n_inst = len(insts)
    # per DIIS iteration: residual + step + dots + sum + combine; plus the start
    return iterations_total * (per + 4) + n_inst * (per + 3)


def roofline(prof: dict, form: str, solver=None) -> dict:
    peak, kind = measured_peaks()
    if form == "chosen" and solver is not None and getattr(solver, "kernel_profile", None):
        kp = solver.kernel_profile
        ach = kp["bytes"] / (kp["ms"] / 1e3) / 1e9
        return {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "traffic": kp.get("traffic"), "traffic_source": kp.get("traffic_source"),
                "peak_kind": kind, "kernel": kp["kernel"],
                "bytes_per_launch": kp["bytes"], "ms_per_launch": kp["ms"]}
    ach = prof["bytes_bwd"] / (prof["ms_bwd"] / 1e3) / 1e9
    return {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "traffic": None,
            "peak_kind": kind, "kernel": "step1 (backward step + fused composition)",
            "bytes_per_launch": prof["bytes_bwd"], "ms_per_launch": prof["ms_bwd"],
            "forward_step": {"bytes": prof["bytes_fwd"], "ms": prof["ms_fwd"],
                             "achieved": prof["bytes_fwd"] / (prof["ms_fwd"] / 1e3) / 1e9}}


@dataclass
class BatchResult:
    x: np.ndarray
    status: np.ndarray
    iterations: np.ndarray
    errors: np.ndarray

    @property
    def converged(self) -> np.ndarray:
        return self.status == 0


def residual_bytes(spec) -> float:
    """Algorithmic bytes of one residual evaluation's propagation: forward
    step 8*(K+1+K) per site, backward step with composition 8*(3K+3) per site
    (read Gb(s+1), G, Gf(s), phi; write Gb(s), phi), per molecule."""
    K = spec.lattice.components
    M = spec.M
    tot = 0.0
    for mol in spec.molecules:
        N = mol.N
        used = len({b[0] for b in mol.blocks})
        if N == 1:
            continue
        if used == 1 and K == 1:
            nf, nb = N // 2 - 1, N - N // 2
        else:
            nf, nb = N - 1, N - 1
        tot += nf * 8.0 * (2 * K + 1) * M + nb * 8.0 * (3 * K + 3) * M
    return tot


class BatchSolver:
    """Many independent instances solved by Pure_DIIS in one persistent
    kernel launch (sfgpu_batch_solve)."""

    def __init__(self, specs, method: str = "diis", m: int = 10, eta: float = 0.1):
        if method != "diis":
            raise ValueError("the batched path implements Pure_DIIS")
        self.lib = nat.load()
        self.specs = list(specs)
        self.m, self.eta = m, eta
        descs = (SystemDesc * len(self.specs))()
        for i, sp in enumerate(self.specs):
            descs[i] = sp.to_c()
        self._descs = descs
        h = C.c_void_p()
        nat.check(self.lib.sfgpu_batch_create(len(self.specs), descs, m, C.byref(h)), "sfgpu_batch_create")
        self.h = h
        n, tot = C.c_int(), C.c_longlong()
        offs = (C.c_longlong * len(self.specs))()
        nat.check(self.lib.sfgpu_batch_info(h, C.byref(n), C.byref(tot), offs), "sfgpu_batch_info")
        self.n, self.total = n.value, tot.value
        self.offsets = np.array(list(offs), dtype=np.int64)
        self.launches_in_last_solve_total = 0
        self.kernel_profile = None

    def close(self):
        if getattr(self, "h", None):
            self.lib.sfgpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def use_stream(self, stream_handle: int):
        nat.check(self.lib.sfgpu_batch_set_stream(self.h, C.c_void_p(stream_handle)), "sfgpu_batch_set_stream")

    def split(self, x):
        ends = list(self.offsets[1:]) + [self.total]
        return [x[a:b] for a, b in zip(self.offsets, ends)]

    def solve(self, x0, tol=1e-7, maxit=2000, out=None) -> BatchResult:
        """Host API: guesses in, iterates out (``out`` may be a caller-owned,
        e.g. pinned, float64 array; by default a new array)."""
        x = np.ascontiguousarray(x0, dtype=np.float64)
        if x.size != self.total:
            raise ValueError(f"x has {x.size} values, batch has {self.total}")
        y = np.empty(self.total) if out is None else out
        st = np.zeros(self.n, dtype=np.int32)
        it = np.zeros(self.n, dtype=np.int32)
        er = np.zeros(self.n)
        dp = C.POINTER(C.c_double)
        nat.check(self.lib.sfgpu_batch_solve(self.h, x.ctypes.data_as(dp), y.ctypes.data_as(dp), tol, maxit,
                                             self.eta, st.ctypes.data_as(C.POINTER(C.c_int)),
                                             it.ctypes.data_as(C.POINTER(C.c_int)), er.ctypes.data_as(dp)),
                  "sfgpu_batch_solve")
        self.launches_in_last_solve_total += 1
        return BatchResult(y, st, it, er)

    def set_launch(self, threads: int, stage: bool = True):
        """Threads per block and shared-memory staging of the persistent
        kernel (sfgpu_batch_set_launch)."""
        nat.check(self.lib.sfgpu_batch_set_launch(self.h, int(threads), int(bool(stage))), "sfgpu_batch_set_launch")

    def autotune(self, x0, tol=1e-7, maxit=2000, candidates=((1024, True), (512, True), (512, False),
                                                             (384, True), (256, True))):
        """Time one solve per launch shape from x0 and keep the fastest;
        returns {(threads, stage): ms}."""
        times = {}
        for th, stg in candidates:
            try:
                self.set_launch(th, stg)
            except nat.SfgpuError:
                continue
            self.load(x0)
            self.solve_resident(tol, maxit)
            self.results()
            times[(th, stg)] = self.kernel_ms()
        best = min(times, key=times.get)
        self.set_launch(*best)
        return times

    def load(self, x0):
        x = np.ascontiguousarray(x0, dtype=np.float64)
        if x.size != self.total:
            raise ValueError(f"x has {x.size} values, batch has {self.total}")
        nat.check(self.lib.sfgpu_batch_load(self.h, x.ctypes.data_as(C.POINTER(C.c_double))), "sfgpu_batch_load")

    def solve_resident(self, tol=1e-7, maxit=2000):
        """Launch the solve on the device-resident iterate (asynchronous)."""
        nat.check(self.lib.sfgpu_batch_solve_resident(self.h, tol, maxit, self.eta), "sfgpu_batch_solve_resident")
        self.launches_in_last_solve_total += 1

    def results(self, want_x: bool = False) -> BatchResult:
        st = np.zeros(self.n, dtype=np.int32)
        it = np.zeros(self.n, dtype=np.int32)
        er = np.zeros(self.n)
        x = np.empty(self.total) if want_x else None
        xp = x.ctypes.data_as(C.POINTER(C.c_double)) if want_x else C.POINTER(C.c_double)()
        nat.check(self.lib.sfgpu_batch_results(self.h, xp, st.ctypes.data_as(C.POINTER(C.c_int)),
                                               it.ctypes.data_as(C.POINTER(C.c_int)),
                                               er.ctypes.data_as(C.POINTER(C.c_double))), "sfgpu_batch_results")
        return BatchResult(x, st, it, er)

    def kernel_ms(self) -> float:
        v = C.c_double()
        nat.check(self.lib.sfgpu_batch_kernel_ms(self.h, C.byref(v)), "sfgpu_batch_kernel_ms")
        return v.value

    def phi(self, inst: int, seg: int) -> np.ndarray:
        out = np.empty(self.specs[inst].M)
        nat.check(self.lib.sfgpu_batch_get_phi(self.h, inst, seg, out.ctypes.data_as(C.POINTER(C.c_double))),
                  "sfgpu_batch_get_phi")
        return out

    def algorithmic_bytes(self, iterations) -> float:
        """Propagator bytes plus DIIS vector traffic of one batch solve."""
        tot = 0.0
        for sp, it in zip(self.specs, iterations):
            nv = sp.n_itvar()
            tot += (int(it) + 1) * residual_bytes(sp)
            tot += int(it) * 8.0 * nv * (self.m + 7)
        return tot
