"""Batched solving of many SF-SCF instances and the measurement helpers used
by bench.py (roofline figures and launch counts)."""
from __future__ import annotations

import json
import os

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
    K = 6 if spec.lattice.order == 2 else 1
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
                "traffic": kp.get("traffic"), "peak_kind": kind, "kernel": kp["kernel"],
                "bytes_per_launch": kp["bytes"], "ms_per_launch": kp["ms"]}
    ach = prof["bytes_bwd"] / (prof["ms_bwd"] / 1e3) / 1e9
    return {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "traffic": None,
            "peak_kind": kind, "kernel": "step1 (backward step + fused composition)",
            "bytes_per_launch": prof["bytes_bwd"], "ms_per_launch": prof["ms_bwd"],
            "forward_step": {"bytes": prof["bytes_fwd"], "ms": prof["ms_fwd"],
                             "achieved": prof["bytes_fwd"] / (prof["ms_fwd"] / 1e3) / 1e9}}
