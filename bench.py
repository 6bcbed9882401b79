"""Benchmark: converged SCF solves per second.

Default workload (the headline): the cylindrical diblock system
(Lat2DCyl1stO 128x128, A20B20 in W, phibulk 0.005, chi_AW 1.6, seeded micelle
+ N(0, 0.1) noise, residual < 1e-7).  ``--config c4`` runs the batching
configuration instead: 256 uneven Lat1DFlat1stO instances (layers 50..400,
N 20..1000) from x = 0.

One step = one batch of instances solved to convergence.  ``--form chosen``
runs the batched persistent solver (one launch per batch), ``--form plain``
the per-instance host-driven form.  The line also carries ``plain_gpu_form``:
per-instance Pure_DIIS with one launch per propagator step on the cylinder,
SFbox's own Newton iteration (pseudohessian) over the device residual on the
1D instances, where its dense Hessian fits.

``--impl reference`` times SFbox itself -- the reference's C++ sources built
by oracle/refbuild (oracle/_ref/sfref) -- on all host cores, one process per
instance, on the same systems and settings; without that build it times the
CPU restatement (oracle) instead and says so.  Under torchrun every rank
solves its own instances, split by estimated cost (weak scaling, no
data-path collective); the timed region is bracketed by a barrier and a
synchronize and the max over ranks is reported.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "converged SCF solves/s (resid<1e-7)"
SFREF = os.path.join(ROOT, "oracle", "_ref", "sfref")
TOL = 1e-7

# workload table: one entry per benchmarked configuration
WORKLOADS = {
    "c2": {"name": "cyl_micelle Lat2DCyl1stO 128x128 (r,z), (A)20(B)20 + W solvent, phibulk 0.005, chi_AW 1.6",
           "m": 10, "eta": 0.1, "maxit": 2000},
    "c4": {"name": "sweep1d: 256 uneven Lat1DFlat1stO instances (layers 50..400, N 20..1000 log-uniform, "
                   "chi_AW grid over [0,1], phibulk 1e-4..1e-1, chi_AS -2..0), (A)N + W at a frozen surface, x0 = 0",
           "m": 5, "eta": 0.1, "maxit": 5000},
}
# ncu: 93.36 GB read + 76.00 GB written by one batch_diis_kernel launch of
# 148 cylinder instances that made 148 * (33.63 + 1) residual evaluations
DRAM_BYTES_PER_INSTANCE_ITERATION_C2 = (93.365e9 + 76.002e9) / (148 * 34.63)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--form", default="chosen", choices=["chosen", "plain"])
    ap.add_argument("--batch", type=int, default=0, help="instances per rank per step (0: form default)")
    ap.add_argument("--cpu-sample", type=int, default=8, help="instances in the CPU-baseline sample")
    ap.add_argument("--plain-sample", type=int, default=16, help="instances timed in the plain GPU form")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# instances: (spec, x0, SFbox input text) per instance
def instances(config: str, rank: int, world: int, count: int):
    from field_b200 import configs
    if config == "c2":
        from field_b200.shard import instance_seeds
        w = WORKLOADS["c2"]
        text = configs.cyl_micelle_input(m=w["m"], eta=w["eta"], tol=TOL, maxit=w["maxit"])
        out = []
        for sd in instance_seeds(rank, count, configs.BASE_SEED + 2):
            spec, x0 = configs.cyl_micelle(seed=sd)
            out.append((spec, x0, text))
        return out
    from field_b200.shard import estimate_cost, partition
    texts = configs.sweep1d_inputs(count=256, tolerance=TOL)
    allinst = [(s, x, t) for (s, x), t in zip(configs.sweep1d(count=256), texts)]
    parts = partition([estimate_cost(s) for s, _, _ in allinst], world)
    mine = [allinst[i] for i in parts[rank]]
    return mine[:count] if count else mine


def reference_text(config: str, text: str) -> str:
    """The SFbox input of one instance with the bench's solver settings."""
    w = WORKLOADS[config]
    if config == "c4":
        text = text.replace("start\n", f"newton : isaac : iterationlimit : {w['maxit']}\nstart\n")
    return text


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [v.strip() for v in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU legs: SFbox itself (oracle/_ref/sfref) when built, else the oracle port
def _sfbox_solve(args):
    """One instance solved by SFbox's own Pure_DIIS in a child process; 1 if
    it stopped on its tolerance test with finite numbers."""
    text, x0_bytes = args
    import numpy as np
    with tempfile.TemporaryDirectory() as wd:
        inp, xf, out = (os.path.join(wd, n) for n in ("c.in", "c.x", "c.out"))
        with open(inp, "w") as f:
            f.write(text)
        with open(xf, "wb") as f:
            f.write(x0_bytes)
        r = subprocess.run([SFREF, "solve", inp, xf, out], capture_output=True, text=True, cwd=wd)
        if r.returncode != 0:
            return 0
        its = [int(ln.split()[2]) for ln in r.stdout.splitlines() if ln.startswith("i = ")]
        g = None
        for line in open(out):
            p = line.split()
            if p[0] == "g":
                g = np.array([float(v) for v in p[2:]])
    maxit = int(text.split("iterationlimit : ")[1].split()[0]) if "iterationlimit : " in text else 5000
    ok = g is not None and bool(np.all(np.isfinite(g))) and (not its or its[-1] < maxit)
    return int(ok)


def _port_solve(args):
    """One instance solved by the oracle's Pure_DIIS (the CPU restatement)."""
    text, x0_bytes = args
    sys.path.insert(0, ROOT)
    import numpy as np
    from field_b200.sfinput import build_system, parse_input
    from oracle.oracle import Oracle
    spec, st = build_system(parse_input(text)[0])
    x0 = np.frombuffer(x0_bytes, dtype="<f8").copy()
    _, rc, _, _ = Oracle(spec).solve_diis(x0, tol=st.tolerance, maxit=st.iterationlimit, m=st.m, eta=st.deltamax)
    return int(rc == 0)


def _cpu_kind():
    return "reference" if os.path.exists(SFREF) else "port"


def _cpu_jobs(config, insts):
    import numpy as np
    return [(reference_text(config, t), np.ascontiguousarray(x, dtype="<f8").tobytes()) for _, x, t in insts]


def cpu_baseline(config: str, sample: int):
    """SFbox (or the port) on one host core over a bounded sample."""
    insts = instances(config, 0, 1, 0)[:sample] if config == "c4" else instances(config, 0, 1, sample)
    fn = _sfbox_solve if _cpu_kind() == "reference" else _port_solve
    jobs = _cpu_jobs(config, insts)
    t0 = time.perf_counter()
    ok = sum(fn(j) for j in jobs)
    dt = time.perf_counter() - t0
    what = "SFbox built from its own sources (oracle/_ref/sfref), Pure_DIIS" if fn is _sfbox_solve else \
        "the oracle's restatement of SFbox's Pure_DIIS"
    w = WORKLOADS[config]
    return {"value": ok / dt, "unit": "solves/s", "cores": 1, "kind": _cpu_kind(),
            "sample": f"{len(jobs)} instances of the workload solved to 1e-7 by {what} (m={w['m']}, "
                      f"eta={w['eta']}) sequentially on one host core, {dt:.1f} s, {ok} converged"}


def run_reference(a, rank, world):
    """--impl reference: SFbox itself on all host cores of rank 0."""
    import multiprocessing as mp
    if rank != 0:
        return None
    cores = os.cpu_count() or 1
    kind = _cpu_kind()
    fn = _sfbox_solve if kind == "reference" else _port_solve
    if a.config == "c2":
        def jobs_for(k):
            from field_b200 import configs
            w = WORKLOADS["c2"]
            text = configs.cyl_micelle_input(m=w["m"], eta=w["eta"], tol=TOL, maxit=w["maxit"])
            out = []
            for i in range(cores):
                _, x0 = configs.cyl_micelle(seed=configs.BASE_SEED + 2 + 1000 + k * cores + i)
                out.append((text, x0.astype("<f8").tobytes()))
            return out
        per_step = cores
    else:
        # one step is the whole sweep, as the batched launch solves it
        allj = _cpu_jobs("c4", instances("c4", 0, 1, 0))

        def jobs_for(k):
            return allj
        per_step = len(allj)
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        for w in range(a.warmup):
            pool.map(fn, jobs_for(10_000 + w))
        times, solved = [], 0
        for k in range(a.steps):
            jobs = jobs_for(k)
            t0 = time.perf_counter()
            solved += sum(pool.map(fn, jobs))
            times.append(time.perf_counter() - t0)
    total = sum(times)
    value = solved / total
    w = WORKLOADS[a.config]
    what = "SFbox built from its own sources (oracle/_ref/sfref), one process per instance" if kind == "reference" \
        else "the oracle's restatement of SFbox (oracle/_ref/sfref not built), one process per instance"
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1000 * total / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": w["name"], "instances_per_step": per_step,
                       "method": "Pure_DIIS, m=%d, eta=%g" % (w["m"], w["eta"]), "tolerance": TOL},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": kind,
                             "sample": f"{per_step} instances per step on {cores} spawned processes: {what}"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return line


# ---------------------------------------------------------------------------
def plain_form(config, insts, stream, steps=1):
    """Per-instance host-driven GPU form: Pure_DIIS with one launch per
    propagator step on the cylinder, SFbox's Newton iteration over the device
    residual on the 1D instances.  Returns (solves/s, a System, iterations,
    converged)."""
    import torch
    from field_b200.system import System
    w = WORKLOADS[config]
    systems = [System(s) for s, _, _ in insts]
    for s in systems:
        s.use_stream(stream.cuda_stream)
    x_host = [torch.from_numpy(x0).pin_memory() for _, x0, _ in insts]

    def run():
        conv, iters = 0, 0
        for s, xh in zip(systems, x_host):
            if config == "c4":
                r = s.solve_newton(xh.numpy(), tol=TOL, maxit=w["maxit"])
            else:
                r = s.solve(xh.numpy(), tol=TOL, maxit=w["maxit"], m=w["m"], eta=w["eta"])
            conv += r.converged
            iters += r.iterations
        return conv, iters
    if config == "c2":
        run()        # warm-up (the 1D Newton form is timed once: its solves take seconds)
    torch.cuda.synchronize()
    t = 0.0
    conv = iters = 0
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        c, it = run()
        e1.record(stream)
        torch.cuda.synchronize()
        t += e0.elapsed_time(e1) / 1000.0
        conv += c
        iters += it
    return conv / t, systems[0], iters, conv


def run_ours(a, rank, world, local_rank):
    import numpy as np
    import torch
    import torch.distributed as dist
    from field_b200 import batch as fbatch

    cfg = a.config
    w = WORKLOADS[cfg]
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()
    if cfg == "c2":
        B = a.batch or (fbatch.default_batch() if a.form == "chosen" else 4)
        insts = instances(cfg, rank, world, B)
    else:
        insts = instances(cfg, rank, world, a.batch)
        B = len(insts)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)   # 256 MB > 126 MB L2

    def barrier():
        if world > 1:
            dist.barrier()

    solver = None
    if a.form == "chosen":
        solver = fbatch.BatchSolver([s for s, _, _ in insts], method="diis", m=w["m"], eta=w["eta"])
        solver.use_stream(stream.cuda_stream)
        x_all = np.concatenate([x for _, x, _ in insts])
        x_pinned = torch.from_numpy(x_all).pin_memory()
        y_pinned = torch.empty_like(x_pinned).pin_memory()
        for _ in range(a.warmup):
            solver.load(x_all)
            solver.solve_resident(TOL, w["maxit"])
            solver.results()
    torch.cuda.synchronize()

    sampler = ClockSampler(local_rank) if rank == 0 else None
    times, conv_total, iters_total, kms = [], 0, 0, []
    barrier()
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
    if a.form == "chosen":
        for _ in range(a.steps):
            flush.zero_()
            solver.load(x_all)                 # inputs resident in HBM before the timed region
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            solver.solve_resident(TOL, w["maxit"])
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1000.0)
            res = solver.results()
            conv_total += int(res.converged.sum())
            iters_total += int(res.iterations.sum())
            kms.append(solver.kernel_ms())
        last_iters = res.iterations
    else:
        v, prof_sys, iters_total, conv_total = plain_form(cfg, insts, stream, steps=a.steps)
        times = [conv_total / v]
    barrier()
    torch.cuda.synchronize()
    clocks = sampler.stop() if sampler else None
    from field_b200.shard import aggregate
    t_max, solved_all = aggregate(sum(times), conv_total, world, dev)
    value = solved_all / t_max

    # e2e through the public API: pinned host guesses in, iterates out, every step
    h2d = sum(x.size for _, x, _ in insts) * 8
    if a.form == "chosen":
        et, econv = 0.0, 0
        for _ in range(a.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = solver.solve(x_pinned.numpy(), tol=TOL, maxit=w["maxit"], out=y_pinned.numpy())
            e1.record(stream)
            torch.cuda.synchronize()
            et += e0.elapsed_time(e1) / 1000.0
            econv += int(r.converged.sum())
        el, ec = aggregate(et, econv, world, dev)
        e2e_value = ec / el
    else:
        e2e_value = value
    e2e = {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d,
           "note": "sfgpu_batch_solve / per-instance solves on pinned host arrays; copies inside every timed step"}

    # plain GPU form on a sample of the same workload, same run
    plain = None
    if a.form == "chosen":
        ns = min(a.plain_sample, len(insts))
        pv, prof_sys, _, pconv = plain_form(cfg, insts[:ns], stream, steps=1)
        plain = {"value": pv, "unit": "solves/s", "instances": ns, "converged": int(pconv),
                 "form": ("per-instance host-driven Pure_DIIS, one launch per propagator step" if cfg == "c2" else
                          "per-instance SFbox Newton iteration (pseudohessian, Scheutjens step search) "
                          "over the device residual, host-driven")}
        kp_bytes = solver.algorithmic_bytes(last_iters)
        prof_k = {"kernel": "batch_diis_kernel (persistent, one launch per batch solve)",
                  "bytes": kp_bytes, "ms": statistics.median(kms)}
        if cfg == "c2":
            # DRAM traffic measured by ncu (dram__bytes_read.sum +
            # dram__bytes_write.sum) on one launch of 148 instances of this
            # workload, per instance and DIIS iteration, scaled to this
            # launch's iterations
            prof_k["traffic"] = DRAM_BYTES_PER_INSTANCE_ITERATION_C2 * float(sum(int(i) + 1 for i in last_iters))
            prof_k["traffic_source"] = "ncu capture of 148 instances, scaled by residual evaluations"
        solver.kernel_profile = prof_k
    prof = prof_sys.profile_propagator(reps=400)
    roof = fbatch.roofline(prof, a.form, solver)
    if a.form == "chosen":
        roof["per_step_kernel"] = fbatch.roofline(prof, "plain", None)

    if rank == 0:
        cpu = cpu_baseline(cfg, a.cpu_sample) if world == 1 else None
        line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": 1000 * t_max / a.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": w["name"], "form": a.form, "instances_per_rank_per_step": B,
                           "method": "Pure_DIIS, m=%d, eta=%g" % (w["m"], w["eta"]),
                           "tolerance": TOL, "iteration_limit": w["maxit"], "converged": int(solved_all),
                           "mean_iterations": iters_total / max(1, conv_total),
                           "l2": "256 MB buffer written between timed steps",
                           "parallelism": f"instances x{world}"},
                "e2e": e2e, "roofline": roof, "plain_gpu_form": plain,
                "chosen_over_plain": (value / plain["value"]) if plain and plain["value"] > 0 else None,
                "cpu_baseline": cpu, "clocks": clocks,
                "gpu_launches": fbatch.launch_count(a.form, iters_total, [(s, x) for s, x, _ in insts], solver)}
        print(json.dumps(line), flush=True)


def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        run_reference(a, rank, world)
        return
    import torch
    import torch.distributed as dist
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    try:
        run_ours(a, rank, world, local_rank)
    finally:
        if world > 1:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
