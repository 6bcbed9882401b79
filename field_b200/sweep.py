"""Parameter sweeps: SFbox's ``var :`` statement solved as batched instances.

SFbox runs the calculations of a sweep one after another
(``Vary::NextCalculation``, Vary.cpp:127-204, driven by SF_Box.cpp:145-177),
each starting from the previous calculation's result (``newton : initial_guess
: previous_result``, the default, SF_Solve.cpp:367-404).  Here the sweep's
calculations are expanded up front (:func:`sweep_calculations`, the same
values in the same order as ``Vary``) and solved together by the batched
persistent kernel (:class:`field_b200.batch.BatchSolver`) in ``waves``:

* wave 0 holds every ``waves``-th point starting at the first, solved from
  the base initial guess;
* wave j holds the points one after those of wave j-1, each started from
  its predecessor's converged potentials -- exactly the start SFbox gives
  it.

``waves=1`` solves every point in one launch from the base guess; ``waves``
equal to the number of points reproduces SFbox's chain point by point.
Warm starts need the same iteration-variable layout; when the varied
parameter changes it (for example ``n_layers``) every point starts cold.
With Pure_DIIS, whose first step replaces the guess by -eta g(guess)
(sfnewton.cpp:578-584), a warm start changes only that first gradient.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from .sfinput import Key, build_system

# Vary.h:12
MAX_CALCULATIONS = 10000000

_VAR_KEYWORDS = ("type", "scale", "end_value", "output_name", "step")


@dataclass
class Variation:
    """One ``var : <class> : <instance> : <parameter>`` statement with its
    ``step``, ``end_value``, ``scale`` and ``type`` (Vary.cpp:4-104)."""
    cls: str
    instance: str
    parameter: str
    start: float
    end: float
    step: float
    scale: str              # "linear" or "exponential"
    vtype: str              # "integer" or "real"
    output_name: str = ""
    values: List[float] = field(default_factory=list)

    @property
    def name(self) -> str:
        """Vary::GetVariableName (Vary.cpp:215-221)."""
        return self.output_name or self.parameter


def _set_value(v: float, vtype: str) -> float:
    """The value SFbox writes back into the input (Text::Putint of int(v), or
    Putreal with 15 digits) and reads again as a number."""
    if vtype == "integer":
        return float(int(v))
    return float(f"{v:.15g}")


def expand_variation(calc: Dict[Key, str]) -> Optional[Variation]:
    """The sequence of values of the varied parameter, as Vary's
    constructor and NextCalculation produce them; None without a ``var``."""
    classes = []
    for (c, n, _p) in calc:
        if c == "var" and n not in classes:
            classes.append(n)
    if not classes:
        return None
    if len(classes) > 1:
        raise ValueError("var : only one class can be varied per calculation")
    cn = classes[0]
    params = {p: v for (c, n, p), v in calc.items() if c == "var" and n == cn}
    inst = [p for p in params if p not in _VAR_KEYWORDS]
    if len(inst) != 1:
        raise ValueError("var : name exactly one parameter to vary (Vary.cpp:30-46)")
    instance = inst[0]
    parameter = params[instance]
    if (cn, instance, parameter) not in calc:
        raise ValueError("var : you can only vary a variable that is set in the input file")
    if "step" not in params or "end_value" not in params or "type" not in params:
        raise ValueError("var : needs step, end_value and type")
    scale = params.get("scale", "linear")
    vtype = params["type"]
    if scale not in ("linear", "exponential") or vtype not in ("integer", "real"):
        raise ValueError("var : scale is linear or exponential, type integer or real")
    start = float(calc[(cn, instance, parameter)])
    step = float(params["step"])
    end = float(int(float(params["end_value"]))) if vtype == "integer" else float(params["end_value"])
    var = Variation(cn, instance, parameter, start, end, step, scale, vtype, params.get("output_name", ""))
    # constructor: number of calculations and the direction of the step
    if scale == "linear":
        q = (end - start) / step
        ncalc = int(q) + 1 + (1 if int(q) < q else 0)
        if ncalc <= 1:
            raise ValueError("var : invalid end_value/step combination; maybe step should be of opposite sign")
        if end - start < 0 and step > 0:
            step = -step
        if end - start > 0 and step < 0:
            step = -step
    else:
        q = abs((math.log10(abs(end)) - math.log10(abs(start))) * step)
        ncalc = int(q) + 1 + (1 if int(q) < q else 0)
        if abs(math.log10(abs(end)) - math.log10(abs(start))) <= 0:
            raise ValueError("var : invalid end_value/step combination")
        if math.log(end) - math.log(start) < 0 and step > 0:
            step = -step
        if math.log(end) - math.log(start) > 0 and step < 0:
            step = -step
    if ncalc > MAX_CALCULATIONS:
        raise ValueError("var : maximum number of calculations exceeded")
    var.step = step
    # NextCalculation: the first call keeps the start value
    cur = start
    values = [start]
    while True:
        if vtype == "integer":
            if int(cur) - int(end) >= 0 and step > 0:
                break
            if int(cur) - int(end) <= 0 and step < 0:
                break
        if scale == "linear":
            if vtype == "real" and abs(cur - end) < abs(step / MAX_CALCULATIONS):
                break
            old = cur
            if vtype == "integer":
                while int(cur) - int(old) == 0:
                    cur += step
            else:
                cur += step
        else:
            if vtype == "real" and abs(cur - end) < abs(cur / MAX_CALCULATIONS):
                break
            old = cur
            f = math.exp(math.log(10.0) / step)
            if vtype == "integer":
                while int(cur) - int(old) == 0:
                    cur *= f
            else:
                cur *= f
        if cur > end and step > 0:
            cur = end
        elif cur < end and step < 0:
            cur = end
        values.append(_set_value(cur, vtype))
        if len(values) > MAX_CALCULATIONS:
            raise ValueError("var : maximum number of calculations exceeded")
    var.values = values
    return var


def sweep_calculations(calc: Dict[Key, str]) -> Tuple[Optional[Variation], List[Dict[Key, str]]]:
    """The calculations of one input calculation's sweep: copies of calc with
    the varied parameter set to each value (and the var statements removed)."""
    var = expand_variation(calc)
    base = {k: v for k, v in calc.items() if k[0] != "var"}
    if var is None:
        return None, [base]
    out = []
    for v in var.values:
        c = dict(base)
        c[(var.cls, var.instance, var.parameter)] = str(int(v)) if var.vtype == "integer" else repr(v)
        out.append(c)
    return var, out


def batchable(spec) -> bool:
    """Whether the batched persistent kernel takes this system: first order,
    no overflow protection, no charges, and linear chains (the FCC, HEX and
    stencils lattice types and the force ensemble run in the kernel's wide
    instantiation; dendrimers, branched molecules, rings and charged systems
    on the single-system path)."""
    return (spec.lattice.order == 1 and not getattr(spec, "overflow_protection", False)
            and not getattr(spec, "charged", False)
            and all(not m.generations and m.bond_parent is None and not m.ring for m in spec.molecules))


@dataclass
class SweepResult:
    variation: Optional[Variation]
    specs: list
    x: List[np.ndarray]
    status: np.ndarray
    iterations: np.ndarray
    wave: np.ndarray            # wave in which each point was solved

    @property
    def converged(self) -> np.ndarray:
        return self.status == 0


def solve_sweep(calc: Dict[Key, str], waves: int = 1, x0: Optional[np.ndarray] = None, tol: Optional[float] = None,
                maxit: Optional[int] = None, m: Optional[int] = None, eta: float = 0.1) -> SweepResult:
    """Solve every point of the sweep of ``calc`` with Pure_DIIS on the
    device, ``waves`` batched launches (see the module docstring).  x0 is the
    base initial guess (zeros when None); tol / maxit / m default to the
    input's ``newton`` settings."""
    from .batch import BatchSolver
    from .system import System
    var, calcs = sweep_calculations(calc)
    built = [build_system(c) for c in calcs]
    specs = [s for s, _ in built]
    st = built[0][1]
    tol = st.tolerance if tol is None else tol
    maxit = st.iterationlimit if maxit is None else maxit
    m = st.m if m is None else m
    n = len(specs)
    waves = max(1, min(int(waves), n))
    nv = [s.n_itvar() for s in specs]
    same_layout = all(v == nv[0] for v in nv)
    if not same_layout:
        waves = 1
    xs: List[Optional[np.ndarray]] = [None] * n
    status = np.zeros(n, dtype=np.int32)
    iters = np.zeros(n, dtype=np.int32)
    wave_of = np.array([i % waves for i in range(n)], dtype=np.int32)
    for w in range(waves):
        idx = [i for i in range(n) if i % waves == w]
        guesses = []
        for i in idx:
            if w > 0:
                guesses.append(xs[i - 1])
            elif x0 is not None and same_layout:
                guesses.append(np.asarray(x0, dtype=np.float64))
            else:
                guesses.append(np.zeros(nv[i]))
        if all(batchable(specs[i]) for i in idx):
            bs = BatchSolver([specs[i] for i in idx], m=m, eta=eta)
            res = bs.solve(np.concatenate(guesses), tol=tol, maxit=maxit)
            parts = bs.split(res.x)
            for j, i in enumerate(idx):
                xs[i] = np.array(parts[j])
                status[i] = res.status[j]
                iters[i] = res.iterations[j]
            bs.close()
        else:
            # second-order and twelve-neighbour lattices: the host-driven device
            # iteration, one point at a time
            for j, i in enumerate(idx):
                r = System(specs[i]).solve(guesses[j], tol=tol, maxit=maxit, m=m, eta=eta)
                xs[i] = r.x
                status[i] = r.status
                iters[i] = r.iterations
    return SweepResult(var, specs, xs, status, iters, wave_of)
