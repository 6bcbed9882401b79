"""Output files of a calculation in SFbox's formats (Output.cpp).

A solved calculation is turned into SFbox's output lines -- ``class : name :
key : value`` with profiles attached -- restricted to what the SCF path
computes: the system's free energy and grand potential (with their
densities), the lattice description, the chi list, per segment phibulk / theta /
theta excess with the phi and G profiles, per molecule the quantities of
SF_Molecule::GetOutput (SF_Molecule.cpp:355-465) that need no analysis
beyond the path, and the solver's iteration record (SF_Solve.cpp:191-211).
The keys are SFbox's.  Two writers:

* ``ana`` (Output::OutputAna, Output.cpp:322-416): a ``system delimiter``
  header on a new file, then every line ``c : n : k : v``; a profile line is
  followed by its values one per line (boundary layers included unless
  ``write_bounds`` is false), and each calculation ends with ``system
  delimiter`` and a blank line.
* ``kal`` (Output::OutputKal, Output.cpp:640-726): one header row of
  ``c : n : k`` names of the scalar lines, tab separated, on a new file, then
  one row of values per calculation.
* ``vtk`` (Output::OutputVtkProfiles, Output.cpp:727-905): one file per
  calculation (numbered names) with the profiles a template selects.
* ``profiles`` (Output::OutputProfiles, Output.cpp:998-1196): one file per
  calculation (numbered names), the selected profiles as columns beside the
  site coordinates.

Reals -- scalars and profile values -- are printed as SFbox's output streams
print them: scientific with ``accuracy`` significant digits (default
int(-log10(tolerance) + 0.5), SF_Box.cpp:93; Output.cpp:1398-1410).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from .desc import (BOUND_NAMES, GEOM_CYLINDRICAL, GEOM_SPHERICAL, MOL_FREE, MOL_RESTRICTED, SEG_FROZEN,
                   SEG_PINNED)
from .sfinput import Key

_BOUND_TEXT = {v: k for k, v in BOUND_NAMES.items()}


@dataclass
class OutputLine:
    cls: str
    name: str
    key: str
    value: str
    profile: Optional[np.ndarray] = None
    acc: int = 12                     # significant digits of the profile values


def _names(calc: Dict[Key, str], cls: str, default: str) -> str:
    for (c, n, _p) in calc:
        if c == cls:
            return n
    return default


def _real(v: float, acc: int) -> str:
    """A real as SFbox's output streams print it: scientific, acc - 1 digits
    after the point, the point always shown (Output::open, Output.cpp:1398-1410)."""
    return f"{v:.{max(acc - 1, 0)}e}"


def output_lines(calc: Dict[Key, str], spec, sys_, x: np.ndarray, iterations: int, error: float,
                 tolerance: float, iterationlimit: int, calc_number: int,
                 accuracy: Optional[int] = None) -> List[OutputLine]:
    """The output lines of one solved calculation.  sys_ is a
    field_b200.system.System; x its converged iteration variables."""
    acc = accuracy if accuracy is not None else int(-math.log10(tolerance) + 0.5)
    sys_.residual(x)
    F, Om, fe, gp = sys_.thermo()
    w_lngn, w_sum = sys_.lattice_weights()
    out: List[OutputLine] = []
    R = lambda c, n, k, v: out.append(OutputLine(c, n, k, _real(float(v), acc)))
    T = lambda c, n, k, v: out.append(OutputLine(c, n, k, str(v)))
    P = lambda c, n, k, p: out.append(OutputLine(c, n, k, "profile", np.asarray(p, dtype=float), acc))
    sname = _names(calc, "sys", "noname")
    T("sys", sname, "calculation number", calc_number)
    T("sys", sname, "matrix_approach", "second_order" if spec.lattice.order == 2 else "first_order")
    T("sys", sname, "overflow_protection", "true" if getattr(spec, "overflow_protection", False) else "false")
    R("sys", sname, "grand potential", Om)
    R("sys", sname, "free energy", F)
    P("sys", sname, "free energy density", fe)
    P("sys", sname, "grand potential density", gp)
    lat = spec.lattice
    lname = _names(calc, "lat", "lat")
    T("lat", lname, "gradients", lat.gradients)
    geom = {GEOM_CYLINDRICAL: "cylindrical", GEOM_SPHERICAL: "spherical"}.get(lat.geometry, "flat")
    if lat.gradients > 1:
        geom = "flat"   # what Lat2DCylinder::GetOutput writes for the cylinder too (Lat2DCylinder.cpp:91)
    T("lat", lname, "geometry", geom)
    axes = [""] if lat.gradients == 1 else ["_x", "_y", "_z"][:lat.gradients]
    for d, a in enumerate(axes):
        T("lat", lname, "n_layers" + a, lat.n_layers[d])
        T("lat", lname, "lowerbound" + a, _BOUND_TEXT.get(lat.bound_lo[d], "?"))
        T("lat", lname, "upperbound" + a, _BOUND_TEXT.get(lat.bound_hi[d], "?"))
    R("lat", lname, "lambda", lat.lam)
    sites = float(w_sum.sum())
    mols = spec.molecules
    N = [m.N for m in mols]
    phib_m = [sys_.mol_scalars(m)["phibulk"] for m in range(len(mols))]
    # molecules (SF_Molecule::GetOutput, SF_Molecule.cpp:355-465)
    for m, mol in enumerate(mols):
        sc = sys_.mol_scalars(m)
        fr = {MOL_FREE: "free", MOL_RESTRICTED: "restricted"}.get(mol.freedom, "solvent")
        T("mol", mol.name, "freedom", fr)
        R("mol", mol.name, "phibulk", sc["phibulk"])
        R("mol", mol.name, "log(phibulk)", math.log10(sc["phibulk"]) if sc["phibulk"] > 0 else 0.0)
        used = sorted({s for s, _ in mol.blocks})
        phi = sum(sys_.mol_phi(m, s) for s in used)
        theta = float((w_sum * phi).sum())
        exc = float((w_sum * np.where(phi > 0, phi - sc["phibulk"], phi)).sum())
        R("mol", mol.name, "phi-av", theta / sites)
        R("mol", mol.name, "theta", theta)
        R("mol", mol.name, "theta excess", exc)
        R("mol", mol.name, "n", theta / N[m])
        R("mol", mol.name, "n exc", exc / N[m])
        if mol.generations:
            parts = [f"{len(mol.generations)}"]
            for blocks, (_nb, f) in zip(mol.generation_blocks(), mol.generations):
                parts += ["".join(f"({spec.segments[s].name}){n}" for s, n in blocks), str(f)]
            comp = "@dend(" + ",".join(parts) + ")"
        else:
            comp = "".join(f"({spec.segments[s].name}){n}" for s, n in mol.blocks)
        T("mol", mol.name, "composition", comp)
        T("mol", mol.name, "chainlength", N[m])
        R("mol", mol.name, "ln(G(N|1))", sc["lngn"])
        R("mol", mol.name, "force", getattr(mol, "force", 0.0))
        R("mol", mol.name, "ln(norm_restricted)" if mol.freedom == MOL_RESTRICTED else "ln(norm_free)", sc["lnc"])
        P("mol", mol.name, "phi", phi)
    # chi list, then the segments (SF_SegmentList::GetOutput, SF_SegmentList.cpp:387-405;
    # SF_Segment::GetOutput, SF_Segment.cpp:345-402), after the molecules as SFbox
    # writes them
    ns = len(spec.segments)
    chi = np.asarray(spec.chi, dtype=float).reshape(ns, ns)
    for i in range(ns):
        for j in range(ns):
            if i != j:
                R("chi list", spec.segments[i].name, "chi - " + spec.segments[j].name, chi[i, j])
    for i, seg in enumerate(spec.segments):
        fr = {SEG_FROZEN: "frozen", SEG_PINNED: "pinned"}.get(seg.freedom, "free")
        T("mon", seg.name, "freedom", fr)
        phi = sys_.phi(i)
        pb = 0.0
        if seg.freedom != SEG_FROZEN:
            for m, mol in enumerate(mols):
                cnt = mol.count(i)
                pb += phib_m[m] * cnt / N[m]
        R("mon", seg.name, "phibulk", pb)
        theta = float((w_sum * phi).sum())
        R("mon", seg.name, "theta", theta)
        R("mon", seg.name, "theta excess", theta - sites * pb)
        R("mon", seg.name, "valence", getattr(seg, "valence", 0.0))
        R("mon", seg.name, "epsilon", getattr(seg, "epsilon", 80.0) or 80.0)
        R("mon", seg.name, "int.free energy", 0.0)   # internal states: none without reactions
        P("mon", seg.name, "phi", phi)
        if seg.freedom != SEG_FROZEN:
            P("mon", seg.name, "G", sys_.swf(i))
    nname = _names(calc, "newton", "noname")
    T("newton", nname, "iterations", int(iterations))
    T("newton", nname, "iterationlimit", int(iterationlimit))
    R("newton", nname, "accuracy", error)
    R("newton", nname, "tolerance", tolerance)
    T("newton", nname, "number iter var", spec.n_itvar())
    return out


def write_ana(path: str, lines: List[OutputLine], first: bool, write_bounds: bool = True,
              lattice_shape: Tuple[int, ...] = ()) -> None:
    """Append one calculation in the ana format (see the module docstring)."""
    interior = None
    if not write_bounds and lattice_shape:
        mask = np.zeros(lattice_shape, bool)
        mask[(slice(1, -1),) * len(lattice_shape)] = True
        interior = mask.ravel()
    with open(path, "w" if first else "a") as f:
        if first:
            f.write("system delimiter\n\n")
        for ln in lines:
            f.write(f"{ln.cls} : {ln.name} : {ln.key} : {ln.value}\n")
            if ln.profile is not None:
                vals = ln.profile if interior is None else ln.profile[interior]
                f.write("".join(_real(v, ln.acc) + "\n" for v in vals))
        f.write("system delimiter\n\n")


def write_kal(path: str, lines: List[OutputLine], first: bool) -> None:
    """Append one calculation in the kal format (see the module docstring)."""
    scal = [ln for ln in lines if ln.profile is None]
    with open(path, "w" if first else "a") as f:
        if first:
            f.write("\t".join(f"{ln.cls} : {ln.name} : {ln.key}" for ln in scal) + "\n")
        f.write("\t".join(ln.value for ln in scal) + "\n")


def _wild(pattern: str, text: str) -> bool:
    """WildCompare (Input.cpp:977-1030): '*' stands for any run of characters."""
    import re
    return re.fullmatch(".*".join(re.escape(p) for p in pattern.split("*")), text) is not None


def read_template(path: str) -> List[Tuple[str, str, str]]:
    """The ``class : name : key`` triples of an output template file (an
    input file whose lines name the output lines to write)."""
    out = []
    with open(path) as f:
        for raw in f:
            parts = [p.strip() for p in raw.split(":")]
            if len(parts) >= 3 and parts[0] and not parts[0].startswith("//"):
                out.append((parts[0], parts[1], parts[2]))
    return out


def in_template(template, line: OutputLine) -> bool:
    """Output::ValueInTemplate (Output.cpp:1264-1268)."""
    return any(_wild(a, line.cls) and _wild(b, line.name) and _wild(c, line.key) for a, b, c in template)


def vary_value_text(variation, value: float) -> str:
    """Vary::GetCurrValue (Vary.cpp:227-290), the value put into numbered
    file names: integers zero-padded to the digits of the larger end point;
    linear reals as %.5f of the value over 10^e followed by 'e' and e printed
    unsigned, e = int(log10 of the larger end point); exponential sweeps
    (Text::Putreal there) as %g with that many significant digits."""
    big = max(abs(variation.start), abs(variation.end))
    if variation.scale == "linear":
        if variation.vtype == "integer":
            width = min(int(math.log10(big)) + 1, 100) if big > 0 else 1
            return f"{int(value):0{width}d}"
        expo = int(math.log10(big)) if big > 0 else 0
        return f"{value / 10.0 ** expo:.5f}e{expo & 0xFFFFFFFF}"
    f = math.exp(math.log(10.0) / variation.step)
    width = int(math.log10(abs(value / (value * f - value)))) + 1
    if width == 1:
        width = 2
    return f"{value:.{width}g}"


def numbered_filename(name: str, calc_number: int, total_calcs: int, variation=None, value=None) -> str:
    """Output::getNumberedFilename (Output.cpp:1291-1350): the calculation
    number, zero-padded, when the input has more than one calculation, and
    ``_<variable>=<value>`` during a sweep, inserted before the extension."""
    insert = ""
    if total_calcs > 1:
        digits = int(math.log10(total_calcs)) + 1
        insert = "_" + str(calc_number).zfill(digits)
    if variation is not None:
        insert += "_" + variation.name + "=" + vary_value_text(variation, value)
    base, dot, ext = name.rpartition(".")
    return (base + insert + dot + ext) if dot else (name + insert)


def write_vtk(path: str, lines: List[OutputLine], lattice_shape: Tuple[int, ...], template=None,
              hex_lattice: bool = False) -> None:
    """Output::OutputVtkProfiles (Output.cpp:727-905), as it writes the file:
    a structured-points header ('DIMENSIONS' and the layer count run together
    in 1D; the HEX lattice as a structured grid with its sheared points),
    one 'SFBox_profile double' per profile written, and the data of the
    interior sites -- in 1D the selected profiles side by side for the layers
    1..n-1 (0-based), in 2D the template's first profile at (x, y-1) for
    y = 1..n_y, x = 1..n_x, in 3D at (x, y, z) with x fastest."""
    prof = [ln for ln in lines if ln.profile is not None and (template is None or in_template(template, ln))]
    acc = prof[0].acc if prof else 12
    n = [int(s) - 2 for s in lattice_shape]
    g = len(n)
    out = ["# vtk DataFile Version 3.0", "vtk output", "ASCII",
           "DATASET STRUCTURED_GRID" if hex_lattice else "DATASET STRUCTURED_POINTS"]
    if g == 1:
        out += [f"DIMENSIONS{n[0]}", "SPACING 1", "ORIGIN 0", f"POINT_DATA {n[0]}"]
    elif g == 2:
        out += [f"DIMENSIONS {n[0]} {n[1]} 1", "SPACING 1 1 1", "ORIGIN 0 0 0", f"POINT_DATA {n[0] * n[1]}"]
    else:
        out.append(f"DIMENSIONS {n[0]} {n[1]} {n[2]}")
        if hex_lattice:
            out.append(f"POINTS {n[0] * n[1] * n[2]} double")
            yc1, yc2 = 0.75 ** 0.5, 0.1875 ** 0.5
            for i in range(n[2]):
                for j in range(n[1]):
                    for k in range(n[0]):
                        out.append(" ".join(_real(v, acc) for v in (k + 0.5 * j + 0.5 * i, yc1 * j + yc2 * i,
                                                                         0.75 * i)))
        else:
            out += ["SPACING 1 1 1", "ORIGIN 0 0 0"]
        out.append(f"POINT_DATA {n[0] * n[1] * n[2]}")
    out.append("SCALARS " + "\n".join("SFBox_profile double" for _ in prof))
    out.append("LOOKUP_TABLE default ")
    if g == 1:
        for z in range(1, n[0]):
            out.append("".join(_real(ln.profile[z], ln.acc) for ln in prof))
    else:
        sel = None
        for ln in lines:
            if template is not None and in_template(template, ln):
                sel = ln
                break
        if sel is None or sel.profile is None:
            raise ValueError("vtk output of a 2D or 3D lattice needs a template naming a profile")
        p = np.asarray(sel.profile).reshape(lattice_shape)
        if g == 2:
            for y in range(1, n[1] + 1):
                for x in range(1, n[0] + 1):
                    out.append(_real(p[x, y - 1], sel.acc))
        else:
            for z in range(1, n[2] + 1):
                for y in range(1, n[1] + 1):
                    for x in range(1, n[0] + 1):
                        out.append(_real(p[x, y, z], sel.acc))
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def write_profiles(path: str, lines: List[OutputLine], lattice_shape: Tuple[int, ...], template=None,
                   write_bounds: bool = True, blank_lines: bool = True) -> None:
    """Output::OutputProfiles (Output.cpp:998-1196): one file per calculation
    (numbered names, as vtk files), a header row -- 'layer' (1D), 'layer x',
    'layer y' (2D) or also 'layer z' (3D), then 'c : n : k' of every profile
    line the template selects -- and one row per site with its 0-based
    coordinates and those profiles' values, every field followed by a tab.
    Boundary sites are written only with write_bounds (1D, 2D; never in 3D);
    in 2D each x row ends with a blank line and the file with one more
    (write_blank_lines)."""
    prof = [ln for ln in lines if ln.profile is not None and (template is None or in_template(template, ln))]
    g = len(lattice_shape)
    head = {1: ["layer"], 2: ["layer x", "layer y"], 3: ["layer x", "layer y", "layer z"]}[g]
    out = ["".join(h + "\t" for h in head) + "".join(f"{ln.cls} : {ln.name} : {ln.key}\t" for ln in prof)]
    vals = [np.asarray(ln.profile, dtype=float) for ln in prof]

    def row(coords, z):
        return "".join(f"{c}\t" for c in coords) + "".join(_real(v[z], ln.acc) + "\t" for v, ln in zip(vals, prof))

    n = [int(s) for s in lattice_shape]
    if g == 1:
        for z in range(n[0]):
            if write_bounds or 0 < z < n[0] - 1:
                out.append(row((z,), z))
    elif g == 2:
        z = 0
        for x in range(n[0]):
            for y in range(n[1]):
                if write_bounds or (0 < x < n[0] - 1 and 0 < y < n[1] - 1):
                    out.append(row((x, y), z))
                z += 1
            if blank_lines:
                out.append("")
        if blank_lines:
            out.append("")
    else:
        z = 0
        for x in range(n[0]):
            for y in range(n[1]):
                for w in range(n[2]):
                    if 0 < x < n[0] - 1 and 0 < y < n[1] - 1 and 0 < w < n[2] - 1:
                        out.append(row((x, y, w), z))
                    z += 1
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def output_requests(calc: Dict[Key, str]) -> List[Tuple[str, str, Dict[str, str]]]:
    """The ``output : <file> : ...`` statements: (file name, type, parameters)."""
    names: List[str] = []
    for (c, n, _p) in calc:
        if c == "output" and n not in names:
            names.append(n)
    out = []
    for n in names:
        params = {p: v for (c, nn, p), v in calc.items() if c == "output" and nn == n}
        t = params.get("type")
        if t not in ("ana", "kal", "vtk", "profiles"):
            raise ValueError(f"output : {n} : type : {t} is not written here (ana, kal, vtk and profiles are)")
        out.append((n, t, params))
    return out
