"""SFbox input files: ``class : name : parameter : value`` lines.

Restates the reader of SFbox's ``Input`` class (Input.cpp:20-102): one
statement per line, four fields separated by ':', ``//`` and ``#`` start a
comment, a line ``start`` closes a calculation, and every calculation starts
from the values of the previous one (later statements override earlier ones).

``build_system`` turns one calculation into a :class:`SystemSpec` restricted
to the SCF hot path (``lat``, ``mon``, ``mol``, ``sys`` and ``newton``
statements).  Unsupported features raise ``ValueError`` naming the statement.
"""
from __future__ import annotations

import re
from dataclasses import dataclass
from typing import Dict, List, Optional, Tuple

import numpy as np

from .desc import (BOUND_NAMES, BOUND_MIRROR1, BOUND_PERIODIC, GEOM_CYLINDRICAL, GEOM_FLAT, GEOM_SPHERICAL,
                   LATTICE_FCC, LATTICE_HEX, LATTICE_STANDARD, LATTICE_STENCILS, Lattice, Molecule, MOL_FREE, MOL_NEUTRALIZER,
                   MOL_RESTRICTED, MOL_SOLVENT, Segment,
                   SEG_FREE, SEG_FROZEN, SEG_PINNED, SystemSpec)

Key = Tuple[str, str, str]


def parse_input(text: str) -> List[Dict[Key, str]]:
    """Split an input text into calculations (Input.cpp:36-102)."""
    calcs: List[Dict[Key, str]] = []
    cur: Dict[Key, str] = {}
    dirty = False
    for lineno, raw in enumerate(text.splitlines(), 1):
        line = raw
        for mark in ("//", "#"):
            p = line.find(mark)
            if p >= 0:
                line = line[:p]
        line = line.strip()
        if not line:
            continue
        if line == "start":
            if dirty:
                calcs.append(dict(cur))
                dirty = False
            continue
        parts = [p.strip() for p in line.split(":")]
        if len(parts) > 4:
            # values such as ranges never contain ':'; more fields is an error
            raise ValueError(f"line {lineno}: line contains too many elements")
        if len(parts) < 4 or any(p == "" for p in parts):
            raise ValueError(f"line {lineno}: statement missing")
        cur[(parts[0], parts[1], parts[2])] = parts[3]
        dirty = True
    if dirty:
        calcs.append(dict(cur))
    return calcs


def _names(calc: Dict[Key, str], cls: str) -> List[str]:
    out: List[str] = []
    for (c, n, _p) in calc:
        if c == cls and n not in out:
            out.append(n)
    return out


def _get(calc, cls, name, param, default=None):
    return calc.get((cls, name, param), default)


def parse_composition(text: str) -> List[Tuple[str, int]]:
    """Linear compositions '(A)20(B)20' (SF_MolStructure); branches are not
    on this path."""
    blocks = re.findall(r"\(([^()]+)\)(\d+)", text.replace(" ", ""))
    if not blocks or "".join(f"({a}){b}" for a, b in blocks) != text.replace(" ", ""):
        raise ValueError(f"composition '{text}' is not a linear block sequence")
    return [(a, int(b)) for a, b in blocks]


def _expand_branch_repeats(t: str) -> str:
    """SF_ParserBranched::ExpandBrackets (SF_ParserBranched.cpp:94-122): the
    first '[' that sits inside round brackets expands its enclosing group,
    '((A)5[(B)1](C)5)2' -> '(A)5[(B)1](C)5(A)5[(B)1](C)5', until none is left."""
    while True:
        depth = 0
        for i, ch in enumerate(t):
            if ch == "(":
                depth += 1
            elif ch == ")":
                depth -= 1
            elif ch == "[" and depth > 0:
                break
        else:
            return t
        # the enclosing '(' to the left and its matching ')' to the right
        d, lo = -1, i
        while d < 0 and lo > 0:
            lo -= 1
            d += (t[lo] == "(") - (t[lo] == ")")
        d, hi = 1, i
        while d > 0 and hi < len(t) - 1:
            hi += 1
            d += (t[hi] == "(") - (t[hi] == ")")
        if d != 0 or t[lo] != "(":
            raise ValueError(f"composition '{t}': unbalanced brackets around a branch")
        m = re.match(r"\d*", t[hi + 1:])
        rep = int(m.group(0)) if m.group(0) else 1
        t = t[:lo] + t[lo + 1:hi] * rep + t[hi + 1 + len(m.group(0)):]


def parse_branched(text: str) -> Optional[Tuple[List[Tuple[str, int]], List[int]]]:
    """Branched compositions with square brackets (SF_ParserBranched,
    SF_ParserBranched.h:20-45): the linear fragments between brackets in
    order, ranked from 1 ('[' raises the next fragment's rank, ']' lowers it,
    a fragment after '][' takes the previous rank and the ranks before it
    that are not lower move up by one), and every fragment's first segment
    bonded to the last segment of the nearest preceding fragment of lower or
    equal rank (FillLinks, SF_ParserBranched.cpp:43-60).  Returns the blocks
    of all fragments in order and, per segment, the segment it is bonded to
    towards segment 0 (-1 for segment 0); None without square brackets."""
    t = text.replace(" ", "")
    if "[" not in t and "]" not in t:
        return None
    t = _expand_branch_repeats(t)
    if not t.startswith("["):
        t = "[" + t + "]"
    br = [(i, 1 if ch == "[" else -1) for i, ch in enumerate(t) if ch in "[]"]
    if sum(b for _, b in br) != 0:
        raise ValueError(f"composition '{text}': square brackets do not match")
    frags, ranks = [], [0]
    multi = False
    for (p0, typ), (p1, _t1) in zip(br, br[1:]):
        body = t[p0 + 1:p1]
        if body:
            if not multi:
                r = ranks[-1] + typ
                ranks.append(r)
            else:
                r = ranks[-1]
                k = len(ranks) - 1
                while k > 0 and ranks[k] >= r:
                    ranks[k] += 1
                    k -= 1
                ranks.append(r)
                multi = False
            frags.append(parse_composition(body))
        elif t[p0:p1 + 1] == "][":
            multi = True
        else:
            raise ValueError(f"composition '{text}': unnecessary square brackets")
    ranks = ranks[1:]
    if sum(n for _, n in frags[0]) == 1:
        raise ValueError(f"composition '{text}': the first linear fragment contains only one monomer")
    blocks, parent, last = [], [], []
    for b, fr in enumerate(frags):
        n = sum(k for _, k in fr)
        start = len(parent)
        if b == 0:
            parent.append(-1)
        else:
            i = b - 1
            while i > 0 and ranks[i] > ranks[b]:
                i -= 1
            if ranks[i] > ranks[b]:
                raise ValueError(f"composition '{text}': fragment {b + 1} has no fragment to branch from")
            parent.append(last[i])
        parent.extend(range(start, start + n - 1))
        last.append(start + n - 1)
        blocks.extend(fr)
    return blocks, parent


def parse_comb(text: str) -> Optional[Tuple[List[Tuple[str, int]], List[int]]]:
    """Combs '@dend(NA. Main1, Spacer, Side, Main2)' = Main1-(Spacer-[Side])NA-Main2
    (SF_MolStructure.cpp:167-181, :242-326; SF_Comb1stO::Matrix1,
    SF_Comb1stO.cpp:636-760) with linear fragments: the backbone Main1, NA
    spacers each carrying the side chain on its last segment, then Main2.
    Returns the blocks in that order and the bond parent of every segment;
    None for other compositions."""
    t = text.replace(" ", "")
    m = re.fullmatch(r"@dend\((\d+)\.(.*)\)", t)
    if not m:
        return None
    na = int(m.group(1))
    parts = m.group(2).split(",")
    if na < 1 or len(parts) != 4 or any(";" in q or "@" in q for q in parts) or \
            any("[" in parts[i] or "]" in parts[i] for i in (0, 1, 3)):
        raise ValueError(f"composition '{text}': combs of linear main, spacer and end fragments with a linear or "
                         "branched side chain only")
    main1, spacer, main2 = (parse_composition(parts[i]) for i in (0, 1, 3))
    # a branched side chain hangs from its first segment (SF_Comb1stO.cpp:675-681)
    side = parse_branched(parts[2]) or (parse_composition(parts[2]), None)
    blocks, parent = [], []

    def chain(fr, attach):
        start = len(parent)
        n = sum(k for _, k in fr)
        parent.append(attach)
        parent.extend(range(start, start + n - 1))
        blocks.extend(fr)
        return start + n - 1

    def hang(tree, attach):
        fr, par = tree
        if par is None:
            chain(fr, attach)
            return
        start = len(parent)
        parent.extend([attach] + [p + start for p in par[1:]])
        blocks.extend(fr)

    end = chain(main1, -1)
    for _ in range(na):
        end = chain(spacer, end)
        hang(side, end)
    chain(main2, end)
    return blocks, parent


def _drop_first(fr: List[Tuple[str, int]]) -> List[Tuple[str, int]]:
    """A linear fragment without its first segment."""
    if not fr:
        return []
    (a, n), rest = fr[0], list(fr[1:])
    return ([(a, n - 1)] if n > 1 else []) + rest


def parse_asym_dendrimer(text: str) -> Optional[Tuple[List[Tuple[str, int]], List[int]]]:
    """Asymmetric dendrimers '@dend(G; S11, S12, S21, S22, ..., SG1, SG2)'
    (SF_MolStructure.cpp:141-160, :328-347: one ';' after G and 2G - 1
    commas; the two fragments of a generation start with the same segment):
    generation 1's shared first segment is the core with the two arms S11
    and S12 (the rest of each fragment); every arm end of generation i - 1
    carries a branch point of generation i, the shared first segment of
    S_i1 and S_i2, with those two arms (SF_AsymDend1stO::ComputePhi,
    SF_AsymDend1stO.cpp:206-300).  Returns the blocks in order of
    construction and the bond parent of every segment; None for other
    compositions."""
    t = text.replace(" ", "")
    m = re.fullmatch(r"@dend\((\d+);(.*)\)", t)
    if not m:
        return None
    G = int(m.group(1))
    parts = m.group(2).split(",")
    if G < 1 or len(parts) != 2 * G:
        raise ValueError(f"composition '{text}': @dend(G; ...) needs two fragments per generation")
    gens = [(parse_composition(parts[2 * i]), parse_composition(parts[2 * i + 1])) for i in range(G)]
    for f1, f2 in gens:
        if f1[0][0] != f2[0][0]:
            raise ValueError(f"composition '{text}': the two fragments of a generation must start with the same "
                             "segment (SF_MolStructure.cpp:344-345)")
    blocks, parent = [], []

    def chain(fr, attach):
        """append a linear fragment bonded to `attach`; its last segment (or
        `attach` for an empty fragment)"""
        n = sum(k for _, k in fr)
        if n == 0:
            return attach
        start = len(parent)
        parent.append(attach)
        parent.extend(range(start, start + n - 1))
        blocks.extend(fr)
        return start + n - 1

    def generation(f1, f2, attach):
        first = len(parent)
        e1 = chain(f1, attach)            # the branch point is f1's first segment
        e2 = chain(_drop_first(f2), first)
        return [e1, e2]

    ends = generation(gens[0][0], gens[0][1], -1)
    for f1, f2 in gens[1:]:
        ends = [e for a in ends for e in generation(f1, f2, a)]
    return blocks, parent


def parse_dendrimer(text: str) -> Optional[List[Tuple[List[Tuple[str, int]], int]]]:
    """Symmetric dendrimer compositions '@dend(G, T1, f1, ..., TG, fG)'
    (SF_MolStructure.cpp:116-140, :348-359): per generation its linear block
    sequence Ti and its functionality fi.  None for other compositions."""
    t = text.replace(" ", "")
    if not t.startswith("@"):
        return None
    m = re.fullmatch(r"@dend\((.*)\)", t)
    if not m:
        raise ValueError(f"composition '{text}': only symmetric dendrimers @dend(G, T1, f1, ...) are on this path")
    args = m.group(1).split(",")
    if not args[0].isdigit():
        raise ValueError(f"composition '{text}': asymmetric dendrimers are not on this path")
    G = int(args[0])
    if len(args) - 1 != 2 * G or G < 1:
        raise ValueError(f"composition '{text}': @dend(G, ...) needs G generations of (block, functionality)")
    gens = []
    for i in range(G):
        f = args[2 + 2 * i]
        if not f.isdigit() or int(f) < 1:
            raise ValueError(f"composition '{text}': functionality '{f}' is not a positive integer")
        gens.append((parse_composition(args[1 + 2 * i]), int(f)))
    return gens


# newton : method choices on this path: SFbox's Newton with its BFGS-updated
# pseudo-Hessian (the default, SF_Solve.cpp:1867-1869) or a finite-difference
# Hessian, and Pure_DIIS; LBFGS, CG, SD, TN, BRR and experimental are refused
NEWTON_METHODS = ("pseudohessian", "hessian", "Pure_DIIS")


@dataclass
class SolverSettings:
    method: str = "pseudohessian"
    tolerance: float = 1e-7
    iterationlimit: int = 5000
    m: int = 5
    deltamax: float = 0.1
    initial_guess_file: Optional[str] = None


def _range_mask(lat: Lattice, text: str) -> np.ndarray:
    """Lattice ranges (Lat1DFlat.cpp:300-388, Lat2DFlat.cpp:419-609,
    Lat3D.cpp:596-862): 'low;high' boxes of layer coordinates (0 is the lower
    boundary layer; 'lowerbound', 'upperbound', 'lastlayer' allowed in 1D) or
    point lists '=(x,y,z)(x,y,z)...'."""
    shape = lat.shape
    mask = np.zeros(shape, dtype=np.float64)
    t = text.replace(" ", "")
    if t.startswith("="):
        pts = re.findall(r"\(([^()]*)\)", t)
        for p in pts:
            c = tuple(int(v) for v in p.split(","))
            if len(c) != len(shape):
                raise ValueError(f"point '{p}' does not match {len(shape)} gradients")
            mask[c] = 1.0
        return mask.reshape(-1)
    parts = t.split(";")
    if len(parts) == 1:
        parts = parts * 2
    if len(parts) != 2:
        raise ValueError(f"range '{text}'")

    def coord(s: str):
        if len(shape) == 1:
            M = shape[0]
            if s == "lowerbound":
                return (0,)
            if s == "upperbound":
                return (M - 1,)
            if s == "lastlayer":
                return (M - 2,)
        return tuple(int(v) for v in s.split(","))

    lo, hi = coord(parts[0]), coord(parts[1])
    if len(lo) != len(shape) or len(hi) != len(shape):
        raise ValueError(f"range '{text}' does not match {len(shape)} gradients")
    sl = tuple(slice(min(a, b), max(a, b) + 1) for a, b in zip(lo, hi))
    mask[sl] = 1.0
    return mask.reshape(-1)


def _refuse_unbuilt(calc: Dict[Key, str]) -> None:
    """Statements that change the physics of a calculation but are not built
    here: refused by name instead of being ignored."""
    for (c, n, p), v in calc.items():
        lv = v.strip().lower()
        if c == "state" and p == "valence" and float(v) != 0.0:
            raise ValueError(f"{c} : {n} : valence : {v} -- multistate charges are not built")
        if c == "mon" and p.startswith("state"):
            raise ValueError(f"mon : {n} : {p} -- multistate segments are not built")
        if c in ("reaction", "state"):
            raise ValueError(f"{c} : {n} : {p} -- reactions and states are not built")
        if c == "lat" and p == "n_layers_extended":
            raise ValueError(f"lat : {n} : n_layers_extended is not built")


def build_system(calc: Dict[Key, str]) -> Tuple[SystemSpec, SolverSettings]:
    _refuse_unbuilt(calc)
    lats = _names(calc, "lat")
    if len(lats) != 1:
        raise ValueError("exactly one 'lat' is supported")
    ln = lats[0]
    g = int(_get(calc, "lat", ln, "gradients", "1"))
    geom = _get(calc, "lat", ln, "geometry", "flat")
    if geom not in ("flat", "cylindrical", "spherical"):
        raise ValueError(f"lat : {ln} : geometry : {geom} is not on this path")
    order = 1
    for sysname in _names(calc, "sys"):
        if _get(calc, "sys", sysname, "matrix_approach", "first_order") == "second_order":
            order = 2
    ltype = _get(calc, "lat", ln, "latticetype", "standard")
    ltypes = {"standard": LATTICE_STANDARD, "stencils": LATTICE_STENCILS, "FCC": LATTICE_FCC, "HEX": LATTICE_HEX}
    if ltype not in ltypes or (ltype != "standard" and g != 3):
        raise ValueError(f"lat : {ln} : latticetype : {ltype} is not on this path")
    # 3D contact weights of the stencils type (Lat3D.cpp:221-259): lambda0..3
    # default to 1/27 and cannot be combined with lambda
    lam3 = (0.0, 0.0, 0.0, 0.0)
    lam_keys = [k for k in ("lambda0", "lambda1", "lambda2", "lambda3") if ("lat", ln, k) in calc]
    if lam_keys:
        if ("lat", ln, "lambda") in calc:
            raise ValueError(f"lat : {ln} : lambda cannot be combined with {lam_keys[0]}")
        if len(lam_keys) != 4:
            raise ValueError(f"lat : {ln} : lambda0, lambda1, lambda2 and lambda3 go together")
    if ltype == "stencils":
        lam3 = tuple(float(_get(calc, "lat", ln, k, repr(1.0 / 27.0))) for k in ("lambda0", "lambda1", "lambda2",
                                                                             "lambda3"))
    if g == 1:
        n = [int(_get(calc, "lat", ln, "n_layers"))]
        lo = [BOUND_NAMES[_get(calc, "lat", ln, "lowerbound", "mirror1")]]
        hi = [BOUND_NAMES[_get(calc, "lat", ln, "upperbound", "mirror1")]]
        if lo[0] == BOUND_PERIODIC or hi[0] == BOUND_PERIODIC:
            lo = hi = [BOUND_PERIODIC]
    else:
        axes = "xyz"[:g]
        n = [int(_get(calc, "lat", ln, f"n_layers_{a}")) for a in axes]
        default = "periodic" if g == 3 else "mirror1"
        lo, hi = [], []
        for a in axes:
            l = BOUND_NAMES[_get(calc, "lat", ln, f"lowerbound_{a}", default)]
            h = BOUND_NAMES[_get(calc, "lat", ln, f"upperbound_{a}", default)]
            if BOUND_PERIODIC in (l, h):
                l = h = BOUND_PERIODIC
            lo.append(l)
            hi.append(h)
    lam = float(_get(calc, "lat", ln, "lambda", repr(1.0 / 6.0)))
    ladj = float(_get(calc, "lat", ln, "layer_adjustment", "1"))
    if g == 1 and geom != "flat":
        # one-gradient curved lattices read offset_first_layer and may give the
        # first layer's size instead of layer_adjustment
        # (Lat1DCylinder.cpp:43-52, Lat1DSphere.cpp:6-12)
        off = float(_get(calc, "lat", ln, "offset_first_layer", "0"))
        nsites = _get(calc, "lat", ln, "n_sites_first_layer", None)
        if nsites is not None:
            v = float(nsites)
            ladj = np.sqrt(v / np.pi) if geom == "cylindrical" else (3 * v / (4 * np.pi)) ** (1.0 / 3.0)
    else:
        off = float(_get(calc, "lat", ln, "offset_first_layer_x", "0"))
    geometry = {"flat": GEOM_FLAT, "cylindrical": GEOM_CYLINDRICAL, "spherical": GEOM_SPHERICAL}[geom]
    lat = Lattice(gradients=g, n_layers=n + [0] * (3 - g), bound_lo=lo + [0] * (3 - g),
                  bound_hi=hi + [0] * (3 - g), geometry=geometry,
                  order=order, lam=lam,
                  lambda_chi=float(_get(calc, "lat", ln, "lambda_chi", "-1")),
                  layer_adjustment=ladj,
                  dimensions=float(_get(calc, "lat", ln, "dimensions", "3")),
                  offset_first_layer=off, lattice_type=ltypes[ltype], lambda_3d=lam3)
    # lat : stiff_range (Lat3D.cpp:265-268): second-order copolymers stiffen there
    sr = _get(calc, "lat", ln, "stiff_range", None)
    if sr is not None:
        if g != 3:
            raise ValueError(f"lat : {ln} : stiff_range is a 3D lattice parameter")
        lat.stiff_range = _range_mask(lat, sr)
    # segments
    seg_names = _names(calc, "mon")
    segs: List[Segment] = []
    for sn in seg_names:
        fr = _get(calc, "mon", sn, "freedom", "free")
        if fr == "free":
            segs.append(Segment(sn, SEG_FREE))
        elif fr == "frozen":
            segs.append(Segment(sn, SEG_FROZEN, _range_mask(lat, _get(calc, "mon", sn, "frozen_range"))))
        elif fr == "pinned":
            segs.append(Segment(sn, SEG_PINNED, _range_mask(lat, _get(calc, "mon", sn, "pinned_range"))))
        else:
            raise ValueError(f"mon : {sn} : freedom : {fr} is not on this path")
        # charges (SF_Segment.cpp:170-217): valence, relative dielectric constant
        segs[-1].valence = float(_get(calc, "mon", sn, "valence", "0"))
        segs[-1].epsilon = float(_get(calc, "mon", sn, "epsilon", "80"))
    ns = len(segs)
    charged = any(sg.valence != 0 for sg in segs)
    bl = _get(calc, "lat", ln, "bondlength", None)
    if charged and bl is None:   # SF_Solve.cpp:169-170
        raise ValueError(f"lat : {ln} : bondlength must be set in a system with charges")
    lat.bondlength = float(bl) if bl is not None else 3e-10
    chi = np.zeros((ns, ns))
    pf = np.full((ns, ns), 0.2)
    for i, a in enumerate(seg_names):
        for j, b in enumerate(seg_names):
            v = _get(calc, "mon", a, f"chi - {b}")
            if v is not None:
                chi[i, j] = chi[j, i] = float(v)
            v = _get(calc, "mon", a, f"Pf - {b}")
            if v is not None:
                pf[i, j] = pf[j, i] = float(v)
    mols: List[Molecule] = []
    for mn in _names(calc, "mol"):
        ctext = _get(calc, "mol", mn, "composition")
        gens, parent = None, None
        tree = parse_comb(ctext) or parse_asym_dendrimer(ctext) or parse_branched(ctext)
        if tree is not None:
            comp, parent = tree
        else:
            dend = parse_dendrimer(ctext)
            if dend is not None:
                comp = [b for blocks_i, _f in dend for b in blocks_i]
                gens = [(len(blocks_i), f) for blocks_i, f in dend]
            else:
                comp = parse_composition(ctext)
        blocks = [(seg_names.index(a), n_) for a, n_ in comp]
        length = Molecule(mn, blocks, generations=gens).N
        rv = _get(calc, "mol", mn, "ring", "false").strip().lower()
        if rv not in ("true", "false"):
            raise ValueError(f"mol : {mn} : ring : {rv} is not a boolean")
        ring = rv == "true"
        if ring and (parent is not None or gens or len({b[0] for b in blocks}) != 1):
            raise ValueError(f"mol : {mn} : only homopolymer rings are implemented (SF_MolList1stO.cpp:29-30)")
        if ring and length % 2:
            raise ValueError(f"mol : {mn} : rings have an even length (SF_HomoRing1stO.cpp:120)")
        force = float(_get(calc, "mol", mn, "force", "0"))
        if not -1000.0 <= force <= 1000.0:   # SF_Molecule.cpp:42
            raise ValueError(f"mol : {mn} : force must lie in [-1000, 1000]")
        fr = _get(calc, "mol", mn, "freedom", "free")
        if fr == "free":
            mols.append(Molecule(mn, blocks, MOL_FREE, phibulk=float(_get(calc, "mol", mn, "phibulk")),
                                 generations=gens, force=force, bond_parent=parent, ring=ring))
        elif fr == "restricted":
            th = _get(calc, "mol", mn, "theta")
            if th is None:
                nn = _get(calc, "mol", mn, "n")
                if nn is None:
                    raise ValueError(f"mol : {mn} needs theta or n")
                th = float(nn) * length
            mols.append(Molecule(mn, blocks, MOL_RESTRICTED, theta=float(th), generations=gens, force=force,
                                 bond_parent=parent, ring=ring))
        elif fr == "neutralizer":
            # SF_Molecule.cpp:110-126: its bulk fraction neutralises the bulk
            mols.append(Molecule(mn, blocks, MOL_NEUTRALIZER, generations=gens, bond_parent=parent, ring=ring))
        elif fr == "solvent":
            if gens or parent is not None or ring:
                raise ValueError(f"mol : {mn} : a dendrimer, branched molecule or ring cannot be the solvent here")
            mols.append(Molecule(mn, blocks, MOL_SOLVENT))
        else:
            raise ValueError(f"mol : {mn} : freedom : {fr} is not on this path")
    # sys : overflow_protection (SF_System.cpp:67): log-space chain statistics
    overflow = False
    for sysname in _names(calc, "sys"):
        v = _get(calc, "sys", sysname, "overflow_protection", "false").lower()
        if v not in ("true", "false"):
            raise ValueError(f"sys : {sysname} : overflow_protection : {v} is not a boolean")
        overflow |= v == "true"
    if overflow and (order != 1 or g == 3):
        raise ValueError("overflow_protection needs a first-order 1D or 2D lattice (SF_System.cpp:395, :478-481)")
    temperature = 298.15
    for sysname in _names(calc, "sys"):
        temperature = float(_get(calc, "sys", sysname, "temperature", temperature))
    spec = SystemSpec(lat, segs, chi, mols, pf=pf if order == 2 else None, overflow_protection=overflow,
                      temperature=temperature)
    st = SolverSettings()
    for nn in _names(calc, "newton"):
        st.method = _get(calc, "newton", nn, "method", st.method)
        st.tolerance = float(_get(calc, "newton", nn, "tolerance", st.tolerance))
        st.iterationlimit = int(_get(calc, "newton", nn, "iterationlimit", st.iterationlimit))
        st.m = int(_get(calc, "newton", nn, "m", st.m))
        st.deltamax = float(_get(calc, "newton", nn, "deltamax", st.deltamax))
        st.initial_guess_file = _get(calc, "newton", nn, "initial_guess_input_file")
        # deltamax's default is SFbox's 0.5 for every method (SF_Solve.cpp:1885);
        # Pure_DIIS uses it as its step eta
        if ("newton", nn, "deltamax") not in calc and st.method != "Pure_DIIS":
            st.deltamax = 0.5
    if st.method not in NEWTON_METHODS:
        raise ValueError(f"newton : method : {st.method} is not built (methods: {', '.join(NEWTON_METHODS)})")
    return spec, st
