"""Reader of the reference's run input (``input.canard``): Fortran namelist
groups, each read the way the reference reads them (an unformatted namelist
READ per group that searches the file for ``&name``; src/mo_canard_driver.f90:
91-103 and the read_input routines of mo_numerics, mo_physics, mo_gridgen,
mo_sponge and mo_domdcomp).

Supported syntax: ``&group ... /`` blocks; ``name = v1, v2, ...`` (values
separated by commas or blanks, ``r*v`` repeat counts); array elements and
sections ``name(i)``, ``name(:, 1)``, ``name(0, 1, :)``, ``name(lo:hi)``, which
fill the selected elements in Fortran (column-major) order; integers, reals
(``e`` or ``d`` exponents), logicals (``.true.``, ``.false.``, ``t``, ``f``) and
quoted strings; ``!`` comments. A group whose ``&`` is missing is not a group:
its lines are skipped, so its variables keep their defaults, as in the
reference (run/exp.toy writes ``nml_sponge`` without the ``&``).
"""
from __future__ import annotations

import itertools
import re
from typing import Dict, List, Tuple

import numpy as np

# (type, bounds per dimension) of every variable the path reads; "NB" is the
# last block index (nml_driver's mbk). Types: i integer, r real, l logical.
_SCALAR = ()
SCHEMA: Dict[str, Dict[str, Tuple[str, tuple]]] = {
    "nml_driver": {"nio": ("i", _SCALAR), "mbk": ("i", _SCALAR), "ndata": ("i", _SCALAR)},
    "nml_canard": {"nts": ("i", _SCALAR), "nrestart": ("i", _SCALAR), "cfl": ("r", _SCALAR),
                   "tmax": ("r", _SCALAR), "ltimer": ("l", _SCALAR)},
    "nml_domdcomp": {"nbpc": ("i", (("0", "NB"), ("1", "3"))), "lximb": ("i", (("0", "NB"),)),
                     "letmb": ("i", (("0", "NB"),)), "lzemb": ("i", (("0", "NB"),)),
                     "nbbc": ("i", (("0", "NB"), ("1", "3"), ("1", "2"))),
                     "mbcd": ("i", (("0", "NB"), ("1", "3"), ("1", "2")))},
    "nml_numerics": {"fltk": ("r", _SCALAR), "fltrbc": ("r", _SCALAR)},
    "nml_physics": {"reoo": ("r", _SCALAR), "tempoo": ("r", _SCALAR), "amach1": ("r", _SCALAR),
                    "amach2": ("r", _SCALAR), "amach3": ("r", _SCALAR), "timf": ("r", _SCALAR),
                    "nsmf": ("i", _SCALAR)},
    "nml_gridgen": {"gridtype": ("i", _SCALAR), "lxi0": ("i", _SCALAR), "lxi1": ("i", _SCALAR),
                    "lxi2": ("i", _SCALAR), "let0": ("i", _SCALAR), "lze0": ("i", _SCALAR),
                    "nthick": ("i", _SCALAR), "doml0": ("r", _SCALAR), "doml1": ("r", _SCALAR),
                    "domh": ("r", _SCALAR), "span": ("r", _SCALAR), "szth0": ("r", _SCALAR),
                    "szth1": ("r", _SCALAR), "smg": ("r", _SCALAR), "smgvr": ("r", _SCALAR),
                    "spx": ("r", _SCALAR)},
    "nml_sponge": {"szco": ("r", _SCALAR)},
    # Options of this implementation, in a group of its own that the reference's
    # READs never look for (they search their groups by name): nprecision 0
    # FP64, 1 FP32-mixed, 2 fast FP64; lsplit: run nbpc's sub-domains as the reference's
    # ranks; nsteps > 0: stop after that many steps as well; linviscid: the
    # reference built without VISCOUS.
    "nml_gpu": {"nprecision": ("i", _SCALAR), "lsplit": ("l", _SCALAR), "nsteps": ("i", _SCALAR),
                "linviscid": ("l", _SCALAR)},
}


class NamelistError(ValueError):
    pass


def _strip_comments(text: str) -> str:
    out = []
    for line in text.splitlines():
        q = None
        for k, ch in enumerate(line):
            if q:
                if ch == q:
                    q = None
            elif ch in "'\"":
                q = ch
            elif ch == "!":
                line = line[:k]
                break
        out.append(line)
    return "\n".join(out)


_TOKEN = re.compile(r"""\s*(?:
    (?P<end>/|&end\b)
  | (?P<group>&[A-Za-z_]\w*)
  | (?P<target>[A-Za-z_]\w*\s*(?:\([^)]*\))?)\s*=
  | (?P<str>'[^']*'|"[^"]*")
  | (?P<value>[^\s,/=]+)
  | (?P<comma>,)
)""", re.VERBOSE | re.IGNORECASE)


def _tokens(text: str) -> List[Tuple[str, str]]:
    toks = []
    pos = 0
    text = _strip_comments(text)
    while pos < len(text):
        m = _TOKEN.match(text, pos)
        if not m or m.end() == pos:
            if text[pos:].strip() == "":
                break
            raise NamelistError(f"cannot read input near: {text[pos:pos + 30]!r}")
        pos = m.end()
        kind = m.lastgroup
        toks.append((kind, m.group(kind)))
    return toks


def raw_groups(text: str) -> Dict[str, List[Tuple[str, str, List[str]]]]:
    """Per group (lower case): its assignments (name, index text, values)."""
    groups: Dict[str, List[Tuple[str, str, List[str]]]] = {}
    cur = None
    target = None
    for kind, tok in _tokens(text):
        if kind == "group":
            cur = groups.setdefault(tok[1:].lower(), [])
            target = None
        elif kind == "end":
            cur = None
            target = None
        elif cur is None:
            continue  # outside a group: the reference's READ skips it
        elif kind == "target":
            m = re.match(r"([A-Za-z_]\w*)\s*(?:\((.*)\))?", tok.strip())
            target = [m.group(1).lower(), (m.group(2) or "").strip(), []]
            cur.append(target)
        elif kind in ("value", "str"):
            if target is None:
                raise NamelistError(f"value {tok!r} without a variable")
            if kind == "value" and re.fullmatch(r"\d+\*.+", tok):
                r, v = tok.split("*", 1)
                target[2].extend([v] * int(r))
            else:
                target[2].append(tok)
    return {g: [tuple(a) for a in v] for g, v in groups.items()}


def _value(tok: str, typ: str):
    t = tok.strip().lower()
    if typ == "l":
        if t in (".true.", ".t.", "t", "true"):
            return True
        if t in (".false.", ".f.", "f", "false"):
            return False
        raise NamelistError(f"not a logical: {tok!r}")
    t = t.replace("d", "e")
    try:
        return int(t) if typ == "i" else float(t)
    except ValueError:
        raise NamelistError(f"not a number: {tok!r}") from None


def _elements(index: str, bounds: List[Tuple[int, int]]):
    """Multi-indices (Fortran numbering) selected by an index text, first
    dimension fastest."""
    if not index:
        parts = [":"] * len(bounds)
    else:
        parts = [p.strip() for p in index.split(",")]
    if len(parts) != len(bounds):
        raise NamelistError(f"index ({index}) has {len(parts)} subscripts for a rank-{len(bounds)} array")
    ranges = []
    for p, (lo, hi) in zip(parts, bounds):
        if ":" in p:
            a, b = (x.strip() for x in p.split(":", 1))
            ranges.append(range(int(a) if a else lo, (int(b) if b else hi) + 1))
        else:
            ranges.append([int(p)])
        for v in ranges[-1]:
            if not lo <= v <= hi:
                raise NamelistError(f"subscript {v} outside {lo}:{hi}")
    return [tuple(reversed(e)) for e in itertools.product(*reversed(ranges))]


def read(text: str) -> Dict[str, Dict[str, object]]:
    """The variables of every group in SCHEMA: scalars as Python values, arrays
    as (numpy array, lower bounds). Variables not in the input keep the
    default zero / false; a group absent from the input gives all defaults."""
    raw = raw_groups(text)
    mbk = 0
    for name, _, vals in raw.get("nml_driver", []):
        if name == "mbk" and vals:
            mbk = _value(vals[-1], "i")
    out: Dict[str, Dict[str, object]] = {}
    for group, vars_ in SCHEMA.items():
        res: Dict[str, object] = {}
        for name, (typ, bnds) in vars_.items():
            dtype = {"i": np.int64, "r": np.float64, "l": bool}[typ]
            if bnds:
                b = [(int(lo), mbk if hi == "NB" else int(hi)) for lo, hi in bnds]
                res[name] = (np.zeros([hi - lo + 1 for lo, hi in b], dtype=dtype), [lo for lo, _ in b])
            else:
                res[name] = dtype(0)
        for name, index, vals in raw.get(group, []):
            if name not in vars_:
                raise NamelistError(f"&{group}: unknown variable {name!r}")
            typ, bnds = vars_[name]
            if not bnds:
                if index or len(vals) != 1:
                    raise NamelistError(f"&{group}: {name} takes one value")
                res[name] = _value(vals[0], typ)
                continue
            arr, lows = res[name]
            b = [(lo, lo + n - 1) for lo, n in zip(lows, arr.shape)]
            for e, v in zip(_elements(index, b), vals):
                arr[tuple(i - lo for i, lo in zip(e, lows))] = _value(v, typ)
        out[group] = res
    return out


def read_file(path: str) -> Dict[str, Dict[str, object]]:
    with open(path) as f:
        return read(f.read())
