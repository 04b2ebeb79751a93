"""MPS reading and writing for the command line (``sovopt``'s
``src/sovopt/io/mps.py:104, 461`` is the interface this mirrors).

The reader accepts free-format (whitespace-separated) MPS, plain or gzip
compressed, with the standard sections: NAME, OBJSENSE, ROWS, COLUMNS
(integer MARKER blocks), RHS, RANGES, BOUNDS, ENDATA.  It follows the
format's common conventions:

* the first ``N`` row is the objective; further ``N`` rows are dropped;
* an RHS value on the objective row is the negated objective constant;
* RANGES widen an ``L`` row to ``[rhs - |R|, rhs]``, a ``G`` row to
  ``[rhs, rhs + |R|]`` and an ``E`` row to ``[rhs, rhs + R]`` for ``R > 0``
  or ``[rhs + R, rhs]`` for ``R < 0``;
* ``UP`` with a negative value on a column whose lower bound is still the
  default 0 makes the lower bound -inf; ``MI`` sets only the lower bound;
  ``BV`` is a binary column; ``LI``/``UI`` are integer bounds.

Infinite bounds are ``INF = 1e30`` as in the rest of the package.
"""

from __future__ import annotations

import gzip

import numpy as np

from .problem import INF, ObjSense, Problem, SparseMatrix

__all__ = ["read_mps", "write_mps", "MPSError"]


class MPSError(ValueError):
    """Malformed MPS input, with the line number."""

    def __init__(self, msg, lineno=-1):
        super().__init__(f"{msg} (line {lineno})" if lineno >= 0 else msg)
        self.lineno = lineno


def _open(path):
    if str(path).lower().endswith(".gz"):
        return gzip.open(path, "rt", encoding="utf-8", errors="replace")
    return open(path, "r", encoding="utf-8", errors="replace")


def _num(tok, lineno):
    try:
        return float(tok)
    except ValueError:
        raise MPSError(f"expected a number, got {tok!r}", lineno) from None


def read_mps(path) -> Problem:
    """Read an MPS file into a row-bounds ``Problem``."""
    name = "model"
    sense = ObjSense.MINIMISE
    row_kind: dict[str, str] = {}
    row_index: dict[str, int] = {}
    row_names: list[str] = []
    obj_row = None
    col_index: dict[str, int] = {}
    col_names: list[str] = []
    col_int: list[int] = []
    trip_r: list[int] = []
    trip_c: list[int] = []
    trip_v: list[float] = []
    cost: dict[int, float] = {}
    rhs: dict[int, float] = {}
    ranges: dict[int, float] = {}
    obj_const = 0.0
    bounds: list[tuple[str, int, float, int]] = []
    section = None
    integer = False
    with _open(path) as fh:
        for lineno, raw in enumerate(fh, 1):
            line = raw.rstrip("\n")
            if not line.strip() or line.startswith("*"):
                continue
            if not line[0].isspace():
                head = line.split()
                section = head[0].upper()
                if section == "NAME":
                    name = head[1] if len(head) > 1 else name
                elif section in ("OBJSENSE", "OBJSENS") and len(head) > 1:
                    sense = ObjSense.MAXIMISE if head[1].upper().startswith("MAX") \
                        else ObjSense.MINIMISE
                elif section == "ENDATA":
                    break
                elif section not in ("ROWS", "COLUMNS", "RHS", "RANGES", "BOUNDS",
                                     "OBJSENSE", "OBJSENS"):
                    raise MPSError(f"unsupported section {section!r}", lineno)
                continue
            tok = line.split()
            if section in ("OBJSENSE", "OBJSENS"):
                sense = ObjSense.MAXIMISE if tok[0].upper().startswith("MAX") \
                    else ObjSense.MINIMISE
            elif section == "ROWS":
                if len(tok) != 2:
                    raise MPSError("a ROWS line has a type and a name", lineno)
                kind, rn = tok[0].upper(), tok[1]
                if kind not in ("N", "E", "L", "G"):
                    raise MPSError(f"unknown row type {kind!r}", lineno)
                if kind == "N":
                    if obj_row is None:
                        obj_row = rn
                    row_kind[rn] = "N"
                    continue
                row_kind[rn] = kind
                row_index[rn] = len(row_names)
                row_names.append(rn)
            elif section == "COLUMNS":
                if len(tok) >= 3 and tok[1].upper() == "'MARKER'":
                    integer = tok[2].upper() == "'INTORG'"
                    continue
                if len(tok) not in (3, 5):
                    raise MPSError("a COLUMNS line has a column and one or two entries", lineno)
                cn = tok[0]
                j = col_index.get(cn)
                if j is None:
                    j = col_index[cn] = len(col_names)
                    col_names.append(cn)
                    col_int.append(1 if integer else 0)
                for rn, val in zip(tok[1::2], tok[2::2]):
                    v = _num(val, lineno)
                    if rn not in row_kind:
                        raise MPSError(f"unknown row {rn!r}", lineno)
                    if row_kind[rn] == "N":
                        if rn == obj_row:
                            cost[j] = cost.get(j, 0.0) + v
                        continue
                    trip_r.append(row_index[rn])
                    trip_c.append(j)
                    trip_v.append(v)
            elif section in ("RHS", "RANGES"):
                pairs = tok[1:] if len(tok) % 2 == 1 else tok
                for rn, val in zip(pairs[0::2], pairs[1::2]):
                    v = _num(val, lineno)
                    if rn not in row_kind:
                        raise MPSError(f"unknown row {rn!r}", lineno)
                    if row_kind[rn] == "N":
                        if section == "RHS" and rn == obj_row:
                            obj_const = -v
                        continue
                    (rhs if section == "RHS" else ranges)[row_index[rn]] = v
            elif section == "BOUNDS":
                # "<type> [<set name>] <column> [<value>]"
                kind = tok[0].upper()
                if kind in ("FR", "MI", "PL", "BV"):
                    if len(tok) < 2:
                        raise MPSError(f"bound {kind} needs a column", lineno)
                    cn, val = (tok[1] if len(tok) == 2 else tok[2]), 0.0
                else:
                    if len(tok) < 3:
                        raise MPSError(f"bound {kind} needs a column and a value", lineno)
                    cn, val = (tok[1], _num(tok[2], lineno)) if len(tok) == 3 \
                        else (tok[2], _num(tok[3], lineno))
                if cn not in col_index:
                    raise MPSError(f"unknown column {cn!r}", lineno)
                bounds.append((kind, col_index[cn], val, lineno))
    if obj_row is None and not col_names:
        raise MPSError("no ROWS/COLUMNS in the file")
    m, n = len(row_names), len(col_names)
    c = np.zeros(n)
    for j, v in cost.items():
        c[j] = v
    rl = np.full(m, -INF)
    ru = np.full(m, INF)
    for rn, i in row_index.items():
        b = rhs.get(i, 0.0)
        k = row_kind[rn]
        if k == "E":
            rl[i] = ru[i] = b
        elif k == "L":
            ru[i] = b
        else:
            rl[i] = b
        if i in ranges:
            r = ranges[i]
            if k == "L":
                rl[i] = b - abs(r)
            elif k == "G":
                ru[i] = b + abs(r)
            elif r > 0:
                ru[i] = b + r
            else:
                rl[i] = b + r
    lo = np.zeros(n)
    hi = np.full(n, INF)
    kind_arr = np.asarray(col_int, dtype=np.uint8)
    lo_set = np.zeros(n, dtype=bool)
    for kind, j, val, lineno in bounds:
        if kind == "UP":
            hi[j] = val
            if val < 0 and not lo_set[j] and lo[j] == 0.0:
                lo[j] = -INF
        elif kind == "LO":
            lo[j] = val
            lo_set[j] = True
        elif kind == "FX":
            lo[j] = hi[j] = val
            lo_set[j] = True
        elif kind == "FR":
            lo[j], hi[j] = -INF, INF
            lo_set[j] = True
        elif kind == "MI":
            lo[j] = -INF
            lo_set[j] = True
        elif kind == "PL":
            hi[j] = INF
        elif kind == "BV":
            lo[j], hi[j] = 0.0, 1.0
            kind_arr[j] = 1
            lo_set[j] = True
        elif kind == "LI":
            lo[j] = val
            kind_arr[j] = 1
            lo_set[j] = True
        elif kind == "UI":
            hi[j] = val
            kind_arr[j] = 1
            if val < 0 and not lo_set[j] and lo[j] == 0.0:
                lo[j] = -INF
        else:
            raise MPSError(f"unsupported bound type {kind!r}", lineno)
    A = SparseMatrix.from_triplets(np.asarray(trip_r, dtype=np.int64),
                                   np.asarray(trip_c, dtype=np.int64),
                                   np.asarray(trip_v, dtype=float), m, n)
    return Problem(A=A, c=c, row_lb=rl, row_ub=ru, col_lb=lo, col_ub=hi, kind=kind_arr,
                   obj_offset=obj_const, sense=sense, name=name,
                   col_names=col_names, row_names=row_names)


def _fmt(v):
    return repr(float(v))


def write_mps(prob: Problem, path):
    """Write ``prob`` as free-format MPS (ranged rows through RANGES)."""
    m, n = prob.m, prob.n
    rn = prob.row_names or [f"R{i}" for i in range(m)]
    cn = prob.col_names or [f"C{j}" for j in range(n)]
    rl = np.asarray(prob.row_lb, float)
    ru = np.asarray(prob.row_ub, float)
    kinds = []
    for i in range(m):
        lo_f, hi_f = rl[i] > -INF, ru[i] < INF
        if lo_f and hi_f and rl[i] == ru[i]:
            kinds.append("E")
        elif hi_f:
            kinds.append("L")
        elif lo_f:
            kinds.append("G")
        else:
            kinds.append("N")
    A = prob.A
    out = [f"NAME {prob.name}"]
    if int(prob.sense) == int(ObjSense.MAXIMISE):
        out += ["OBJSENSE", "    MAX"]
    out += ["ROWS", " N  OBJ"]
    free_rows = []
    for i in range(m):
        if kinds[i] == "N":       # a free row: keep it as an L row at +INF
            free_rows.append(i)
            out.append(f" L  {rn[i]}")
        else:
            out.append(f" {kinds[i]}  {rn[i]}")
    out.append("COLUMNS")
    integer = False
    kind = np.asarray(prob.kind if prob.kind is not None else np.zeros(n), dtype=np.uint8)
    for j in range(n):
        if bool(kind[j]) != integer:
            integer = bool(kind[j])
            out.append(f"    MARKER 'MARKER' {'INTORG' if integer else 'INTEND'}")
        if prob.c[j] != 0.0:
            out.append(f"    {cn[j]} OBJ {_fmt(prob.c[j])}")
        for p in range(int(A.cp[j]), int(A.cp[j + 1])):
            out.append(f"    {cn[j]} {rn[int(A.ci[p])]} {_fmt(A.cx[p])}")
        if A.cp[j] == A.cp[j + 1] and prob.c[j] == 0.0:
            out.append(f"    {cn[j]} OBJ 0.0")
    if integer:
        out.append("    MARKER 'MARKER' INTEND")
    out.append("RHS")
    if prob.obj_offset != 0.0:
        out.append(f"    RHS OBJ {_fmt(-prob.obj_offset)}")
    rng = []
    for i in range(m):
        k = kinds[i]
        if k == "N":
            out.append(f"    RHS {rn[i]} {_fmt(INF)}")
            continue
        b = ru[i] if k in ("E", "L") else rl[i]
        if b != 0.0:
            out.append(f"    RHS {rn[i]} {_fmt(b)}")
        if k == "L" and rl[i] > -INF:
            rng.append((rn[i], ru[i] - rl[i]))
        elif k == "G" and ru[i] < INF:
            rng.append((rn[i], ru[i] - rl[i]))
    if rng:
        out.append("RANGES")
        out += [f"    RNG {r} {_fmt(v)}" for r, v in rng]
    out.append("BOUNDS")
    lo = np.asarray(prob.col_lb, float)
    hi = np.asarray(prob.col_ub, float)
    for j in range(n):
        l_inf, u_inf = lo[j] <= -INF, hi[j] >= INF
        if l_inf and u_inf:
            out.append(f" FR BND {cn[j]}")
            continue
        if not l_inf and not u_inf and lo[j] == hi[j]:
            out.append(f" FX BND {cn[j]} {_fmt(lo[j])}")
            continue
        if l_inf:
            out.append(f" MI BND {cn[j]}")
        elif lo[j] != 0.0 or (not u_inf and hi[j] < 0.0):
            # an explicit LO keeps a negative UP from implying a -inf lower bound
            out.append(f" LO BND {cn[j]} {_fmt(lo[j])}")
        if not u_inf:
            out.append(f" UP BND {cn[j]} {_fmt(hi[j])}")
    out.append("ENDATA")
    with open(path, "w", encoding="utf-8") as fh:
        fh.write("\n".join(out) + "\n")
