"""The MILP model, the free-MPS reader and the feasibility checks.

Host-side mirror of the reference's model layer, src/milp.jl:1-145:

* ``MILP`` (src/milp.jl:15-26): ``min c'x + c0`` s.t. ``A x <= b`` on rows with
  ``row_sense == "le"``, ``A x = b`` on rows with ``"eq"``, ``l <= x <= u`` and
  integrality on ``int_idx``.  Ranged rows are split into two ``le`` rows and
  ``>=`` rows are negated; infinite bounds are stored as +-inf.
* ``read_mps`` (src/milp.jl:42-94): free-format MPS (optionally ``.gz``).
* ``max_violation`` / ``is_feasible`` / ``write_solution`` (src/milp.jl:102-145).

``A`` is a ``scipy.sparse.csr_matrix`` with sorted column indices (0-based);
``int_idx`` is a 0-based ``numpy`` index array.
"""
from __future__ import annotations

import gzip
import os
import re
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

MPS_INFINITY = 1.0e20  # src/milp.jl:36


def _is_infinite(v: float) -> bool:
    return (not np.isfinite(v)) or abs(v) >= MPS_INFINITY


@dataclass
class MILP:
    """``min c'x + c0`` s.t. ``A x (<=, =) b``, ``l <= x <= u``, ``x_j`` integer on ``int_idx``."""

    c: np.ndarray
    c0: float
    A: sp.csr_matrix
    b: np.ndarray
    row_sense: list  # "le" or "eq" per row
    l: np.ndarray
    u: np.ndarray
    int_idx: np.ndarray
    var_names: list = field(default_factory=list)
    name: str = ""

    def __post_init__(self):
        self.c = np.asarray(self.c, dtype=np.float64)
        self.b = np.asarray(self.b, dtype=np.float64)
        self.l = np.asarray(self.l, dtype=np.float64)
        self.u = np.asarray(self.u, dtype=np.float64)
        self.int_idx = np.asarray(self.int_idx, dtype=np.int64)
        A = self.A
        if not (sp.isspmatrix_csr(A) and A.dtype == np.float64 and A.has_canonical_format):
            A = sp.csr_matrix(A, dtype=np.float64)
            A.sum_duplicates()
            A.sort_indices()
        self.A = A
        self.row_sense = [str(s) for s in self.row_sense]
        if not self.var_names:
            self.var_names = [f"x{j + 1}" for j in range(len(self.c))]

    @property
    def is_eq(self) -> np.ndarray:
        return np.array([s == "eq" for s in self.row_sense], dtype=bool)

    @property
    def is_int(self) -> np.ndarray:
        mask = np.zeros(len(self.c), dtype=bool)
        mask[self.int_idx] = True
        return mask


def num_variables(milp: MILP) -> int:
    return len(milp.c)


def num_constraints(milp: MILP) -> int:
    return len(milp.b)


def num_continuous(milp: MILP) -> int:
    return len(milp.c) - len(milp.int_idx)


# ---------------------------------------------------------------------------
# free MPS reader


def _open_text(path: str):
    if path.endswith(".gz"):
        return gzip.open(path, "rt", encoding="latin-1")
    return open(path, "r", encoding="latin-1")


def read_mps(path: str) -> MILP:
    """Read a free-format MPS file into the canonical ``MILP`` form.

    Follows src/milp.jl:42-94: a maximisation objective is negated; binaries get
    their bounds clipped to [0, 1]; equal finite row bounds give an ``eq`` row;
    otherwise a finite upper bound gives ``A_i x <= hi`` and a finite lower bound
    gives ``-A_i x <= -lo`` (in that order).  Row, bound and range conventions
    are those of standard free MPS (the QPSReader 0.2 semantics the reference
    relies on): default bounds [0, inf), integer columns from MARKER
    INTORG/INTEND blocks, the objective constant is minus the objective row's RHS.
    """
    rows: list[tuple[str, str]] = []  # (name, type) in file order, excluding the objective
    row_index: dict[str, int] = {}
    obj_row = None
    cols: list[str] = []
    col_index: dict[str, int] = {}
    col_int: list[bool] = []
    trip_r: list[int] = []
    trip_c: list[int] = []
    trip_v: list[float] = []
    c_vals: dict[int, float] = {}
    rhs: dict[int, float] = {}
    ranges: dict[int, float] = {}
    lvar: dict[int, float] = {}
    uvar: dict[int, float] = {}
    binary: set[int] = set()
    explicit_int: set[int] = set()
    c0 = 0.0
    objsense = "min"
    name = None
    section = None
    in_int = False

    def col_id(cname: str) -> int:
        j = col_index.get(cname)
        if j is None:
            j = len(cols)
            col_index[cname] = j
            cols.append(cname)
            col_int.append(in_int)
        return j

    with _open_text(path) as fh:
        for raw in fh:
            line = raw.rstrip("\n\r")
            if not line.strip() or line.lstrip().startswith("*"):
                continue
            if not line[0].isspace():
                tok = line.split()
                key = tok[0].upper()
                section = key
                if key == "NAME":
                    name = tok[1] if len(tok) > 1 else None
                elif key == "OBJSENSE" and len(tok) > 1:
                    objsense = "max" if tok[1].upper().startswith("MAX") else "min"
                elif key == "ENDATA":
                    break
                continue
            tok = line.split()
            if section == "OBJSENSE":
                objsense = "max" if tok[0].upper().startswith("MAX") else "min"
            elif section == "ROWS":
                rtype, rname = tok[0].upper(), tok[1]
                if rtype == "N":
                    if obj_row is None:
                        obj_row = rname
                    continue  # further free rows carry no constraint
                row_index[rname] = len(rows)
                rows.append((rname, rtype))
            elif section == "COLUMNS":
                if len(tok) >= 3 and tok[1].strip("'\"").upper() == "MARKER":
                    marker = tok[2].strip("'\"").upper()
                    if marker == "INTORG":
                        in_int = True
                    elif marker == "INTEND":
                        in_int = False
                    continue
                j = col_id(tok[0])
                for k in range(1, len(tok) - 1, 2):
                    rname, val = tok[k], float(tok[k + 1])
                    if rname == obj_row:
                        c_vals[j] = c_vals.get(j, 0.0) + val
                    elif rname in row_index:
                        trip_r.append(row_index[rname])
                        trip_c.append(j)
                        trip_v.append(val)
            elif section in ("RHS", "RANGES"):
                pairs = tok[1:] if len(tok) % 2 == 1 else tok
                for k in range(0, len(pairs) - 1, 2):
                    rname, val = pairs[k], float(pairs[k + 1])
                    if section == "RHS":
                        if rname == obj_row:
                            c0 = -val
                        elif rname in row_index:
                            rhs[row_index[rname]] = val
                    elif rname in row_index:
                        ranges[row_index[rname]] = val
            elif section == "BOUNDS":
                btype = tok[0].upper()
                needs_value = btype in ("UP", "LO", "FX", "LI", "UI", "SC")
                if needs_value:
                    cname, val = (tok[2], float(tok[3])) if len(tok) >= 4 else (tok[1], float(tok[2]))
                else:
                    cname = tok[2] if len(tok) >= 3 else tok[1]
                    val = 0.0
                if cname not in col_index:
                    col_id(cname)
                j = col_index[cname]
                if btype == "UP":
                    uvar[j] = val
                    if val < 0 and lvar.get(j, 0.0) == 0.0 and j not in lvar:
                        lvar[j] = -np.inf
                elif btype == "LO":
                    lvar[j] = val
                elif btype == "FX":
                    lvar[j] = val
                    uvar[j] = val
                elif btype == "FR":
                    lvar[j] = -np.inf
                    uvar[j] = np.inf
                elif btype == "MI":
                    lvar[j] = -np.inf
                elif btype == "PL":
                    uvar[j] = np.inf
                elif btype == "BV":
                    binary.add(j)
                    lvar[j] = 0.0
                    uvar[j] = 1.0
                elif btype == "LI":
                    explicit_int.add(j)
                    lvar[j] = val
                elif btype == "UI":
                    explicit_int.add(j)
                    uvar[j] = val
                elif btype == "SC":
                    uvar[j] = val

    n = len(cols)
    sign = -1.0 if objsense == "max" else 1.0
    c = np.zeros(n)
    for j, v in c_vals.items():
        c[j] = v
    c = sign * c
    c0 = sign * c0
    l = np.zeros(n)
    u = np.full(n, np.inf)
    for j, v in lvar.items():
        l[j] = v
    for j, v in uvar.items():
        u[j] = v
    l = np.array([(-np.inf if v < 0 else np.inf) if _is_infinite(v) else v for v in l])
    u = np.array([(-np.inf if v < 0 else np.inf) if _is_infinite(v) else v for v in u])
    int_idx = []
    for j in range(n):
        if j in binary:
            int_idx.append(j)
            l[j] = max(l[j], 0.0)
            u[j] = min(u[j], 1.0)
        elif col_int[j] or j in explicit_int:
            int_idx.append(j)

    # Row bounds per original row, then the canonical rows (src/milp.jl:66-83).
    canonical: list[list[tuple[int, float]]] = [[] for _ in rows]
    b: list[float] = []
    sense: list[str] = []
    for i, (_, rtype) in enumerate(rows):
        r = rhs.get(i, 0.0)
        if rtype == "E":
            lo, hi = r, r
            if i in ranges:
                R = ranges[i]
                lo, hi = (r, r + abs(R)) if R > 0 else (r - abs(R), r)
        elif rtype == "L":
            lo, hi = -np.inf, r
            if i in ranges:
                lo = r - abs(ranges[i])
        elif rtype == "G":
            lo, hi = r, np.inf
            if i in ranges:
                hi = r + abs(ranges[i])
        else:
            lo, hi = -np.inf, np.inf
        if not _is_infinite(lo) and not _is_infinite(hi) and lo == hi:
            b.append(hi)
            sense.append("eq")
            canonical[i].append((len(b) - 1, 1.0))
            continue
        if not _is_infinite(hi):
            b.append(hi)
            sense.append("le")
            canonical[i].append((len(b) - 1, 1.0))
        if not _is_infinite(lo):
            b.append(-lo)
            sense.append("le")
            canonical[i].append((len(b) - 1, -1.0))

    I, J, V = [], [], []
    for r, cc, v in zip(trip_r, trip_c, trip_v):
        for row, s in canonical[r]:
            I.append(row)
            J.append(cc)
            V.append(s * v)
    A = sp.csr_matrix((np.array(V, dtype=np.float64), (np.array(I, dtype=np.int64),
                       np.array(J, dtype=np.int64))), shape=(len(b), n))
    if name is None:
        name = re.sub(r"\.mps(\.gz)?$", "", os.path.basename(path))
    return MILP(c, c0, A, np.array(b), sense, l, u, np.array(int_idx, dtype=np.int64), cols, name)


def read_mps_native(path: str) -> MILP:
    """``read_mps`` through the library's C++ reader (zlib for .gz; no GPU needed):
    the same canonical model, built without the interpreter's per-line cost."""
    import ctypes as C  # noqa: PLC0415

    from . import _lib as L  # noqa: PLC0415
    h = C.c_void_p()
    L.check(L.lib().pdfp_mps_read(os.fsencode(path), C.byref(h)))
    try:
        m, n, n_int = C.c_int32(), C.c_int32(), C.c_int32()
        nnz = C.c_int64()
        L.check(L.lib().pdfp_mps_dims(h, C.byref(m), C.byref(n), C.byref(nnz), C.byref(n_int)))
        M, N, Z, NI = m.value, n.value, nnz.value, n_int.value
        c, l, u = np.zeros(max(N, 1)), np.zeros(max(N, 1)), np.zeros(max(N, 1))
        b, is_eq = np.zeros(max(M, 1)), np.zeros(max(M, 1), dtype=np.uint8)
        rp = np.zeros(M + 1, dtype=np.int32)
        ci, v = np.zeros(max(Z, 1), dtype=np.int32), np.zeros(max(Z, 1))
        ii = np.zeros(max(NI, 1), dtype=np.int32)
        c0 = C.c_double()
        L.check(L.lib().pdfp_mps_get(h, L.dptr(c), C.byref(c0), L.iptr(rp), L.iptr(ci), L.dptr(v),
                                     L.dptr(b), L.uptr(is_eq), L.dptr(l), L.dptr(u), L.iptr(ii)))
    finally:
        L.lib().pdfp_mps_destroy(h)
    A = sp.csr_matrix((v[:Z], ci[:Z], rp), shape=(M, N))
    name = re.sub(r"\.mps(\.gz)?$", "", os.path.basename(path))
    return MILP(c[:N], c0.value, A, b[:M], ["eq" if e else "le" for e in is_eq[:M]], l[:N], u[:N],
                ii[:NI].astype(np.int64), [], name)


# ---------------------------------------------------------------------------
# checks


def max_violation(milp: MILP, x: np.ndarray) -> float:
    """Largest violation of a linear constraint at ``x`` (src/milp.jl:102-114)."""
    Ax = milp.A @ np.asarray(x, dtype=np.float64)
    d = Ax - milp.b
    eq = milp.is_eq
    v = 0.0
    if len(d):
        le_v = d[~eq]
        eq_v = np.abs(d[eq])
        if le_v.size:
            v = max(v, float(le_v.max()))
        if eq_v.size:
            v = max(v, float(eq_v.max()))
    return max(v, 0.0)


def is_integral(x: np.ndarray, idx: np.ndarray, tol: float = 1e-6) -> bool:
    """``all(|x_j - round(x_j)| <= tol)`` on ``idx`` (src/milp.jl:129-130), ties to even."""
    xi = np.asarray(x, dtype=np.float64)[idx]
    return bool(np.all(np.abs(xi - np.round(xi)) <= tol))


def is_feasible(milp: MILP, x: np.ndarray, tol: float = 1e-6) -> bool:
    """Integrality, bounds and every row to the absolute tolerance ``tol`` (src/milp.jl:122-127)."""
    x = np.asarray(x, dtype=np.float64)
    if len(x) != num_variables(milp):
        return False
    if not is_integral(x, milp.int_idx, tol):
        return False
    if not np.all((milp.l - tol <= x) & (x <= milp.u + tol)):
        return False
    return max_violation(milp, x) <= tol


def write_solution(path: str, milp: MILP, x: np.ndarray) -> str:
    """One ``name<TAB>value`` line per variable (src/milp.jl:138-145)."""
    with open(path, "w") as fh:
        for name, v in zip(milp.var_names, np.asarray(x, dtype=np.float64)):
            fh.write(f"{name}\t{float(v)!r}\n")
    return path
