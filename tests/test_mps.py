"""The C++ MPS reader (pdfp_mps_*) against the Python reader (src/milp.jl:42-94).

Both read the same files -- models written from the golden fixtures, a
hand-written file exercising every section and bound type, and, where the
reference's example files are present, those -- and must give the same
canonical model exactly.  No GPU is needed.
"""
import gzip
import os

import numpy as np
import pytest

from conftest import EXAMPLES, REF_EXAMPLES, load_example
from pdfp_b200.milp import read_mps, read_mps_native


def same_model(a, b):
    assert a.A.shape == b.A.shape
    A, B = a.A.tocsr(), b.A.tocsr()
    A.sort_indices()
    B.sort_indices()
    assert np.array_equal(A.indptr, B.indptr) and np.array_equal(A.indices, B.indices)
    assert np.array_equal(A.data, B.data)
    for x, y in [(a.c, b.c), (a.b, b.b), (a.l, b.l), (a.u, b.u)]:
        assert np.array_equal(x, y)
    assert a.c0 == b.c0
    assert list(a.row_sense) == list(b.row_sense)
    assert np.array_equal(np.asarray(a.int_idx), np.asarray(b.int_idx))


def write_mps(m, path):
    """Free MPS of a canonical model (rows L/E, integer markers, bounds)."""
    A = m.A.tocsc()
    lines = ["NAME t", "ROWS", " N obj"]
    lines += [f" {'E' if s == 'eq' else 'L'} r{i}" for i, s in enumerate(m.row_sense)]
    lines.append("COLUMNS")
    is_int = np.zeros(len(m.c), bool)
    is_int[m.int_idx] = True
    inside = False
    for j in range(A.shape[1]):
        if is_int[j] != inside:
            lines.append(f"    M{j} 'MARKER' '{'INTORG' if is_int[j] else 'INTEND'}'")
            inside = is_int[j]
        if m.c[j] != 0:
            lines.append(f"    x{j} obj {float(m.c[j])!r}")
        for k in range(A.indptr[j], A.indptr[j + 1]):
            lines.append(f"    x{j} r{A.indices[k]} {float(A.data[k])!r}")
        if A.indptr[j] == A.indptr[j + 1] and m.c[j] == 0:
            lines.append(f"    x{j} obj 0")
    if inside:
        lines.append("    Mend 'MARKER' 'INTEND'")
    lines.append("RHS")
    lines += [f"    rhs r{i} {float(v)!r}" for i, v in enumerate(m.b) if v != 0]
    if m.c0 != 0:
        lines.append(f"    rhs obj {float(-m.c0)!r}")
    lines.append("BOUNDS")
    for j in range(len(m.c)):
        lo, hi = m.l[j], m.u[j]
        if np.isinf(lo):
            lines.append(f" MI bnd x{j}")
        elif lo != 0:
            lines.append(f" LO bnd x{j} {float(lo)!r}")
        if np.isfinite(hi):
            lines.append(f" UP bnd x{j} {float(hi)!r}")
    lines.append("ENDATA")
    with gzip.open(path, "wt") as f:
        f.write("\n".join(lines) + "\n")


@pytest.mark.parametrize("name", EXAMPLES)
def test_native_equals_python_on_fixture_models(tmp_path, name):
    p = str(tmp_path / f"{name}.mps.gz")
    write_mps(load_example(name), p)
    same_model(read_mps_native(p), read_mps(p))


@pytest.mark.skipif(not (REF_EXAMPLES and os.path.isdir(REF_EXAMPLES)),
                    reason="no reference checkout (PDFP_REFERENCE_DIR)")
@pytest.mark.parametrize("name", EXAMPLES)
def test_native_equals_python_on_reference_examples(name):
    p = os.path.join(REF_EXAMPLES, f"{name}.mps.gz")
    a, b = read_mps_native(p), read_mps(p)
    same_model(a, b)
    same_model(a, load_example(name))


SPECIAL = """* every section and bound type
NAME          special
OBJSENSE
    MAX
ROWS
 N  cost
 L  lim1
 G  lim2
 E  myeqn
 L  rng
 N  spare
COLUMNS
    MARKER                 'MARKER'                 'INTORG'
    x1        cost         1.0   lim1         1.0
    x1        lim2         1.0
    MARKER                 'MARKER'                 'INTEND'
    x2        cost         2.0   lim1         1.0
    x2        myeqn       -1.0   rng          2.5
    x2        lim1         0.5
    x3        cost        -1.0   myeqn        1.0
    x3        spare        9.0
    x4        lim2         3.0   rng          1.0
    x5        cost         1.0
    x6        lim1         1.0
    x7        rng          1.0
RHS
    RHS       cost        -4.5
    RHS       lim1         4.0   lim2         1.0
    RHS       myeqn        7.0   rng          2.0
RANGES
    RNG       rng          3.0   myeqn        2.0
    RNG       lim2         5.0
BOUNDS
 UP BND       x1           4.0
 LO BND       x2          -1.0
 UP BND       x2           1.0
 MI BND       x3
 BV BND       x4
 FR BND       x5
 LI BND       x6           2
 UI BND       x6           9
 UP BND       x7          -2.0
 PL BND       x1
ENDATA
"""


def test_native_equals_python_on_every_section(tmp_path):
    p = str(tmp_path / "special.mps")
    open(p, "w").write(SPECIAL)
    a, b = read_mps_native(p), read_mps(p)
    same_model(a, b)
    assert a.A.shape[1] == 7 and a.c0 == -4.5  # c0 = -RHS(cost) = 4.5, negated for MAX
    assert list(a.int_idx) == [0, 3, 5]


def test_native_reader_errors(tmp_path):
    with pytest.raises(Exception, match="cannot open"):
        read_mps_native(str(tmp_path / "missing.mps"))
    p = str(tmp_path / "bad.mps")
    open(p, "w").write("ROWS\n N obj\n L r\nCOLUMNS\n    x obj abc\nENDATA\n")
    with pytest.raises(Exception, match="bad number"):
        read_mps_native(p)
