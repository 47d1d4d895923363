"""Shared fixtures: the `gpu` marker, fixture loaders and the oracle."""
import os
import sys

import numpy as np
import pytest
import scipy.sparse as sp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
# A checkout of the reference (MIT-Lu-Lab/PDFP), when one is at hand: tests that read
# its example files directly run only when PDFP_REFERENCE_DIR names it.
REFERENCE_DIR = os.environ.get("PDFP_REFERENCE_DIR", "")
REF_EXAMPLES = os.path.join(REFERENCE_DIR, "examples") if REFERENCE_DIR else ""

# Mixed-precision handles below 2^18 nonzeros compute in FP64 by default; the
# tests run the FP32 kernels on the small example models too (the threshold
# itself is tested in test_gpu_flat.py).
os.environ.setdefault("PDFP_MIXED_MIN_NNZ", "0")
EXAMPLES = ["p0201", "pk1", "gen-ip054", "markshare2"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the library's kernels")


def load_example(name: str):
    """A reference example model from its golden fixture (tests/golden/make_fixtures.py)."""
    from pdfp_b200.milp import MILP
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    A = sp.csr_matrix((d["data"], d["indices"], d["indptr"]), shape=tuple(d["shape"]))
    return MILP(d["c"], float(d["c0"]), A, d["b"], ["eq" if e else "le" for e in d["is_eq"]],
                d["l"], d["u"], d["int_idx"], name=str(d["name"]))


def host_kkt(sc, is_eq, is_int, w, xt_scaled, get, row_unscale=None):
    """compute_residual! (src/pdfp.jl:200-218) in FP64 on the host from a solver's
    vectors: get(name) returns pdhg_x, pdhg_y, pdhg_z or dual_slack (scaled units).
    Returns (rel_primal, rel_dual, rel_gap, l1 distance)."""
    x, y, z, ds = get("pdhg_x"), get("pdhg_y"), get("pdhg_z"), get("dual_slack")
    A, b = sc.A, sc.con_ub
    d = A @ x - b
    viol = np.where(is_eq, np.abs(d), np.maximum(d, 0.0))
    if row_unscale is not None:
        viol = viol * row_unscale
        bnorm = np.linalg.norm(b * row_unscale)
    else:
        bnorm = np.linalg.norm(b)
    rel_p = np.linalg.norm(viol) / (1.0 + bnorm)
    rel_d = np.linalg.norm(A.T @ z - y - ds) / (1.0 + np.linalg.norm(np.where(is_int, w, 0.0)))
    l1 = np.sum(np.where(is_int, w * np.abs(x - xt_scaled), 0.0))
    yt = np.sum(np.where(is_int, y * (xt_scaled - x), 0.0))
    gap = abs(yt + z @ d - l1) / (1.0 + np.sum(np.where(is_int, w * np.abs(xt_scaled), 0.0)))
    return rel_p, rel_d, gap, l1


@pytest.fixture(scope="session")
def examples():
    return {n: load_example(n) for n in EXAMPLES}


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O
