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


@pytest.fixture(scope="session")
def examples():
    return {n: load_example(n) for n in EXAMPLES}


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O
