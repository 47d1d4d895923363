"""CPU checks of the packed layout and the tile/chunk builder of libpdfp_b200.

The C++ checker (tests/native/layout_check.cpp) is compiled from the library's
own layout sources with g++; it verifies the permutations, that A' is the
transpose of A with the reference's summation order, and that every chunk of
every tiling fits its shared-memory stage (the bound the kernels rely on).
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(ROOT, "_build", "liblayout_check.so")


@pytest.fixture(scope="module")
def checker():
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    srcs = [os.path.join(HERE, "native", "layout_check.cpp"),
            os.path.join(ROOT, "pdfp_b200", "csrc", "layout.cpp")]
    subprocess.run(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-o", OUT] + srcs, check=True)
    lib = C.CDLL(OUT)
    lib.layout_check.restype = C.c_int
    return lib


def run(lib, mats, eqs, stage_bytes=40 * 1024):
    K = len(mats)
    keep = []
    ms = (C.c_int32 * K)()
    ns = (C.c_int32 * K)()
    rps = (C.POINTER(C.c_int32) * K)()
    cis = (C.POINTER(C.c_int32) * K)()
    vs = (C.POINTER(C.c_double) * K)()
    es = (C.POINTER(C.c_uint8) * K)()
    for p, (A, e) in enumerate(zip(mats, eqs)):
        A = sp.csr_matrix(A)
        A.sort_indices()
        rp = np.ascontiguousarray(A.indptr, dtype=np.int32)
        ci = np.ascontiguousarray(A.indices if A.nnz else np.zeros(1), dtype=np.int32)
        v = np.ascontiguousarray(A.data if A.nnz else np.zeros(1), dtype=np.float64)
        ee = np.ascontiguousarray(e, dtype=np.uint8) if len(e) else np.zeros(1, np.uint8)
        keep += [rp, ci, v, ee]
        ms[p], ns[p] = A.shape
        rps[p] = rp.ctypes.data_as(C.POINTER(C.c_int32))
        cis[p] = ci.ctypes.data_as(C.POINTER(C.c_int32))
        vs[p] = v.ctypes.data_as(C.POINTER(C.c_double))
        es[p] = ee.ctypes.data_as(C.POINTER(C.c_uint8))
    stats = (C.c_int64 * 3)()
    rc = lib.layout_check(K, ms, ns, rps, cis, vs, es, stage_bytes, stats)
    run.n_seg_long = stats[2]  # long rows taken by the segmented form, summed over its cases
    return rc, stats[0], stats[1]


def rand_csr(rng, m, n, density, long_rows=0, long_len=0):
    A = sp.random(m, n, density=density, random_state=rng, format="lil")
    for i in range(long_rows):
        cols = rng.choice(n, size=min(long_len, n), replace=False)
        A[i, cols] = rng.uniform(-1, 1, size=len(cols))
    return sp.csr_matrix(A)


def test_layout_single_instance(checker):
    rng = np.random.default_rng(0)
    A = rand_csr(rng, 300, 500, 0.02)
    rc, tiles, _ = run(checker, [A], [rng.random(300) < 0.3])
    assert rc == 0 and tiles > 0


def test_layout_long_rows_split_into_chunks(checker):
    rng = np.random.default_rng(1)
    A = rand_csr(rng, 50, 40000, 0.0005, long_rows=3, long_len=30000)
    rc, tiles, n_long = run(checker, [A], [np.zeros(50, bool)], stage_bytes=16 * 1024)
    assert rc == 0 and n_long > 0
    assert run.n_seg_long > 0  # the segmented form took long rows


def test_layout_batch_with_empty_rows_cols_and_instances(checker):
    rng = np.random.default_rng(2)
    mats = [rand_csr(rng, 80, 60, 0.05), sp.csr_matrix((0, 5)), sp.csr_matrix((7, 0)),
            sp.csr_matrix((4, 6)), rand_csr(rng, 1000, 30, 0.3)]
    eqs = [rng.random(A.shape[0]) < 0.5 for A in mats]
    rc, tiles, _ = run(checker, mats, eqs, stage_bytes=8 * 1024)
    assert rc == 0


def test_layout_many_short_rows(checker):
    rng = np.random.default_rng(3)
    A = sp.csr_matrix(sp.eye(20000) * 2.0)
    rc, tiles, _ = run(checker, [A], [np.ones(20000, bool)])
    assert rc == 0 and tiles > 5
