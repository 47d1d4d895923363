"""The reference-structured FP64 step (libpdfp_refform.so), the comparison form.

CPU: the library loads and exports what include/pdfp_refform.h declares, and
rejects bad arguments before touching a device.  GPU: its steps equal the
oracle's steps (the reference's algorithm) on the same scaled problem.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from pdfp_b200 import refform

HEADER = os.path.join(ROOT, "include", "pdfp_refform.h")


def test_refform_library_exports_its_header():
    text = open(HEADER).read()
    syms = sorted(set(re.findall(r"PDFP_API\s+[\w\s\*]+?\b(pdfp_refform_\w+)\s*\(", text)))
    assert len(syms) == 6
    lib = C.CDLL(refform.REF_LIB_PATH)
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(refform.SIGNATURES)


def test_refform_rejects_bad_arguments():
    R = refform.lib()
    h = C.c_void_p()
    assert R.pdfp_refform_create(None, None, None, None, None, None, None, C.byref(h)) != 0
    assert b"null" in R.pdfp_refform_last_error()
    assert R.pdfp_refform_steps(None, 1.0, 1.0, 1, 1, None) != 0
    assert R.pdfp_refform_get(None, 0, None) != 0


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["p0201", "pk1"])
def test_refform_steps_equal_the_oracle_steps(examples, oracle, name):
    m = examples[name]
    sc, is_eq, is_int, w = oracle.projector_inputs(m)
    rng = np.random.default_rng(5)
    xt = np.round(rng.random(len(m.c))) / sc.D_c
    x0 = rng.random(len(m.c)) / sc.D_c
    o = oracle.OraclePDFP(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w)
    o.set_x(x0)
    o.set_target(xt)
    o.steps(0.7, 1.3, 1, 60)
    r = refform.RefFormState(sc.A, sc.con_ub, is_eq, is_int, sc.var_lb, sc.var_ub, w)
    r.reset(xt, x0)
    ms = r.steps(0.7, 1.3, 1, 60)
    assert ms > 0.0
    for which in ("pdhg_x", "current_x", "pdhg_z", "current_z"):
        a, b = r.get(which), o.get(which)
        assert np.allclose(a, b, rtol=1e-11, atol=1e-11), which
