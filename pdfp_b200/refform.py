"""The reference's GPU step as written (libpdfp_refform.so), for comparison.

``RefFormState`` drives the plain FP64 step the reference runs on a CuVector
state -- cuSPARSE SpMV with A', primal kernel, dual_y kernel, cuSPARSE SpMV with
A, dual_z kernel (src/pdfp_kernels.jl:4-86) -- so the benchmark can time the
fused projector against it on the same GPU.  Not part of the drop-in.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib as L

REF_LIB_PATH = os.path.join(os.path.dirname(L.LIB_PATH), "libpdfp_refform.so")
_ref = None

_dp = C.POINTER(C.c_double)
_u8 = C.POINTER(C.c_uint8)
SIGNATURES = {
    "pdfp_refform_last_error": (C.c_char_p, []),
    "pdfp_refform_create": (C.c_int, [C.POINTER(L.Csr), _dp, _u8, _u8, _dp, _dp, _dp,
                                      C.POINTER(C.c_void_p)]),
    "pdfp_refform_reset": (C.c_int, [C.c_void_p, _dp, _dp]),
    "pdfp_refform_steps": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                     C.POINTER(C.c_float)]),
    "pdfp_refform_get": (C.c_int, [C.c_void_p, C.c_int32, _dp]),
    "pdfp_refform_destroy": (C.c_int, [C.c_void_p]),
}


def lib():
    """Load libpdfp_refform.so (raises if it has not been built)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB_PATH):
            raise ImportError(f"{REF_LIB_PATH} is missing: build it with `make -C pdfp_b200/csrc`")
        R = C.CDLL(REF_LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(R, name)
            f.restype = res
            f.argtypes = args
        _ref = R
    return _ref


def _check(rc):
    if rc != L.OK:
        raise L.LibraryError(rc, lib().pdfp_refform_last_error().decode())


class RefFormState:
    """PDFPState{CuVector} of the reference, stepped with pdhg_step! only."""

    def __init__(self, A, b, is_eq, is_int, var_lb, var_ub, w):
        csr, keep = L.make_csr(A)
        self.m, self.n = csr.m, csr.n
        arrs = [L.f64(b), np.ascontiguousarray(is_eq, dtype=np.uint8),
                np.ascontiguousarray(is_int, dtype=np.uint8), L.f64(var_lb), L.f64(var_ub),
                L.f64(w)]
        self._h = C.c_void_p()
        _check(lib().pdfp_refform_create(C.byref(csr), L.dptr(arrs[0]), L.uptr(arrs[1]),
                                         L.uptr(arrs[2]), L.dptr(arrs[3]), L.dptr(arrs[4]),
                                         L.dptr(arrs[5]), C.byref(self._h)))
        del keep, arrs

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().pdfp_refform_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def reset(self, x_tilde, x0):
        _check(lib().pdfp_refform_reset(self._h, L.dptr(L.f64(x_tilde)), L.dptr(L.f64(x0))))

    def steps(self, step_size: float, primal_weight: float, k0: int, count: int) -> float:
        """Run ``count`` steps; returns their device time in ms."""
        ms = C.c_float()
        _check(lib().pdfp_refform_steps(self._h, step_size, primal_weight, k0, count,
                                        C.byref(ms)))
        return float(ms.value)

    def get(self, which: str) -> np.ndarray:
        code = {"pdhg_x": 0, "current_x": 1, "pdhg_z": 2, "current_z": 3}[which]
        out = np.zeros(self.n if code < 2 else self.m)
        _check(lib().pdfp_refform_get(self._h, code, L.dptr(out)))
        return out
