"""ctypes binding of libpdfp_b200.so (the C ABI declared in include/pdfp_b200.h).

The library is built in-tree (``pdfp_b200/lib/libpdfp_b200.so``, see
``pdfp_b200/csrc/Makefile``).  Loading fails loudly if it is missing: there is
no CPU fallback for any solver entry point.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("PDFP_B200_LIB") or os.path.join(_HERE, "lib", "libpdfp_b200.so")

OK = 0
E_INVALID, E_CUDA, E_NOMEM, E_TIMEOUT, E_UNSUPPORTED, E_NODEVICE = -1, -2, -3, -4, -5, -6
FP64, MIXED = 0, 1
VEC = {"pdhg_x": 0, "pdhg_y": 1, "pdhg_z": 2, "current_x": 3, "current_y": 4, "current_z": 5,
       "dual_slack": 6, "reflected_x": 7}

# Every function the header declares, with its ctypes signature.
dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int32)
up = C.POINTER(C.c_uint8)
vp = C.c_void_p


class Csr(C.Structure):
    _fields_ = [("m", C.c_int32), ("n", C.c_int32), ("row_ptr", ip), ("col_idx", ip), ("val", dp)]


class Params(C.Structure):
    _fields_ = [
        ("eps_optimal_relative", C.c_double),
        ("eps_feasible_relative", C.c_double),
        ("iteration_limit", C.c_int64),
        ("time_limit", C.c_double),
        ("termination_evaluation_frequency", C.c_int32),
        ("sv_max_iterations", C.c_int32),
        ("reflection_coefficient", C.c_double),
        ("sv_tolerance", C.c_double),
        ("artificial_restart_threshold", C.c_double),
        ("sufficient_reduction_for_restart", C.c_double),
        ("necessary_reduction_for_restart", C.c_double),
        ("k_p", C.c_double),
        ("k_i", C.c_double),
        ("k_d", C.c_double),
        ("i_smooth", C.c_double),
    ]


class Result(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("restarts", C.c_int32),
        ("total_count", C.c_int64),
        ("rel_primal", C.c_double),
        ("rel_dual", C.c_double),
        ("rel_gap", C.c_double),
        ("primal_weight", C.c_double),
        ("step_size", C.c_double),
        ("max_singular_value", C.c_double),
        ("fixed_point_error", C.c_double),
        ("objective_value", C.c_double),
        ("polished", C.c_int32),
        ("precision", C.c_int32),
        ("device_ms", C.c_double),
        ("kernel_ms_primal", C.c_double),
        ("kernel_ms_dual", C.c_double),
        ("kernel_samples", C.c_int64),
        ("fp64_iterations", C.c_int64),
    ]

    def as_dict(self) -> dict:
        from .params import STATUS_NAMES
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["status"] = STATUS_NAMES.get(self.status, str(self.status))
        return d


class Problem(C.Structure):
    _fields_ = [("A", Csr), ("b", dp), ("is_eq", up), ("is_int", up), ("var_lb", dp),
                ("var_ub", dp), ("w", dp), ("row_unscale", dp)]


SIGNATURES = {
    "pdfp_default_params": (None, [C.POINTER(Params)]),
    "pdfp_last_error": (C.c_char_p, []),
    "pdfp_device_name": (C.c_int, [C.c_char_p, C.c_int32]),
    "pdfp_set_device": (C.c_int, [C.c_int32]),
    "pdfp_version": (C.c_char_p, []),
    "pdfp_create": (C.c_int, [C.POINTER(Csr), dp, up, up, dp, dp, dp, dp, C.c_int32,
                              C.POINTER(vp)]),
    "pdfp_create_batch": (C.c_int, [C.c_int32, C.POINTER(Problem), C.c_int32, C.POINTER(vp)]),
    "pdfp_set_x": (C.c_int, [vp, C.c_int32, dp]),
    "pdfp_set_target": (C.c_int, [vp, C.c_int32, dp]),
    "pdfp_warm_start": (C.c_int, [vp, C.c_int32]),
    "pdfp_solve": (C.c_int, [vp, C.POINTER(Params), C.c_double, C.POINTER(Result)]),
    "pdfp_solve_batch": (C.c_int, [vp, C.POINTER(Params), dp, C.POINTER(Result)]),
    "pdfp_solve_batch_any": (C.c_int, [vp, C.POINTER(Params), dp, up, C.POINTER(Result)]),
    "pdfp_get_vector": (C.c_int, [vp, C.c_int32, C.c_int32, dp]),
    "pdfp_get_x": (C.c_int, [vp, C.c_int32, dp]),
    "pdfp_set_col_scale": (C.c_int, [vp, C.c_int32, dp]),
    "pdfp_set_x_unscaled": (C.c_int, [vp, C.c_int32, dp]),
    "pdfp_set_target_unscaled": (C.c_int, [vp, C.c_int32, dp]),
    "pdfp_get_vector_unscaled": (C.c_int, [vp, C.c_int32, C.c_int32, dp]),
    "pdfp_get_x_unscaled": (C.c_int, [vp, C.c_int32, dp]),
    "pdfp_host_alloc": (C.c_int, [C.c_int64, C.POINTER(C.c_void_p)]),
    "pdfp_host_free": (C.c_int, [C.c_void_p]),
    "pdfp_shape": (C.c_int, [vp, C.c_int32, ip, ip, ip]),
    "pdfp_destroy": (C.c_int, [vp]),
    "pdfp_set_kernel_timing": (C.c_int, [vp, C.c_int32]),
    "pdfp_set_polish": (C.c_int, [vp, C.c_int32, C.c_double]),
    "pdfp_selftest_bounded_wait": (C.c_int, [C.c_int32, C.c_double]),
    "pdfp_get_tuning": (C.c_int, [vp, ip]),
    "pdfp_get_tuning_table": (C.c_int, [vp, C.POINTER(C.c_float), ip, C.c_int32, ip]),
    "pdfp_get_tuning_stages": (C.c_int, [vp, ip]),
    "pdfp_get_tuning_blocks": (C.c_int, [vp, ip]),
    "pdfp_get_tuning_reducers": (C.c_int, [vp, ip]),
    "pdfp_get_tuning_seg": (C.c_int, [vp, ip]),
    "pdfp_get_window_form": (C.c_int, [vp, ip]),
    "pdfp_profile_step": (C.c_int, [vp, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                    dp, dp]),
    "pdfp_scale_problem": (C.c_int, [C.POINTER(Csr), dp, dp, dp, dp, dp, C.c_int32, C.c_double,
                                     C.c_int32, dp, dp, dp, dp, dp, dp, dp, dp, dp, dp]),
    "pdfp_estimate_max_singular_value": (C.c_int, [C.POINTER(Csr), C.c_int32, C.c_double, dp, ip]),
    "pdfp_mps_read": (C.c_int, [C.c_char_p, C.POINTER(vp)]),
    "pdfp_mps_dims": (C.c_int, [vp, ip, ip, C.POINTER(C.c_int64), ip]),
    "pdfp_mps_get": (C.c_int, [vp, dp, dp, ip, ip, dp, dp, up, dp, dp, ip]),
    "pdfp_mps_destroy": (C.c_int, [vp]),
    "pdfp_rounder_create": (C.c_int, [C.POINTER(Csr), dp, up, dp, dp, up, C.POINTER(vp)]),
    "pdfp_rounder_round": (C.c_int, [vp, dp, ip, C.c_int32, C.c_int32, ip, C.c_int32, ip, C.c_int32,
                                     ip, C.c_int32, up, C.c_int64, dp, ip]),
    "pdfp_rounder_destroy": (C.c_int, [vp]),
    "pdfp_checker_create": (C.c_int, [C.POINTER(Csr), dp, up, C.POINTER(vp)]),
    "pdfp_checker_max_violation": (C.c_int, [vp, dp, dp]),
    "pdfp_checker_destroy": (C.c_int, [vp]),
    "pdfp_estimate_max_singular_value_noalloc": (C.c_int, [C.c_int32, C.c_int32, ip, ip, dp, ip,
                                                            ip, dp, C.c_int32, C.c_double,
                                                            C.c_void_p, dp, ip]),
    "pdlp_solve_relaxation": (C.c_int, [C.POINTER(Csr), dp, dp, dp, dp, up, C.c_double,
                                        C.c_double, C.c_int32, C.c_int32, dp, dp,
                                        C.POINTER(Result)]),
}


class LibraryError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libpdfp_b200 error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """Load libpdfp_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C pdfp_b200/csrc` "
                              "(or __graft_entry__.build()); there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != OK:
        msg = lib().pdfp_last_error()
        raise LibraryError(code, msg.decode() if msg else "")


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def dptr(a):
    return a.ctypes.data_as(dp) if a is not None else None


def iptr(a):
    return a.ctypes.data_as(ip)


def uptr(a):
    return a.ctypes.data_as(up) if a is not None else None


def make_csr(A):
    """(Csr struct, keep-alive arrays) for a scipy sparse matrix (sorted CSR, int32)."""
    import scipy.sparse as sp
    if not (sp.isspmatrix_csr(A) and A.dtype == np.float64 and A.has_canonical_format):
        A = sp.csr_matrix(A, dtype=np.float64)
        A.sum_duplicates()
        A.sort_indices()
    rp = np.ascontiguousarray(A.indptr, dtype=np.int32)
    ci = np.ascontiguousarray(A.indices, dtype=np.int32)
    v = np.ascontiguousarray(A.data, dtype=np.float64)
    if len(ci) == 0:
        ci = np.zeros(1, dtype=np.int32)
        v = np.zeros(1, dtype=np.float64)
    m, n = A.shape
    return Csr(m, n, iptr(rp), iptr(ci), dptr(v)), (rp, ci, v)


def make_params(p) -> Params:
    """A ``Params`` struct from a ``SolverParameters`` (or a dict of its flat fields)."""
    flat = p.flat() if hasattr(p, "flat") else dict(p)
    out = Params()
    lib().pdfp_default_params(C.byref(out))
    for k, v in flat.items():
        setattr(out, k, v)
    return out
