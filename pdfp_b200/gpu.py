"""The pump's solver entry points on the B200 library.

Host-side mirror of the reference interface for the hot path:

* ``PDFPState`` -- ``PDFPState(A, b, is_eq, is_int, var_lb, var_ub, w; use_gpu)``
  and its methods ``original_primal_residual!``, ``set_target!``,
  ``warm_start!``, ``pdfp_solve!`` and the fields ``pdhg_x``, ``total_count``,
  ``termination_reason`` (src/pdfp.jl:15-288);
* ``PDFPBatch`` -- many projections in one handle (one launch sequence);
* ``scale_problem`` / ``estimate_max_singular_value`` (src/preconditioner.jl);
* ``solve_lp_relaxation`` (src/pdlp.jl:381-393).

Everything runs in libpdfp_b200.so on the GPU; these classes own the handles
and convert arguments.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp

from . import _lib as L
from .params import STATUS_NAMES, SolverParameters


def device_name() -> str:
    buf = C.create_string_buffer(256)
    L.check(L.lib().pdfp_device_name(buf, 256))
    return buf.value.decode()


class _HostBlock:
    """One pdfp_host_alloc block; freed when the last array viewing it goes."""

    def __init__(self, nbytes: int):
        self.ptr = C.c_void_p()
        L.check(L.lib().pdfp_host_alloc(max(int(nbytes), 1), C.byref(self.ptr)))

    def __del__(self):
        try:
            if self.ptr.value:
                L.lib().pdfp_host_free(self.ptr)
                self.ptr = C.c_void_p()
        except Exception:  # noqa: BLE001 (interpreter shutdown)
            pass


def pinned_zeros(n: int) -> np.ndarray:
    """A float64 array of n zeros in page-locked host memory (pdfp_host_alloc).

    Vectors passed to the setters and getters from such an array cross to and from
    the device at DMA speed; any other array works too, more slowly.
    """
    block = _HostBlock(8 * n)
    raw = (C.c_double * max(n, 1)).from_address(block.ptr.value)
    raw._block = block  # the numpy view keeps raw, raw keeps the block
    a = np.frombuffer(raw, dtype=np.float64)[:n]
    a[:] = 0.0
    return a


def _out(out, size):
    """The caller's output array (float64, contiguous, at least `size` long) or a new one."""
    if out is None:
        return np.zeros(max(size, 1))
    if out.dtype != np.float64 or not out.flags.c_contiguous or out.size < size:
        raise ValueError("out must be a contiguous float64 array of the vector's length")
    return out


def selftest_bounded_wait(which: int, limit_seconds: float = 0.05) -> int:
    """Run the library's bounded-wait self-test (pdfp_selftest_bounded_wait): 0 the
    mbarrier wait, 1 the grid barrier.  Returns the status code (E_TIMEOUT when the
    wait gave up as designed)."""
    return L.lib().pdfp_selftest_bounded_wait(int(which), float(limit_seconds))


def set_device(device: int) -> None:
    """Select the CUDA device of this thread's later library calls (one per rank)."""
    L.check(L.lib().pdfp_set_device(int(device)))


def _precision_code(precision: str) -> int:
    if precision in ("fp64", "FP64", L.FP64):
        return L.FP64
    if precision in ("mixed", "MIXED", L.MIXED):
        return L.MIXED
    raise ValueError("precision must be 'fp64' or 'mixed'")


class PDFPState:
    """Projector state on the GPU for the scaled data (src/pdfp.jl:60-76)."""

    def __init__(self, A, b, is_eq, is_int, var_lb, var_ub, w, *, precision: str = "fp64",
                 row_unscale=None):
        self._h = C.c_void_p()
        csr, keep = L.make_csr(A)
        m, n = csr.m, csr.n
        self.m, self.n = m, n
        self.precision = precision
        arrs = [L.f64(b), np.ascontiguousarray(is_eq, dtype=np.uint8),
                np.ascontiguousarray(is_int, dtype=np.uint8), L.f64(var_lb), L.f64(var_ub),
                L.f64(w)]
        ru = None if row_unscale is None else L.f64(row_unscale)
        self._create_args = (csr, keep, arrs, ru)
        self._created = False
        self._precision_code = _precision_code(precision)
        self._create()
        self.total_count = 0
        self.termination_reason = "UNSPECIFIED"
        self.last = None

    def _create(self):
        csr, keep, arrs, ru = self._create_args
        if self._created:
            L.check(L.lib().pdfp_destroy(self._h))
            self._h = C.c_void_p()
        b, ie, ii, lb, ub, w = arrs
        L.check(L.lib().pdfp_create(C.byref(csr), L.dptr(b), L.uptr(ie), L.uptr(ii), L.dptr(lb),
                                    L.dptr(ub), L.dptr(w), L.dptr(ru), self._precision_code,
                                    C.byref(self._h)))
        self._created = True
        if getattr(self, "_polish", None) is not None:
            L.check(L.lib().pdfp_set_polish(self._h, *self._polish))

    def set_polish(self, stall_evaluations: int = 10, fp32_floor: float = 1e-6):
        """Mixed precision: when the FP64 polish takes over from the FP32 phase
        (pdfp_set_polish): after `stall_evaluations` evaluations without a 10% KKT
        improvement (0: never), or once the residuals reach `fp32_floor` under a
        tighter tolerance."""
        self._polish = (int(stall_evaluations), float(fp32_floor))
        L.check(L.lib().pdfp_set_polish(self._h, *self._polish))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            L.lib().pdfp_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 (interpreter shutdown)
            pass

    def original_primal_residual(self, D_r):
        """original_primal_residual!(s, D_r), src/pdfp.jl:85-90 (rebuilds the handle)."""
        csr, keep, arrs, _ = self._create_args
        self._create_args = (csr, keep, arrs, L.f64(1.0 / np.asarray(D_r, dtype=np.float64)))
        self._create()
        return self

    def set_x(self, x):
        """copyto!(s.current_x, x); copyto!(s.initial_x, x) (src/pump.jl:305-306)."""
        L.check(L.lib().pdfp_set_x(self._h, 0, L.dptr(L.f64(x))))

    def set_target(self, x_tilde):
        """set_target!(s, x_tilde_scaled), src/pdfp.jl:98-101."""
        L.check(L.lib().pdfp_set_target(self._h, 0, L.dptr(L.f64(x_tilde))))
        self.total_count = 0

    def warm_start(self):
        """warm_start!(s), src/pdfp.jl:104-114."""
        L.check(L.lib().pdfp_warm_start(self._h, 0))
        self.total_count = 0

    def solve(self, params: SolverParameters, primal_weight: float) -> str:
        """pdfp_solve!(s, p, primal_weight) -> termination reason, src/pdfp.jl:252-288."""
        r = L.Result()
        L.check(L.lib().pdfp_solve(self._h, C.byref(L.make_params(params)), float(primal_weight),
                                   C.byref(r)))
        self.last = r.as_dict()
        self.total_count = int(r.total_count)
        self.termination_reason = STATUS_NAMES.get(r.status, str(r.status))
        return self.termination_reason

    def get(self, which: str, out=None) -> np.ndarray:
        size = self.m if which.endswith("_z") else self.n
        out = _out(out, size)
        L.check(L.lib().pdfp_get_vector(self._h, 0, L.VEC[which], L.dptr(out)))
        return out[:size]

    @property
    def pdhg_x(self) -> np.ndarray:
        return self.get("pdhg_x")

    # The pump's column scaling on the device (src/pump.jl:305-306, 331, 338):
    # after set_col_scale(D_c), these take and return vectors in the model's
    # own units, bit-identical to x ./ D_c and D_c .* s.pdhg_x on the host.
    def set_col_scale(self, D_c):
        L.check(L.lib().pdfp_set_col_scale(self._h, 0, L.dptr(L.f64(D_c))))

    def set_x_unscaled(self, x):
        L.check(L.lib().pdfp_set_x_unscaled(self._h, 0, L.dptr(L.f64(x))))

    def set_target_unscaled(self, x_tilde):
        L.check(L.lib().pdfp_set_target_unscaled(self._h, 0, L.dptr(L.f64(x_tilde))))
        self.total_count = 0

    def get_unscaled(self, which: str = "pdhg_x", out=None) -> np.ndarray:
        out = _out(out, self.n)
        L.check(L.lib().pdfp_get_vector_unscaled(self._h, 0, L.VEC[which], L.dptr(out)))
        return out[:self.n]

    def tuning(self):
        """The step kernels' configuration (pdfp_get_tuning): A' stage bytes, threads
        per role (0: flat engine, 32: vec engine, whose stage bytes are its nonzeros per
        lane), tiles (vec engine: work items), the same three for A, then the A' and A
        gather policies."""
        out = (C.c_int32 * 8)()
        L.check(L.lib().pdfp_get_tuning(self._h, out))
        return list(out)

    def profile_step(self, iterations: int):
        a, b = C.c_float(), C.c_float()
        ba, bb = C.c_double(), C.c_double()
        L.check(L.lib().pdfp_profile_step(self._h, iterations, C.byref(a), C.byref(b),
                                          C.byref(ba), C.byref(bb)))
        return a.value, b.value, ba.value, bb.value


class PDFPBatch:
    """k projections packed into one handle; one launch sequence advances all of them."""

    def __init__(self, problems, *, precision: str = "fp64"):
        self._h = C.c_void_p()
        structs = []
        self._keep = []
        self.shapes = []
        for pr in problems:
            A, b, is_eq, is_int, lb, ub, w = pr[:7]
            ru = pr[7] if len(pr) > 7 else None
            csr, keep = L.make_csr(A)
            arrs = [L.f64(b), np.ascontiguousarray(is_eq, dtype=np.uint8),
                    np.ascontiguousarray(is_int, dtype=np.uint8), L.f64(lb), L.f64(ub), L.f64(w),
                    None if ru is None else L.f64(ru)]
            self._keep.append((keep, arrs))
            structs.append(L.Problem(csr, L.dptr(arrs[0]), L.uptr(arrs[1]), L.uptr(arrs[2]),
                                     L.dptr(arrs[3]), L.dptr(arrs[4]), L.dptr(arrs[5]),
                                     L.dptr(arrs[6])))
            self.shapes.append((csr.m, csr.n))
        self.k = len(structs)
        arr = (L.Problem * self.k)(*structs)
        L.check(L.lib().pdfp_create_batch(self.k, arr, _precision_code(precision),
                                          C.byref(self._h)))
        self.results = [None] * self.k

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            L.lib().pdfp_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def set_x(self, p: int, x):
        L.check(L.lib().pdfp_set_x(self._h, p, L.dptr(L.f64(x))))

    def set_target(self, p: int, x_tilde):
        L.check(L.lib().pdfp_set_target(self._h, p, L.dptr(L.f64(x_tilde))))

    def warm_start(self, p: int):
        L.check(L.lib().pdfp_warm_start(self._h, p))

    def solve(self, params, primal_weights):
        if isinstance(params, SolverParameters):
            params = [params] * self.k
        ps = (L.Params * self.k)(*[L.make_params(p) for p in params])
        pw = L.f64(np.broadcast_to(np.asarray(primal_weights, dtype=np.float64), (self.k,)))
        rs = (L.Result * self.k)()
        L.check(L.lib().pdfp_solve_batch(self._h, ps, L.dptr(pw), rs))
        self.results = [r.as_dict() for r in rs]
        return [r["status"] for r in self.results]

    def tuning(self):
        """The step kernels' configuration (pdfp_get_tuning), as PDFPState.tuning reports it."""
        out = (C.c_int32 * 8)()
        L.check(L.lib().pdfp_get_tuning(self._h, out))
        return list(out)

    def solve_any(self, params, primal_weights, resume=None):
        """pdfp_solve_batch_any: solve until at least one running member stops.

        Members still running when it returns report "RUNNING"; pass resume[p] =
        True on the next call to continue member p where it stopped (its params
        entry is then not read).  Returns the members' statuses."""
        if isinstance(params, SolverParameters):
            params = [params] * self.k
        ps = (L.Params * self.k)(*[L.make_params(p) for p in params])
        pw = L.f64(np.broadcast_to(np.asarray(primal_weights, dtype=np.float64), (self.k,)))
        rs = (L.Result * self.k)()
        rz = None
        if resume is not None:
            rz = np.ascontiguousarray(np.broadcast_to(np.asarray(resume, dtype=bool), (self.k,)),
                                      dtype=np.uint8)
        L.check(L.lib().pdfp_solve_batch_any(self._h, ps, L.dptr(pw),
                                             L.uptr(rz) if rz is not None else None, rs))
        self.results = [r.as_dict() for r in rs]
        for d in self.results:
            if d["status"] == "UNSPECIFIED":
                d["status"] = "RUNNING"
        return [d["status"] for d in self.results]

    def get(self, p: int, which: str, out=None) -> np.ndarray:
        m, n = self.shapes[p]
        size = m if which.endswith("_z") else n
        out = _out(out, size)
        L.check(L.lib().pdfp_get_vector(self._h, p, L.VEC[which], L.dptr(out)))
        return out[:size]

    def set_col_scale(self, p: int, D_c):
        L.check(L.lib().pdfp_set_col_scale(self._h, p, L.dptr(L.f64(D_c))))

    def set_x_unscaled(self, p: int, x):
        L.check(L.lib().pdfp_set_x_unscaled(self._h, p, L.dptr(L.f64(x))))

    def set_target_unscaled(self, p: int, x_tilde):
        L.check(L.lib().pdfp_set_target_unscaled(self._h, p, L.dptr(L.f64(x_tilde))))

    def get_unscaled(self, p: int, which: str = "pdhg_x", out=None) -> np.ndarray:
        n = self.shapes[p][1]
        out = _out(out, n)
        L.check(L.lib().pdfp_get_vector_unscaled(self._h, p, L.VEC[which], L.dptr(out)))
        return out[:n]


class ConstraintChecker:
    """max_violation(milp, x) (src/milp.jl:102-114) on the device, bit-identical to
    the host evaluation; keeps the original constraints on the GPU."""

    def __init__(self, milp):
        csr, keep = L.make_csr(milp.A)
        self._keep = (keep, L.f64(milp.b), np.ascontiguousarray(milp.is_eq, dtype=np.uint8))
        self.n = csr.n
        self._h = C.c_void_p()
        L.check(L.lib().pdfp_checker_create(C.byref(csr), L.dptr(self._keep[1]),
                                            L.uptr(self._keep[2]), C.byref(self._h)))

    def max_violation(self, x) -> float:
        v = C.c_double()
        xa = L.f64(x)
        if len(xa) != self.n:
            raise ValueError("x has the wrong length")
        L.check(L.lib().pdfp_checker_max_violation(self._h, L.dptr(xa), C.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            L.lib().pdfp_checker_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


@dataclass
class ScaledProblem:
    """src/preconditioner.jl:13-24"""

    A: sp.csr_matrix
    c: np.ndarray
    var_lb: np.ndarray
    var_ub: np.ndarray
    con_lb: np.ndarray
    con_ub: np.ndarray
    D_r: np.ndarray
    D_c: np.ndarray
    bound_scale: float
    objective_scale: float


def scale_problem(A, c, var_lb, var_ub, con_lb, con_ub, ruiz_iterations: int = 10,
                  pock_chambolle_alpha: float = 1.0,
                  bound_objective_rescaling: bool = True) -> ScaledProblem:
    """scale_problem, src/preconditioner.jl:26-99, on the GPU."""
    csr, (rp, ci, v) = L.make_csr(A)
    m, n = csr.m, csr.n
    nnz = int(rp[-1])
    vals = np.zeros(max(nnz, 1))
    on = [np.zeros(max(n, 1)) for _ in range(4)]
    om = [np.zeros(max(m, 1)) for _ in range(3)]
    bs, os_ = C.c_double(), C.c_double()
    L.check(L.lib().pdfp_scale_problem(
        C.byref(csr), L.dptr(L.f64(c)), L.dptr(L.f64(var_lb)), L.dptr(L.f64(var_ub)),
        L.dptr(L.f64(con_lb)), L.dptr(L.f64(con_ub)), ruiz_iterations, pock_chambolle_alpha,
        int(bool(bound_objective_rescaling)), L.dptr(vals), L.dptr(on[0]), L.dptr(on[1]),
        L.dptr(on[2]), L.dptr(om[0]), L.dptr(om[1]), L.dptr(om[2]), L.dptr(on[3]),
        C.byref(bs), C.byref(os_)))
    As = sp.csr_matrix((vals[:nnz].copy(), ci[:nnz].copy(), rp.copy()), shape=(m, n))
    return ScaledProblem(As, on[0][:n], on[1][:n], on[2][:n], om[0][:m], om[1][:m], om[2][:m],
                         on[3][:n], bs.value, os_.value)


def estimate_max_singular_value(A, max_iterations: int = 5000, tolerance: float = 1e-4):
    """estimate_max_singular_value, src/preconditioner.jl:108-125, on the GPU: (sigma, iterations)."""
    csr, keep = L.make_csr(A)
    s = C.c_double()
    it = C.c_int32()
    L.check(L.lib().pdfp_estimate_max_singular_value(C.byref(csr), max_iterations, tolerance,
                                                      C.byref(s), C.byref(it)))
    return s.value, it.value


def solve_lp_relaxation(milp, tolerance: float = 1e-2, time_limit: float = 3600.0,
                        cupdlpx_termination: bool = False, precision: str = "fp64",
                        return_result: bool = False):
    """solve_lp_relaxation, src/pdlp.jl:381-393, on the GPU: (x, dual_slack, status, iterations)."""
    csr, keep = L.make_csr(milp.A)
    n = csr.n
    is_le = np.array([s == "le" for s in milp.row_sense], dtype=np.uint8)
    x = np.zeros(max(n, 1))
    ds = np.zeros(max(n, 1))
    r = L.Result()
    L.check(L.lib().pdlp_solve_relaxation(
        C.byref(csr), L.dptr(L.f64(milp.c)), L.dptr(L.f64(milp.l)), L.dptr(L.f64(milp.u)),
        L.dptr(L.f64(milp.b)), L.uptr(is_le if len(is_le) else np.zeros(1, np.uint8)),
        float(tolerance), float(time_limit), int(bool(cupdlpx_termination)),
        _precision_code(precision), L.dptr(x), L.dptr(ds), C.byref(r)))
    status = STATUS_NAMES.get(r.status, str(r.status))
    out = (x[:n], ds[:n], status, int(r.total_count))
    return out + (r.as_dict(),) if return_result else out
