"""The C ABI of libpdfp_b200.so: the library loads, exports every entry point
include/pdfp_b200.h declares, and its host-only entry points behave without a GPU."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT
from pdfp_b200 import _lib as L

HEADER = os.path.join(ROOT, "include", "pdfp_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"PDFP_API\s+[\w\s\*]+?\b((?:pdfp|pdlp)_\w+)\s*\(", text)))


def test_library_exists_and_loads():
    assert os.path.exists(L.LIB_PATH), "build the library first (make -C pdfp_b200/csrc)"
    L.lib()


def test_every_declared_symbol_is_exported():
    lib = C.CDLL(L.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 19
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) <= set(L.SIGNATURES), "binding is missing a declared function"


def test_default_params_are_the_reference_defaults():
    p = L.Params()
    L.lib().pdfp_default_params(C.byref(p))
    # src/pdlp.jl:10-31
    assert (p.eps_optimal_relative, p.eps_feasible_relative) == (1e-4, 1e-4)
    assert p.iteration_limit == 100_000 and p.termination_evaluation_frequency == 200
    assert p.sv_max_iterations == 5000 and p.sv_tolerance == 1e-4
    assert (p.artificial_restart_threshold, p.sufficient_reduction_for_restart,
            p.necessary_reduction_for_restart) == (0.36, 0.2, 0.5)
    assert (p.k_p, p.k_i, p.k_d, p.i_smooth) == (0.99, 0.01, 0.0, 0.3)


def test_version_and_last_error_strings():
    assert b"sm_100a" in L.lib().pdfp_version()
    assert isinstance(L.lib().pdfp_last_error(), bytes)


def test_struct_layouts_match_the_header(tmp_path):
    """ctypes layouts equal the C compiler's (sizes and every field offset)."""
    import subprocess
    structs = {"pdfp_params": L.Params, "pdfp_result": L.Result, "pdfp_csr": L.Csr,
               "pdfp_problem": L.Problem}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                 check=True).stdout.splitlines())
    for cname, cls in structs.items():
        assert int(got[cname]) == C.sizeof(cls), cname
        for f, _ in cls._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(cls, f).offset, f"{cname}.{f}"


def test_null_arguments_are_rejected_without_touching_the_device():
    h = C.c_void_p()
    rc = L.lib().pdfp_create(None, None, None, None, None, None, None, None, 0, C.byref(h))
    assert rc == L.E_INVALID
    assert b"null" in L.lib().pdfp_last_error()
    assert L.lib().pdfp_set_target(None, 0, None) == L.E_INVALID
    assert L.lib().pdfp_solve(None, None, 1.0, None) == L.E_INVALID


def bench_lib():
    """libpdfp_bench.so: the benchmark's gather-ceiling probe, outside the solver library."""
    lib = C.CDLL(os.path.join(ROOT, "pdfp_b200", "lib", "libpdfp_bench.so"))
    lib.pdfp_measure_gather_rate.argtypes = [C.c_int64, C.c_int32, C.c_int32, C.POINTER(C.c_double)]
    lib.pdfp_bench_last_error.restype = C.c_char_p
    return lib


def test_gather_probe_lives_outside_the_solver_library():
    assert not hasattr(C.CDLL(L.LIB_PATH), "pdfp_measure_gather_rate")
    text = open(os.path.join(ROOT, "include", "pdfp_bench.h")).read()
    syms = set(re.findall(r"PDFP_API\s+[\w\s\*]+?\b(pdfp_\w+)\s*\(", text))
    lib = bench_lib()
    assert syms == {"pdfp_measure_gather_rate", "pdfp_bench_last_error"}
    for s in syms:
        assert hasattr(lib, s), s
    assert lib.pdfp_measure_gather_rate(1024, 100, 1, None) == L.E_INVALID
    assert b"null output" in lib.pdfp_bench_last_error()


@pytest.mark.gpu
def test_gather_rate_probe_reports_a_plausible_rate():
    lib = bench_lib()
    r = C.c_double()
    assert lib.pdfp_measure_gather_rate(4_000_000, 1_000_000, 3, C.byref(r)) == L.OK
    assert 1e10 < r.value < 1e13  # gathers per second
    assert lib.pdfp_measure_gather_rate(1023, 100, 1, C.byref(r)) == L.E_INVALID
