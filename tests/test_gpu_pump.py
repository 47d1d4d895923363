"""The full pump with the GPU solvers (test/runtests.jl:73-95 on the GPU path).

* every example model: a feasible point is found (`is_feasible` at 1e-6) and
  the objective equals c'x + c0, in both arithmetic forms;
* p0201 with the FP64 form reproduces the published log's first iteration
  (README.md:36-48): root LP after 600 iterations, first rounding violating by
  9, iteration 1 with distance 8.08613, violation 1, 600 PDHG iterations.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from pdfp_b200.milp import is_feasible
from pdfp_b200.pump import feasibility_pump

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["p0201", "gen-ip054", "pk1", "markshare2"])
def test_pump_finds_feasible(examples, name, precision):
    m = examples[name]
    r = feasibility_pump(m, time_limit=120.0, precision=precision)
    assert r.found, (name, precision)
    assert is_feasible(m, r.x)
    assert r.objective == pytest.approx(float(np.dot(m.c, r.x) + m.c0))


def test_p0201_first_iteration_matches_published_log(examples, capsys):
    log = json.load(open(os.path.join(GOLDEN, "reference_log.json")))["p0201"]
    feasibility_pump(examples["p0201"], time_limit=120.0, verbose=True, precision="fp64")
    out = capsys.readouterr().out.splitlines()
    assert any(l.startswith("root LP     OPTIMAL after 600 iterations") for l in out)
    assert any("first rounding violates by 9)" in l for l in out)
    first = [l for l in out if l.strip().startswith("1 ")][0].split()
    it1 = log["iterations"][0]
    assert float(first[1]) == pytest.approx(it1["distance"], rel=1e-5)
    assert int(first[2]) == it1["violation"] and int(first[3]) == it1["pdhg"]
    assert any(l.startswith("device      NVIDIA") for l in out)


@pytest.mark.parametrize("name", ["pk1", "gen-ip054"])
def test_pump_fp64_takes_the_oracle_pumps_steps(examples, oracle, name):
    """With the deterministic rounding policy the FP64 GPU pump and the pump on the
    oracle's solvers take the same steps and return the same point.

    p0201 is left out: many coordinates of its root-LP point are equal in exact
    arithmetic, so the rounder's order among them follows last-bit differences
    between the GPU's and the oracle's FP64 sums (the two root-LP points differ by
    1e-15; their first roundings differ in 30 coordinates with the same violation
    and distance), and from the second pump iteration on the trajectories part.
    Its first iteration still matches the published log (tested above)."""
    m = examples[name]
    r_o = feasibility_pump(m, time_limit=120.0, solvers=oracle.OracleSolvers(), seed=3,
                           batch_policy="always")
    r_g = feasibility_pump(m, time_limit=120.0, precision="fp64", seed=3, batch_policy="always")
    assert (r_g.found, r_g.iterations, r_g.perturbations) == (r_o.found, r_o.iterations,
                                                             r_o.perturbations)
    assert r_g.pdhg_iterations == r_o.pdhg_iterations
    # integer columns are rounded: identical; continuous ones come from the
    # projection: equal to the FP64 last bits
    I = m.int_idx
    assert np.array_equal(r_g.x[I], r_o.x[I])
    assert np.allclose(r_g.x, r_o.x, rtol=1e-9, atol=1e-9)
