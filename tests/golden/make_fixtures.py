"""Generate the golden fixtures under tests/golden/ from the reference checkout.

Run in a container where the reference is mounted (it is not on the GPU box):

    python tests/golden/make_fixtures.py <path of the reference checkout>

It converts the reference's four example models (examples/*.mps.gz, the
MIPLIB 2017 instances the reference's own tests use, test/runtests.jl:30-79)
into compact .npz files with this package's MPS reader, so that GPU tests can
load them without the reference tree, and writes reference_log.json with the
published p0201 log lines (README.md:36-48) that pin the oracle.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from pdfp_b200.milp import read_mps  # noqa: E402

NAMES = ["p0201", "pk1", "gen-ip054", "markshare2"]


def main(ref_root: str) -> None:
    for name in NAMES:
        m = read_mps(os.path.join(ref_root, "examples", f"{name}.mps.gz"))
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            indptr=m.A.indptr.astype(np.int32), indices=m.A.indices.astype(np.int32),
            data=m.A.data, shape=np.array(m.A.shape), b=m.b,
            is_eq=np.array([s == "eq" for s in m.row_sense]), l=m.l, u=m.u,
            int_idx=m.int_idx, c=m.c, c0=np.array(m.c0), name=np.array(m.name))
    # The p0201 run printed in the reference README (README.md:36-48, H100).
    log = {
        "p0201": {
            "rows": 133, "columns": 201, "integer": 201, "continuous": 0, "nonzeros": 1923,
            "root_lp": {"status": "OPTIMAL", "iterations": 600, "tolerance": 1e-2},
            "first_rounding_violation": 9,
            "schedule": "all",
            "iterations": [
                {"iter": 1, "distance": 8.08613, "violation": 1, "pdhg": 600, "gap": 1.00e-02, "action": "round"},
                {"iter": 2, "distance": 1.23237, "violation": 5, "pdhg": 400, "gap": 9.80e-03, "action": "round"},
                {"iter": 3, "distance": 0.116077, "violation": 5, "pdhg": 200, "gap": 9.60e-03, "action": "flip"},
                {"iter": 4, "distance": 6.22643, "violation": 39, "pdhg": 400, "gap": 9.41e-03, "action": "cycle"},
                {"iter": 5, "distance": 32.6474, "violation": 83, "pdhg": 400, "gap": 9.22e-03, "action": "round"},
            ],
            "objective": 11020,
        },
        "pk1": {"continuous": 31},
    }
    with open(os.path.join(HERE, "reference_log.json"), "w") as fh:
        json.dump(log, fh, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_fixtures.py <path of the reference checkout>")
    main(sys.argv[1])
