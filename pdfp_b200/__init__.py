"""pdfp_b200 -- the PDFP feasibility pump's projector and root-LP solver on B200.

The pump's interface (src/pump.jl, src/milp.jl of MIT-Lu-Lab/PDFP):

    from pdfp_b200 import read_mps, feasibility_pump, is_feasible
    milp = read_mps("p0201.mps.gz")
    r = feasibility_pump(milp, time_limit=600.0, seed=1, verbose=True)

The projector, root LP and preconditioner run in libpdfp_b200.so (see
pdfp_b200.gpu); rounding and propagation run on the CPU.
"""
from .milp import MILP, is_feasible, max_violation, num_constraints, num_continuous, num_variables, read_mps, write_solution
from .params import RestartParameters, SolverParameters
from .pump import PumpResult, TrajectoryResult, feasibility_pump, feasibility_pump_batched

__all__ = ["MILP", "read_mps", "max_violation", "is_feasible", "write_solution", "num_variables",
           "num_constraints", "num_continuous", "feasibility_pump", "PumpResult",
           "feasibility_pump_batched", "TrajectoryResult",
           "SolverParameters", "RestartParameters"]
