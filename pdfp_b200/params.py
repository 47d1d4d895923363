"""Solver parameters shared by the projector and the root-LP solver.

Mirror of ``RestartParameters`` / ``SolverParameters`` (src/pdlp.jl:10-31); the
defaults are the reference's (cuPDLPx's).  ``precision`` is this library's own
knob: ``"fp64"`` is the plain FP64 form, ``"mixed"`` runs the iterates and the
sparse products in FP32 with FP64 reductions, restart logic and polish.
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace

STATUS_NAMES = {0: "UNSPECIFIED", 1: "OPTIMAL", 2: "ITERATION_LIMIT", 3: "TIME_LIMIT",
                4: "PRIMAL_INFEASIBLE", 5: "DUAL_INFEASIBLE"}


@dataclass(frozen=True)
class RestartParameters:
    artificial_restart_threshold: float = 0.36
    sufficient_reduction_for_restart: float = 0.2
    necessary_reduction_for_restart: float = 0.5
    k_p: float = 0.99
    k_i: float = 0.01
    k_d: float = 0.0
    i_smooth: float = 0.3


@dataclass(frozen=True)
class SolverParameters:
    eps_optimal_relative: float = 1e-4
    eps_feasible_relative: float = 1e-4
    iteration_limit: int = 100_000
    time_limit: float = 3600.0
    termination_evaluation_frequency: int = 200
    reflection_coefficient: float = 1.0
    sv_max_iterations: int = 5000
    sv_tolerance: float = 1e-4
    restart: RestartParameters = field(default_factory=RestartParameters)

    def with_(self, **kw) -> "SolverParameters":
        return replace(self, **kw)

    def flat(self) -> dict:
        """The flat field set of the C ``pdfp_params`` struct."""
        r = self.restart
        return dict(
            eps_optimal_relative=self.eps_optimal_relative,
            eps_feasible_relative=self.eps_feasible_relative,
            iteration_limit=int(self.iteration_limit),
            time_limit=float(self.time_limit),
            termination_evaluation_frequency=int(self.termination_evaluation_frequency),
            sv_max_iterations=int(self.sv_max_iterations),
            reflection_coefficient=self.reflection_coefficient,
            sv_tolerance=self.sv_tolerance,
            artificial_restart_threshold=r.artificial_restart_threshold,
            sufficient_reduction_for_restart=r.sufficient_reduction_for_restart,
            necessary_reduction_for_restart=r.necessary_reduction_for_restart,
            k_p=r.k_p, k_i=r.k_i, k_d=r.k_d, i_smooth=r.i_smooth,
        )
