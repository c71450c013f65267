"""B200-native PMG (Galerkin multigrid) solver of the linearized
Poisson-Boltzmann equation: a drop-in for the reference's pmgc kernels and
its PBE_linear_problem class, computing in libpmg_b200.so (CUDA, sm_100a).
"""
from . import _lib  # noqa: F401  (raises if the CUDA library is not built)
from .molecule import (DEFAULT_PHYSICS, REFERENCE_PHYSICS, WORKLOADS,
                       Workload, batch_workloads, level_n)
from .problem import PBELinearProblem, SolveResult, kappa, setup_fine

__all__ = [
    "PBELinearProblem", "SolveResult", "Workload", "WORKLOADS",
    "batch_workloads", "level_n", "setup_fine", "kappa", "DEFAULT_PHYSICS",
    "REFERENCE_PHYSICS",
]
