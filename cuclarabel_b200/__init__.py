"""cuclarabel_b200 -- B200 (sm_100a) implementation of the Clarabel GPU
interior-point hot path (cone kernels, KKT refresh, batched LDL^T, residual
and variable updates, device-resident IPM driver) behind Clarabel's
Solver/solve! API.  See include/clgpu.h for the C ABI."""
from .api import (BatchSolver, DefaultSolution, ExponentialConeT,  # noqa: F401
                  NonnegativeConeT, PowerConeT, PSDTriangleConeT, SecondOrderConeT,
                  Settings, Solver, SolverStatus, SupportedCone, ZeroConeT,
                  cones_from_dict)
from .json_io import read_from_file, write_to_file  # noqa: F401

__all__ = ["BatchSolver", "DefaultSolution", "ExponentialConeT", "NonnegativeConeT",
           "PowerConeT", "PSDTriangleConeT", "SecondOrderConeT", "Settings", "Solver",
           "SolverStatus", "SupportedCone", "ZeroConeT", "cones_from_dict", "read_from_file",
           "write_to_file"]
