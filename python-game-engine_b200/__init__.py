"""B200-native (sm_100a) smoke-simulation step with the reference simulator's interface.

Drop-in for the src/cfd smoke path of LCEBurton/python-game-engine: the same
operator/solver registries (backend "cuda"), solver parameter dataclasses, config
dataclasses and a ``SmokeSimulation2D`` whose fields are torch CUDA tensors. The
compute path is the CUDA library ``lib/libsmoke_b200.so`` (C ABI:
include/smoke_b200.h); there is no CPU fallback.

The package directory name is not a Python identifier; import it with
``importlib.import_module("python-game-engine_b200")``.
"""
from . import _lib, adjoint, batch, profiling, scenes
from .config import Backend, GridConfig, OperatorBackendConfig, PressureSolverConfig, SimulationConfig
from .operators import OPEN_BOX, RING_BOX, AnalyticMask, register_operators
from .params import (DEFAULT_SOLVER_PARAMS, SOLVER_PARAM_TYPES, GaussSeidelParams, GeometricMultigridParams,
                     JacobiParams, MultigridParams, SORParams, SORToleranceParams)
from .registry import OPERATOR_REGISTRY, SOLVER_REGISTRY, get_operator, get_solver, register_operator, register_solver
from .simulation import Emitter2D, FieldReadback, NullProfileSession, PlumeSource, SmokeSimulation2D
from .solvers import (GeometricMultigridSolver, MultigridSolver, SORToleranceSolver, calculate_alpha,
                      calculate_optimal_omega, calculate_reciprocal_beta, register_solvers, solve_pressure)
from ._lib import NotConverged, SmokeCudaError
from .profiling import ProfileConfig, ProfileSession

register_operators()
register_solvers()

__all__ = [
    "Backend", "GridConfig", "OperatorBackendConfig", "PressureSolverConfig", "SimulationConfig",
    "OPEN_BOX", "RING_BOX", "AnalyticMask", "DEFAULT_SOLVER_PARAMS", "SOLVER_PARAM_TYPES", "GaussSeidelParams",
    "GeometricMultigridParams", "JacobiParams", "MultigridParams", "SORParams", "SORToleranceParams",
    "OPERATOR_REGISTRY", "SOLVER_REGISTRY", "get_operator", "get_solver", "register_operator", "register_solver",
    "Emitter2D", "FieldReadback", "NullProfileSession", "PlumeSource", "SmokeSimulation2D", "GeometricMultigridSolver",
    "MultigridSolver", "SORToleranceSolver", "calculate_alpha", "calculate_optimal_omega",
    "calculate_reciprocal_beta", "solve_pressure", "NotConverged", "SmokeCudaError", "ProfileConfig",
    "ProfileSession",
]
