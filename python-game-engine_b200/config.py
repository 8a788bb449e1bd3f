"""Simulation configuration with the reference's field names and JSON shape.

Mirrors src/cfd/common/config.py:7-163 (Backend, GridConfig, OperatorBackendConfig,
PressureSolverConfig, SimulationConfig with to_dict / from_dict / JSON / validation)
so configs written for the reference load unchanged; the defaults select the CUDA
backend. ``SmokeSimulation2D`` also accepts the reference's own config objects
(duck-typed on the same attributes).
"""
from __future__ import annotations

import json
from dataclasses import dataclass, field
from enum import Enum

from .params import SOLVER_PARAM_TYPES, JacobiParams, SolverParams


class Backend(str, Enum):
    NUMBA = "numba"
    CPP = "cpp"
    CUDA = "cuda"

    def __str__(self):
        return self.value


@dataclass
class GridConfig:
    size: tuple[int, int]  # (width, height), as the reference (simulation.py:45)
    cell_size: float


@dataclass
class OperatorBackendConfig:
    advection: Backend = Backend.CUDA
    boundaries: Backend = Backend.CUDA
    divergence: Backend = Backend.CUDA
    forces: Backend = Backend.CUDA
    pressure_gradient: Backend = Backend.CUDA
    residual: Backend = Backend.CUDA


@dataclass
class PressureSolverConfig:
    method: str = "jacobi"
    backend: Backend = Backend.CUDA
    params: SolverParams = field(default_factory=JacobiParams)


@dataclass
class SimulationConfig:
    grid: GridConfig
    pressure_solver: PressureSolverConfig = field(default_factory=PressureSolverConfig)
    operators: OperatorBackendConfig = field(default_factory=OperatorBackendConfig)
    debug: bool = False

    def to_dict(self) -> dict:
        from dataclasses import asdict
        return {
            "grid": {"size": list(self.grid.size), "cell_size": self.grid.cell_size},
            "pressure_solver": {
                "method": self.pressure_solver.method,
                "backend": Backend(self.pressure_solver.backend).value,
                "params": asdict(self.pressure_solver.params),
            },
            "operators": {name: Backend(b).value for name, b in vars(self.operators).items()},
        }

    def to_json(self, path: str) -> None:
        with open(path, "w") as f:
            json.dump(self.to_dict(), f, indent=4)

    @classmethod
    def from_dict(cls, data: dict) -> "SimulationConfig":
        g = data.get("grid", {})
        grid = GridConfig(size=tuple(g.get("size", (16, 16))), cell_size=g.get("cell_size", 1.0))
        s = data.get("pressure_solver", {})
        method = s.get("method", "jacobi")
        ptype = SOLVER_PARAM_TYPES.get(method, JacobiParams)
        return cls(
            grid=grid,
            pressure_solver=PressureSolverConfig(method=method, backend=Backend(s.get("backend", "cuda")),
                                                 params=ptype(**s.get("params", {}))),
            operators=OperatorBackendConfig(**{k: Backend(v) for k, v in data.get("operators", {}).items()}),
        )

    @classmethod
    def from_json(cls, path: str) -> "SimulationConfig":
        with open(path) as f:
            return cls.from_dict(json.load(f))

    def validate_config(self) -> None:
        size = self.grid.size
        if not (isinstance(size, tuple) and len(size) == 2):
            raise ValueError("Grid size must be a tuple of two integers.")
        if not all(isinstance(d, int) and d > 0 for d in size):
            raise ValueError("Grid dimensions must be positive integers.")
        if not isinstance(self.grid.cell_size, (int, float)) or self.grid.cell_size <= 0:
            raise ValueError("Cell size must be a positive number.")
        if self.pressure_solver.method not in SOLVER_PARAM_TYPES:
            raise ValueError(f"Unsupported pressure solver method: {self.pressure_solver.method}")
        if not isinstance(self.pressure_solver.backend, Backend):
            raise ValueError(f"Unsupported pressure solver backend: {self.pressure_solver.backend}")
        ptype = SOLVER_PARAM_TYPES[self.pressure_solver.method]
        if not isinstance(self.pressure_solver.params, ptype):
            raise ValueError(f"Pressure solver params must be of type {ptype.__name__} for method "
                             f"{self.pressure_solver.method}")
        if not isinstance(self.operators, OperatorBackendConfig):
            raise ValueError("Operators must be an instance of OperatorBackendConfig.")
        if not all(isinstance(getattr(self.operators, op), Backend) for op in vars(self.operators)):
            raise ValueError("All operator backends must be instances of Backend.")
        if not isinstance(self.debug, bool):
            raise ValueError("Debug flag must be a boolean.")
