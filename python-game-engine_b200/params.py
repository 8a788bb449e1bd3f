"""Pressure-solver parameter dataclasses.

The first four keep the field names, defaults and string helpers of the reference
(src/cfd/solvers/params.py:5-76) so a reference config selects the same solver
behaviour. The last two configure solvers the reference does not have: a
tolerance-driven red-black SOR and the convergent geometric multigrid (optionally
mixed precision); they are registered under new method names so the reference's
own parameter types keep their meaning.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Union


@dataclass
class JacobiParams:
    iterations: int = 40

    def string(self):
        return f"JacobiParams_iters_{self.iterations}"

    def to_fn(self):
        return f"i_{self.iterations}"


@dataclass
class GaussSeidelParams:
    iterations: int = 40

    def string(self):
        return f"GaussSeidelParams_iters_{self.iterations}"

    def to_fn(self):
        return f"i_{self.iterations}"


@dataclass
class SORParams:
    iterations: int = 40
    omega: float = 0.0  # 0.0 selects min(2 / (1 + sin(pi / n)), 1.95)

    def string(self):
        return f"SORParams_iters_{self.iterations}_omega_{self.omega}"

    def to_fn(self):
        return f"i_{self.iterations}_o_{self.omega}"


@dataclass
class MultigridParams:
    smoother_type: str = "jacobi"
    smoother_backend: str = "cuda"
    num_levels: int = 4
    v_cycles: int = 2
    smoother_iterations: int = 2
    coarsest_iterations: int = 30
    rebuild_masks: bool = False

    def string(self):
        return (f"MultigridParams_smoother_{self.smoother_type}_{self.smoother_backend}"
                f"_vcycles_{self.v_cycles}_levels_{self.num_levels}"
                f"_smoother_iters_{self.smoother_iterations}_coarsest_{self.coarsest_iterations}")

    def to_fn(self):
        return (f"st_{self.smoother_type}_{self.smoother_backend}_v{self.v_cycles}_l{self.num_levels}"
                f"_si{self.smoother_iterations}_ci{self.coarsest_iterations}")


@dataclass
class SORToleranceParams:
    """Red-black SOR run until ||r|| / ||r(0)|| <= tol (checked every check_every sweeps).
    precision: "native" (the field's dtype) or "mixed" (float32 sweeps in float64 refinement)."""
    omega: float = 1.9
    tol: float = 1e-6
    max_iterations: int = 200000
    check_every: int = 100
    precision: str = "native"

    def string(self):
        suffix = "" if self.precision == "native" else f"_{self.precision}"
        return f"SORToleranceParams_omega_{self.omega}_tol_{self.tol}{suffix}"

    def to_fn(self):
        suffix = "" if self.precision == "native" else f"_{self.precision}"
        return f"o_{self.omega}_t_{self.tol}{suffix}"


@dataclass
class GeometricMultigridParams:
    """Convergent geometric multigrid (see the C ABI: sg_gmg_*)."""
    tol: float = 1e-6
    max_cycles: int = 50
    cycle: str = "V"            # "V" or "W"
    pre_sweeps: int = 2
    post_sweeps: int = 2
    omega: float = 1.3          # red-black Gauss-Seidel over-relaxation (1.0 = plain GS)
    coarsest: int = 8           # coarsen until both extents <= coarsest
    precision: str = "fp64"     # "fp32" | "fp64" | "mixed" (FP32 cycles in FP64 refinement)
    check_every: int = 1        # host convergence check interval (cycles)
    fixed_cycles: int = 0       # > 0: run exactly this many cycles without host checks
    rebuild_masks: bool = False
    remove_mean: bool = False   # subtract the fluid mean of the rhs (rounding of sum(div)) before solving
    inner_cycles: int = 1       # >= 2: classical refinement, that many FP32 cycles per FP64 residual

    def string(self):
        return (f"GeometricMultigridParams_{self.cycle}{self.pre_sweeps}{self.post_sweeps}_w{self.omega}"
                f"_tol_{self.tol}_{self.precision}")

    def to_fn(self):
        return f"{self.cycle}{self.pre_sweeps}{self.post_sweeps}_t{self.tol}_{self.precision}"


SolverParams = Union[JacobiParams, GaussSeidelParams, SORParams, MultigridParams, SORToleranceParams,
                     GeometricMultigridParams]

DEFAULT_SOLVER_PARAMS: dict[str, SolverParams] = {
    "jacobi": JacobiParams(),
    "gauss_seidel": GaussSeidelParams(),
    "rb_sor_gauss_seidel": SORParams(),
    "multigrid": MultigridParams(),
    "rb_sor_tolerance": SORToleranceParams(),
    "geometric_multigrid": GeometricMultigridParams(),
}

SOLVER_PARAM_TYPES: dict[str, type] = {
    "jacobi": JacobiParams,
    "gauss_seidel": GaussSeidelParams,
    "rb_sor_gauss_seidel": SORParams,
    "multigrid": MultigridParams,
    "rb_sor_tolerance": SORToleranceParams,
    "geometric_multigrid": GeometricMultigridParams,
}
