"""Seeded synthetic scenes for the benchmark configurations.

Every scene is a closed box on the unit square: an H x W MAC grid with cell size
1/max(H, W), dt = 0.5 * cell size, walls as the reference simulator builds them
(outer faces closed, 1-cell solid ring enforced after projection). Density and
velocity start at zero. Sources are overwriting discs (PlumeSource); positions and
radii are in cells. Buoyancy "c * density" is the reference's density force with
gravity = -c (forces.py:44: force = -density_coefficient * d * gravity).

  plume_128       128^2, one source r=8 at (0.5, 0.1) of the domain, density 1 and v 1
                  each step plus uniform +-0.05 velocity noise inside the source;
                  Jacobi x100, float64, 200 steps.
  plume_512       512^2, same plume with r=32 (variant 0) or a seeded random inflow
                  x on the bottom edge (variants 1, 2); 500 steps; red-black SOR
                  omega=1.9 or multigrid V(2,2), both to 1e-6.
  mixed_2048      2048^2, four seeded sources, r ~ U[16, 64] cells, inflow speed
                  ~ U[0.5, 1.5], zero initial velocity; 200 steps; multigrid to 1e-8
                  (float32 state + mixed-precision solve, or float64 throughout).
  batch_256       256 scenes, H = W ~ U{64, 96, 128, 192, 256}, seeded source position,
                  r = 4-16 % of W, buoyancy ~ U[0.5, 2.0]; float32 multigrid to 1e-6.
  inverse_256     256^2, 64 steps, one seeded source; control forces (see adjoint).

Seeds: plume_128 0; plume_512 variants 1, 2 (variant 0 uses no random draw);
mixed_2048 3; batch_256 1000 + k for scene k; inverse_256 7.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Scene:
    name: str
    H: int
    W: int
    steps: int
    gravity: float = -1.0
    plumes: list = field(default_factory=list)  # rows (cx, cy, r, density, v, noise_amp) in cells
    seed: int = 0

    @property
    def cell_size(self) -> float:
        return 1.0 / max(self.H, self.W)

    @property
    def dt(self) -> float:
        return 0.5 * self.cell_size

    @property
    def cells(self) -> int:
        return self.H * self.W


def plume_128(steps: int = 200) -> Scene:
    n = 128
    return Scene("plume_128", n, n, steps, -1.0, [[0.5 * n, 0.1 * n, 8.0, 1.0, 1.0, 0.05]], seed=0)


def plume_512(variant: int = 0, steps: int = 500) -> Scene:
    n = 512
    if variant == 0:
        x = 0.5 * n
    else:
        rng = np.random.default_rng(variant)
        x = float(rng.uniform(0.1, 0.9)) * n
    return Scene(f"plume_512_v{variant}", n, n, steps, -1.0, [[x, 0.1 * n, 32.0, 1.0, 1.0, 0.05]], seed=variant)


def mixed_2048(steps: int = 200) -> Scene:
    n = 2048
    rng = np.random.default_rng(3)
    plumes = []
    for _ in range(4):
        r = float(rng.uniform(16.0, 64.0))
        speed = float(rng.uniform(0.5, 1.5))
        x = float(rng.uniform(0.15, 0.85)) * n
        y = float(rng.uniform(0.05, 0.2)) * n
        plumes.append([x, y, r, 1.0, speed, 0.0])
    return Scene("mixed_2048", n, n, steps, -1.0, plumes, seed=3)


BATCH_SIZES = (64, 96, 128, 192, 256)


def batch_scene(k: int, steps: int = 300) -> Scene:
    rng = np.random.default_rng(1000 + k)
    n = int(rng.choice(BATCH_SIZES))
    r = float(rng.uniform(0.04, 0.16)) * n
    x = float(rng.uniform(0.2, 0.8)) * n
    y = float(rng.uniform(0.08, 0.25)) * n
    c = float(rng.uniform(0.5, 2.0))
    return Scene(f"batch_{k}", n, n, steps, -c, [[x, y, r, 1.0, 1.0, 0.0]], seed=1000 + k)


def batch_256(count: int = 256, steps: int = 300) -> list:
    return [batch_scene(k, steps) for k in range(count)]


def inverse_256(steps: int = 64) -> Scene:
    n = 256
    rng = np.random.default_rng(7)
    x = float(rng.uniform(0.3, 0.7)) * n
    return Scene("inverse_256", n, n, steps, -1.0, [[x, 0.1 * n, 12.0, 1.0, 1.0, 0.0]], seed=7)


def target_blob(n: int = 256, sigma: float = 20.0, seed: int = 7):
    """Gaussian blob target for the inverse problem, centred in the upper half."""
    rng = np.random.default_rng(seed + 1)
    cx = float(rng.uniform(0.3, 0.7)) * n
    cy = float(rng.uniform(0.55, 0.85)) * n
    j, i = np.indices((n, n))
    return np.exp(-((i + 0.5 - cx) ** 2 + (j + 0.5 - cy) ** 2) / (2.0 * sigma * sigma))


def make_sim(scene: Scene, method: str = "jacobi", params=None, dtype=None, device=None):
    """A SmokeSimulation2D set up for ``scene`` (sim.dt = scene dt, gravity, plume table)."""
    import torch

    from .config import GridConfig, PressureSolverConfig, SimulationConfig
    from .params import DEFAULT_SOLVER_PARAMS
    from .simulation import PlumeSource, SmokeSimulation2D

    cfg = SimulationConfig(grid=GridConfig(size=(scene.W, scene.H), cell_size=scene.cell_size),
                           pressure_solver=PressureSolverConfig(method=method,
                                                                params=params or DEFAULT_SOLVER_PARAMS[method]))
    sim = SmokeSimulation2D(cfg, device=device, dtype=dtype or torch.float32, seed=scene.seed)
    sim.dt = scene.dt
    sim.gravity = scene.gravity
    sim.set_plumes([PlumeSource(*row) for row in scene.plumes])
    return sim
