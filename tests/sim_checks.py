"""Checks shared by the multi-step scene tests.

recording(method): the CUDA solver `method` registered once more (backend "cuda") under a
test name, recording the norm of the divergence it is handed, i.e. the pre-projection
divergence of the substep.

check_divergence_bound(sim, div_before, tol): after a substep whose solve reached relative
residual tol, the post-projection divergence on cells two or more cells from the wall ring
equals r / alpha (r the solve's residual, alpha = -h^2 rho / dt; the projection subtracts
exactly the discrete gradient the residual's Laplacian is built from), so its norm there is at
most tol * ||divergence before the solve|| plus the rounding of the projected faces
(8 eps |u|max / h per cell).
"""
import numpy as np
import torch

from conftest import package

sg = package()
_RECORDED = {}


def recording(method):
    """The CUDA solver `method` registered once more under a test name that first records the
    norm of the divergence it is handed (the pre-projection divergence)."""
    name = f"test_recorded_{method}"
    if name not in _RECORDED:
        inner = sg.get_solver(method, "cuda")
        norms = []

        def fn(pressure, divergence, *args, **kw):
            norms.append(float(divergence.double().norm()))
            inner(pressure, divergence, *args, **kw)

        sg.register_solver(name, "cuda", fn)
        _RECORDED[name] = norms
    return name, _RECORDED[name]


def check_divergence_bound(sim, div_before, tol):
    """||div after projection|| on cells >= 2 from the ring <= tol ||div before|| + rounding."""
    d = sim.divergence.double()[2:-2, 2:-2]
    eps = 6e-8 if sim.divergence.dtype == torch.float32 else 1.2e-16
    vmax = max(float(sim.velocity_u.abs().max()), float(sim.velocity_v.abs().max()))
    rounding = 8 * eps * vmax / sim.cell_size * np.sqrt(d.numel())
    got = float(d.norm())
    assert got <= tol * div_before * 1.001 + rounding, (got, tol * div_before, rounding)
    return got
