"""The reference-side binding a maintainer would add to the reference (as
src/cfd/backends/cuda/registrations.py, called next to register_solvers()): the CUDA solvers
and operators registered into the reference's own registries under backend "cuda", working on
the reference's numpy arrays. The code below is the integration guide's snippet unchanged;
tests/test_reference_adapter.py imports it."""
# src/cfd/backends/cuda/registrations.py  (reference side)
import importlib
import numpy as np
import torch

from cfd.operators.registry import register_operator
from cfd.solvers.registry import register_solver

sg = importlib.import_module("python-game-engine_b200")  # repo root on sys.path


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _numpy_solver(method):
    fn = sg.get_solver(method, "cuda")

    def solve(pressure, divergence, face_mask_u, face_mask_v, fluid_density, cell_size, dt, **kw):
        kw.pop("profiler", None)
        if kw.get("smoother_backend") == "numba":
            kw["smoother_backend"] = "cuda"
        p = _dev(pressure)
        fn(p, _dev(divergence), _dev(face_mask_u), _dev(face_mask_v), fluid_density, cell_size, dt, **kw)
        pressure[...] = p.cpu().numpy()
    return solve


def _numpy_operator(name, outputs):
    fn = sg.get_operator(name, "cuda")

    def op(*args):
        dev = [_dev(a) if isinstance(a, np.ndarray) else a for a in args]
        fn(*dev)
        for k in outputs:                       # positional indices written in place
            args[k][...] = dev[k].cpu().numpy()
    return op


def register_cuda_backend():
    for m in ("jacobi", "gauss_seidel", "rb_sor_gauss_seidel", "multigrid",
              "rb_sor_tolerance", "geometric_multigrid"):
        register_solver(m, "cuda", _numpy_solver(m))
    for name, outs in {"advection_scalar": (1,), "advection_velocity_u": (1,),
                       "advection_velocity_v": (1,), "compute_divergence": (2,),
                       "apply_forces": (0,), "cool_temperature": (0,),
                       "apply_pressure_gradient": (0, 1), "enforce_boundary_conditions": (0, 1),
                       "compute_residual": (7,)}.items():
        register_operator(name, "cuda", _numpy_operator(name, outs))
