"""ctypes binding of libsmoke_b200.so (declarations: include/smoke_b200.h).

The library is the only compute path: if it is missing, or no CUDA device is
present, calls raise instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
# SG_LIBRARY_VARIANT=bounds selects the bounds-check build (index checks in the tiled kernels)
LIB_PATH = os.path.join(_HERE, "lib", "libsmoke_b200_bc.so" if os.environ.get("SG_LIBRARY_VARIANT") == "bounds"
                        else "libsmoke_b200.so")

SG_F32, SG_F64 = 0, 1
SG_MASK_PLANES, SG_MASK_OPEN, SG_MASK_RING, SG_MASK_NONE = 0, 1, 2, 3
SG_GMG_FP32, SG_GMG_FP64, SG_GMG_MIXED = 0, 1, 2
SG_OK, SG_ERR_ARG, SG_ERR_DTYPE, SG_ERR_CUDA, SG_ERR_NOT_CONVERGED, SG_ERR_NONFINITE = 0, 1, 2, 3, 4, 5
SG_ERR_WORKSPACE, SG_ERR_CAPACITY = 6, 7

P = ctypes.c_void_p
I64 = ctypes.c_int64
I = ctypes.c_int
D = ctypes.c_double
U64 = ctypes.c_uint64
PD = ctypes.POINTER(ctypes.c_double)
PI = ctypes.POINTER(ctypes.c_int)

# name -> argtypes (all return int status unless listed in _RESTYPE)
SIGNATURES = {
    "sg_advect_scalar": [I, I64, I64, P, I64, P, I64, P, I64, I64, I64, P, I64, I64, I64, I, P, I64, D, D, D, P],
    "sg_advect_velocity_u": [I, I64, I64, P, I64, P, I64, P, I64, I64, I64, I, P, I64, D, D, P],
    "sg_advect_velocity_v": [I, I64, I64, P, I64, P, I64, P, I64, I64, I64, I, P, I64, D, D, P],
    "sg_advect_velocity": [I, I64, I64, P, I64, P, I64, P, I64, P, I64, I, P, I64, P, I64, D, D, P],
    "sg_advect_velocity_f32": [I64, I64, P, I64, P, I64, P, I64, P, I64, I, P, I64, P, I64, D, D, P],
    "sg_advect_scalar_f32": [I64, I64, P, I64, P, I64, P, I64, P, I64, I, P, I64, D, D, D, P],
    "sg_apply_forces": [I, I64, I64, P, I64, P, I64, P, I64, D, D, D, D, D, I, P],
    "sg_cool_temperature": [I, I64, I64, P, I64, D, D, D, P],
    "sg_compute_divergence": [I, I64, I64, P, I64, P, I64, P, I64, I, P, I64, P, I64, D, P],
    "sg_compute_residual": [I, I64, I64, P, I64, P, I64, I, P, I64, P, I64, P, I64, D, D, P, I64, P, P],
    "sg_apply_pressure_gradient": [I, I64, I64, P, I64, P, I64, P, I64, I, P, I64, P, I64, D, D, D, P],
    "sg_enforce_boundary_conditions": [I, I64, I64, P, I64, P, I64, I, P, I64, P],
    "sg_project": [I, I64, I64, P, I64, P, I64, P, I64, I, P, I64, P, I64, I, P, I64, D, D, D, P],
    "sg_emit_scalar": [I, I64, I64, P, I64, D, D, D, D, D, I, P],
    "sg_plume_sources": [I, I64, I64, P, I64, P, I64, P, I64, I, P, U64, I64, P],
    "sg_build_masks": [I64, I64, P, I64, P, I64, P, I64, P, I64, P],
    "sg_jacobi_solve": [I, I64, I64, P, I64, P, I64, I, P, I64, P, I64, D, D, I, P, P],
    "sg_jacobi_solve_noalloc": [I, I64, I64, P, I64, P, I64, I, P, I64, P, I64, D, D, I, P],
    "sg_rbsor_solve": [I, I64, I64, P, I64, P, I64, I, P, I64, P, I64, D, D, D, I, P],
    "sg_gauss_seidel_solve": [I, I64, I64, P, I64, P, I64, I, P, I64, P, I64, D, D, I, P],
    "sg_rbsor_split_workspace_bytes": [I, I64, I64],
    "sg_rbsor_split_pack": [I, I64, I64, P, I64, I, P, I64, P],
    "sg_rbsor_split_unpack": [I, I64, I64, P, I64, P, I64, P],
    "sg_rbsor_split_sweeps": [I, I64, I64, P, I64, I, P, I64, P, I64, D, D, D, I64, I, P],
    "sg_rbsor_split_sumsq": [I, I64, I64, P, I64, I, P, I64, P, I64, D, D, I, P, P],
    "sg_rbsor_tol_solve": [I, I64, I64, P, I64, P, I64, I, P, I64, P, I64, D, D, D, D, I64, I64, I, P, I64,
                           ctypes.POINTER(ctypes.c_int64), PD, P],
    "sg_rbsor_mixed_workspace_bytes": [I64, I64],
    "sg_rbsor_mixed_solve": [I64, I64, P, I64, P, I64, I, P, I64, P, I64, D, D, D, D, I64, I64, I, P, I64,
                             ctypes.POINTER(ctypes.c_int64), PD, ctypes.POINTER(ctypes.c_int64), P],
    "sg_mg_restrict_average": [I, I64, I64, P, I64, I, P, I64, P, I64, I64, I64, D, P],
    "sg_mg_prolong": [I, I64, I64, P, I64, I64, I64, I, P, I64, P, I64, I, P],
    "sg_mg_coarsen_solid": [I64, I64, P, I64, P, I64, P],
    "sg_gmg_plan_create": [ctypes.POINTER(P), I64, I64, I, P, P, P, I, D, I, I, I, I],
    "sg_gmg_plan_destroy": [P],
    "sg_gmg_workspace_bytes": [P],
    "sg_gmg_num_levels": [P],
    "sg_gmg_bind": [P, P, P],
    "sg_gmg_solve_async": [P, P, I64, P, I64, I, D, D, I, P],
    "sg_gmg_solve_from_zero_async": [P, P, I64, P, I64, I, D, D, I, P],
    "sg_gmg_stats": [P, PI, PD, PI, ctypes.POINTER(ctypes.c_longlong), P],
    "sg_gmg_counters": [P, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                        ctypes.POINTER(ctypes.c_longlong), P],
    "sg_gmg_solve": [P, P, I64, P, I64, I, D, D, I, PI, PD, P],
    "sg_gmg_cycles_async": [P, P, I64, P, I64, I, D, I, PD, P],
    "sg_gmg_graph_nodes": [P, PI, PI],
    "sg_gmg_tail_start": [P],
    "sg_gmg_level_shape": [P, I, PI, PI],
    "sg_gmg_smooth_async": [P, I, I, P],
    "sg_gmg_fine_fused": [P],
    "sg_gmg_coarse_solve_kind": [P],
    "sg_gmg_set_post_events": [P, P, I],
    "sg_stage_copy": [I64, I64, P, I64, P, I64, P],
    "sg_gmg_relres_async": [P, P, P],
    "sg_project_metrics": [I, I64, I64, P, I64, P, I64, P, I64, P, I64, P, I64, I, P, I64, P, I64, P, I64, I, P, I64,
                           D, D, D, D, D, P, I64, P, I64, P],
    "sg_gmg_fine_kernel_async": [P, I, P, I64, P],
    "sg_apply_forces_f32": [I64, I64, P, I64, P, I64, P, I64, D, D, D, D, D, P],
    "sg_project_metrics_f32": [I64, I64, P, I64, P, I64, P, I64, P, I64, P, I64, I, P, I64, P, I64, P, I64, I, P,
                               I64, D, D, D, D, D, P, I64, P, I64, P],
    "sg_add_control": [I, I64, I64, P, I64, P, I64, P, I64, P, I64, D, P],
    "sg_adjoint_advect_scalar_workspace": [I, I64, I64, I],
    "sg_adjoint_advect_scalar": [I, I64, I64, P, I64, P, I64, P, I64, P, I64, I, P, I64, D, D, D, P, I64, P, I64, P,
                                 I64, I, P, I64, P],
    "sg_adjoint_advect_velocity": [I, I64, I64, P, I64, P, I64, P, I64, P, I64, I, P, I64, P, I64, D, D, P, I64, P,
                                   I64, P],
    "sg_adjoint_forces": [I, I64, I64, P, I64, P, I64, P, I64, P, I64, P, I64, D, D, D, P],
    "sg_adjoint_project": [I, I64, I64, P, I64, P, I64, P, I64, P, I64, P, I64, I, P, I64, P, I64, I, P, I64, D, D,
                           D, P],
    "sg_adjoint_divergence": [I, I64, I64, P, I64, P, I64, P, I64, I, P, I64, P, I64, D, P],
    "sg_batch_create": [P, I, P, P, P, D, I, U64],
    "sg_batch_destroy": [P],
    "sg_batch_workspace_bytes": [P],
    "sg_batch_bind": [P, P, I64, P],
    "sg_batch_configure": [P, I, I, I],
    "sg_batch_tile_shape": [I, PI, PI],
    "sg_batch_step": [P, I, P],
    "sg_batch_layout": [P, I, P, P, P, P],
    "sg_batch_current": [P],
    "sg_batch_loops": [P, P, P],
    "sg_batch_graph_nodes": [P, PI, PI],
    "sg_batch_stats": [P, P, P, P, P],
    "sg_batch_snapshot_bytes": [P],
    "sg_batch_autotune": [P, I, P, I64, P, PI, PI, PI, PD],
    "sg_gmg_set_remove_mean": [P, I],
    "sg_gmg_set_inner_cycles": [P, I],
    "sg_field_stats_workspace_bytes": [],
    "sg_field_stats": [I, I64, I64, P, I64, P, P, P],
    "sg_bounds_check_enabled": [],
    "sg_bounds_check": [ctypes.POINTER(ctypes.c_uint), PI, I],
    "sg_version": [],
    "sg_last_error": [],
    "sg_launch_count": [],
}
_RESTYPE = {
    "sg_version": ctypes.c_char_p,
    "sg_last_error": ctypes.c_char_p,
    "sg_gmg_plan_destroy": None,
    "sg_gmg_workspace_bytes": ctypes.c_int64,
    "sg_launch_count": ctypes.c_uint64,
    "sg_adjoint_advect_scalar_workspace": ctypes.c_int64,
    "sg_batch_destroy": None,
    "sg_batch_workspace_bytes": ctypes.c_int64,
    "sg_batch_snapshot_bytes": ctypes.c_int64,
    "sg_field_stats_workspace_bytes": ctypes.c_int64,
    "sg_rbsor_split_workspace_bytes": ctypes.c_int64,
    "sg_rbsor_mixed_workspace_bytes": ctypes.c_int64,
}

_lib = None


class SmokeCudaError(RuntimeError):
    """A CUDA-side failure (status SG_ERR_CUDA / SG_ERR_NONFINITE)."""


class NotConverged(RuntimeError):
    """A tolerance solve stopped at its cycle/iteration cap (status SG_ERR_NOT_CONVERGED)."""

    def __init__(self, msg, cycles=None, relres=None):
        super().__init__(msg)
        self.cycles = cycles
        self.relres = relres


def load():
    """Load the library once; raise if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"CUDA library not built: {LIB_PATH} is missing. Build it with "
                "`python python-game-engine_b200/build.py` (nvcc, sm_100a)."
            )
        lib = ctypes.CDLL(LIB_PATH)
        for name, argtypes in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = argtypes
            fn.restype = _RESTYPE.get(name, ctypes.c_int)
        _lib = lib
    return _lib


def bounds_check(clear=True):
    """(first failed source line, unit) recorded by the bounds-check build since the last
    clear, (0, -1) when none (and always in the normal build)."""
    line, unit = ctypes.c_uint(0), ctypes.c_int(-1)
    check(load().sg_bounds_check(ctypes.byref(line), ctypes.byref(unit), 1 if clear else 0), "sg_bounds_check")
    return line.value, unit.value


def exported_symbols():
    return list(SIGNATURES)


def check(status: int, what: str = ""):
    if status == SG_OK:
        return
    msg = load().sg_last_error().decode(errors="replace")
    text = f"{what}: {msg}" if what else msg
    if status in (SG_ERR_ARG, SG_ERR_WORKSPACE, SG_ERR_CAPACITY):
        raise ValueError(text)
    if status == SG_ERR_DTYPE:
        raise TypeError(text)
    if status == SG_ERR_NOT_CONVERGED:
        raise NotConverged(text)
    raise SmokeCudaError(text)


def call(name: str, *args):
    """Call an entry point and raise on a non-zero status."""
    check(getattr(load(), name)(*args), name)


def stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def dtype_code(t: torch.Tensor) -> int:
    if t.dtype == torch.float32:
        return SG_F32
    if t.dtype == torch.float64:
        return SG_F64
    raise TypeError(f"unsupported field dtype {t.dtype} (float32 or float64)")


def field(t: torch.Tensor, name: str = "field", dtype=None):
    """(pointer, row stride) of a 2-D CUDA tensor with unit column stride."""
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor on a CUDA device, got {type(t).__name__}")
    if not t.is_cuda:
        raise ValueError(f"{name} must live on a CUDA device")
    if t.dim() != 2:
        raise ValueError(f"{name} must be 2-D, got shape {tuple(t.shape)}")
    if dtype is not None and t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    if t.stride(1) != 1 and t.shape[1] > 1:
        raise ValueError(f"{name} must have unit column stride")
    ld = t.stride(0) if t.shape[0] > 1 else t.shape[1]
    return ctypes.c_void_p(t.data_ptr()), max(ld, t.shape[1])


def mask_plane(t: torch.Tensor, name: str, shape):
    """(pointer, stride) of a bool/uint8 CUDA mask plane of the given shape."""
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if t.dtype not in (torch.bool, torch.uint8):
        raise TypeError(f"{name} must be bool or uint8, got {t.dtype}")
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} must have shape {tuple(shape)}, got {tuple(t.shape)}")
    if t.stride(1) != 1 and t.shape[1] > 1:
        raise ValueError(f"{name} must have unit column stride")
    ld = t.stride(0) if t.shape[0] > 1 else t.shape[1]
    return ctypes.c_void_p(t.data_ptr()), max(ld, t.shape[1])
