"""CUDA operators with the reference's call signatures (src/cfd/operators/base.py:4-139).

Each function takes torch CUDA tensors (float32 or float64; bool/uint8 masks),
works in place on the caller's destination and returns None (compute_residual
returns its output, as residual.py:42 does). All launches go to the current
torch CUDA stream. Masks may also be the analytic sentinels ``OPEN_BOX`` (every
interior face open -- what SmokeSimulation2D builds at construction) or
``RING_BOX`` (a box whose outermost cells are solid); the kernels then evaluate
the mask instead of reading a plane.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib as L
from .registry import get_operator, register_operator


class AnalyticMask:
    """A mask the kernels evaluate from its definition instead of reading a plane."""

    def __init__(self, mode: int, name: str):
        self.mode = mode
        self.name = name

    def __repr__(self):
        return f"<{self.name}>"


OPEN_BOX = AnalyticMask(L.SG_MASK_OPEN, "OPEN_BOX")
RING_BOX = AnalyticMask(L.SG_MASK_RING, "RING_BOX")

_NULL = (None, 0)


def _masks(m, name, shape):
    """(mode, ptr, ld) for a face/fluid mask argument."""
    if isinstance(m, AnalyticMask):
        return m.mode, None, 0
    p, ld = L.mask_plane(m, name, shape)
    return L.SG_MASK_PLANES, p, ld


def _face_pair(fmu, fmv, H, W):
    mu, pu, lu = _masks(fmu, "face_mask_u", (H, W + 1))
    mv, pv, lv = _masks(fmv, "face_mask_v", (H + 1, W))
    if mu != mv:
        raise ValueError("face_mask_u and face_mask_v must both be planes or the same analytic mask")
    return mu, pu, lu, pv, lv


def _same_dtype(*ts):
    d = ts[0].dtype
    for t in ts[1:]:
        if t.dtype != d:
            raise TypeError(f"all fields must share one dtype, got {d} and {t.dtype}")
    return L.dtype_code(ts[0])


def _arithmetic(arithmetic, dt_code):
    if arithmetic == "reference":
        return False
    if arithmetic == "float32":
        if dt_code != L.SG_F32:
            raise TypeError("arithmetic='float32' takes float32 fields")
        return True
    raise ValueError(f"arithmetic must be 'reference' or 'float32', got {arithmetic!r}")


def advect_scalar_field(field_source, field_dest, velocity_u, velocity_v, is_fluid, dt, cell_size,
                        dissipation: float = 1.0, arithmetic: str = "reference", **_ignored):
    """advection.py:112-128; ``dissipation`` fuses simulation.py:232 (density *= 0.999).
    ``arithmetic="float32"`` (float32 fields): backtrace and interpolation in float32
    relative to the cell (``sg_advect_scalar_f32``), equal to the reference's float64
    arithmetic up to rounding; "reference" (default) reproduces it bit for bit."""
    dt_code = _same_dtype(field_source, field_dest, velocity_u, velocity_v)
    H, W = field_source.shape
    if tuple(field_dest.shape) != (H, W):
        raise ValueError("field_dest must match field_source")
    s, lds = L.field(field_source, "field_source")
    d, ldd = L.field(field_dest, "field_dest")
    u, ldu = L.field(velocity_u, "velocity_u")
    v, ldv = L.field(velocity_v, "velocity_v")
    mode, pf, ldf = _masks(is_fluid, "is_fluid", (H, W))
    if _arithmetic(arithmetic, dt_code):
        if tuple(velocity_u.shape) != (H, W + 1) or tuple(velocity_v.shape) != (H + 1, W):
            raise ValueError("velocity fields must have MAC shapes (H, W+1) and (H+1, W)")
        L.call("sg_advect_scalar_f32", H, W, s, lds, d, ldd, u, ldu, v, ldv, mode, pf, ldf, float(dt),
               float(cell_size), float(dissipation), L.stream_ptr())
        return
    L.call("sg_advect_scalar", dt_code, H, W, s, lds, d, ldd, u, velocity_u.shape[0], velocity_u.shape[1], ldu,
           v, velocity_v.shape[0], velocity_v.shape[1], ldv, mode, pf, ldf, float(dt), float(cell_size),
           float(dissipation), L.stream_ptr())


def advect_velocity_u(velocity_u_source, velocity_u_dest, velocity_v, face_mask_u, dt, cell_size, **_ignored):
    """advection.py:130-154."""
    dt_code = _same_dtype(velocity_u_source, velocity_u_dest, velocity_v)
    ur, uc = velocity_u_source.shape
    s, lds = L.field(velocity_u_source, "velocity_u_source")
    d, ldd = L.field(velocity_u_dest, "velocity_u_dest")
    v, ldv = L.field(velocity_v, "velocity_v")
    mode, pm, ldm = _masks(face_mask_u, "face_mask_u", (ur, uc))
    L.call("sg_advect_velocity_u", dt_code, ur, uc, s, lds, d, ldd, v, velocity_v.shape[0], velocity_v.shape[1], ldv,
           mode, pm, ldm, float(dt), float(cell_size), L.stream_ptr())


def advect_velocity_v(velocity_v_source, velocity_v_dest, velocity_u, face_mask_v, dt, cell_size, **_ignored):
    """advection.py:156-180."""
    dt_code = _same_dtype(velocity_v_source, velocity_v_dest, velocity_u)
    vr, vc = velocity_v_source.shape
    s, lds = L.field(velocity_v_source, "velocity_v_source")
    d, ldd = L.field(velocity_v_dest, "velocity_v_dest")
    u, ldu = L.field(velocity_u, "velocity_u")
    mode, pm, ldm = _masks(face_mask_v, "face_mask_v", (vr, vc))
    L.call("sg_advect_velocity_v", dt_code, vr, vc, s, lds, d, ldd, u, velocity_u.shape[0], velocity_u.shape[1], ldu,
           mode, pm, ldm, float(dt), float(cell_size), L.stream_ptr())


def advect_velocity(u_src, u_dst, v_src, v_dst, face_mask_u, face_mask_v, dt, cell_size, arithmetic="reference"):
    """Both velocity advections of simulation.py:280-286 in one launch (MAC shapes);
    ``arithmetic`` as for advect_scalar_field."""
    dt_code = _same_dtype(u_src, u_dst, v_src, v_dst)
    H, W1 = u_src.shape
    W = W1 - 1
    if tuple(v_src.shape) != (H + 1, W):
        raise ValueError("velocity fields must have MAC shapes (H, W+1) and (H+1, W)")
    mode, pu, lu, pv, lv = _face_pair(face_mask_u, face_mask_v, H, W)
    a, lda = L.field(u_src, "u_src")
    b, ldb = L.field(u_dst, "u_dst")
    c, ldc = L.field(v_src, "v_src")
    d, ldd = L.field(v_dst, "v_dst")
    if _arithmetic(arithmetic, dt_code):
        L.call("sg_advect_velocity_f32", H, W, a, lda, b, ldb, c, ldc, d, ldd, mode, pu, lu, pv, lv, float(dt),
               float(cell_size), L.stream_ptr())
        return
    L.call("sg_advect_velocity", dt_code, H, W, a, lda, b, ldb, c, ldc, d, ldd, mode, pu, lu, pv, lv, float(dt),
           float(cell_size), L.stream_ptr())


def apply_forces(velocity_v, density, temperature, dt, gravity, buoyancy_coefficient, density_coefficient,
                 ambient_temperature, f32_temporaries: bool = True, arithmetic="reference", **_ignored):
    """forces.py:78-105. ``temperature`` may be None (ambient everywhere). ``arithmetic``:
    "reference" (the reference's float64 terms, bit for bit) or, for float32 fields,
    "float32" (``sg_apply_forces_f32``: equal up to rounding)."""
    dt_code = _same_dtype(velocity_v, density, *( [temperature] if temperature is not None else []))
    H, W = density.shape
    if tuple(velocity_v.shape) != (H + 1, W):
        raise ValueError("velocity_v must be (H+1, W)")
    v, ldv = L.field(velocity_v, "velocity_v")
    d, ldd = L.field(density, "density")
    t, ldt = L.field(temperature, "temperature") if temperature is not None else _NULL
    if _arithmetic(arithmetic, dt_code):
        L.call("sg_apply_forces_f32", H, W, v, ldv, d, ldd, t, ldt, float(dt), float(gravity),
               float(buoyancy_coefficient), float(density_coefficient), float(ambient_temperature), L.stream_ptr())
        return
    L.call("sg_apply_forces", dt_code, H, W, v, ldv, d, ldd, t, ldt, float(dt), float(gravity),
           float(buoyancy_coefficient), float(density_coefficient), float(ambient_temperature),
           1 if f32_temporaries else 0, L.stream_ptr())


def cool_temperature(temperature, ambient_temperature, cooling_rate, dt, **_ignored):
    """forces.py:108-123."""
    H, W = temperature.shape
    t, ld = L.field(temperature, "temperature")
    L.call("sg_cool_temperature", L.dtype_code(temperature), H, W, t, ld, float(ambient_temperature),
           float(cooling_rate), float(dt), L.stream_ptr())


def compute_divergence(velocity_u, velocity_v, divergence, mask_u, mask_v, cell_size, **_ignored):
    """divergence.py:4-25."""
    dt_code = _same_dtype(velocity_u, velocity_v, divergence)
    H, W = divergence.shape
    mode, pu, lu, pv, lv = _face_pair(mask_u, mask_v, H, W)
    u, ldu = L.field(velocity_u, "velocity_u")
    v, ldv = L.field(velocity_v, "velocity_v")
    d, ldd = L.field(divergence, "divergence")
    L.call("sg_compute_divergence", dt_code, H, W, u, ldu, v, ldv, d, ldd, mode, pu, lu, pv, lv, float(cell_size),
           L.stream_ptr())


def compute_residual(pressure, divergence, is_fluid, face_mask_u, face_mask_v, alpha, reciprocal_beta, residual_out,
                     sumsq=None, **_ignored):
    """residual.py:6-42; returns ``residual_out``. ``sumsq`` (a CUDA float64 tensor of one
    element) optionally accumulates the sum of squared residuals over fluid cells."""
    dt_code = _same_dtype(pressure, divergence, residual_out)
    H, W = pressure.shape
    mode, pu, lu, pv, lv = _face_pair(face_mask_u, face_mask_v, H, W)
    fmode, pf, ldf = _masks(is_fluid, "is_fluid", (H, W))
    if fmode != mode:
        raise ValueError("is_fluid and the face masks must both be planes or the same analytic mask")
    p, ldp = L.field(pressure, "pressure")
    d, ldd = L.field(divergence, "divergence")
    o, ldo = L.field(residual_out, "residual_out")
    sq = None
    if sumsq is not None:
        if sumsq.dtype != torch.float64 or not sumsq.is_cuda:
            raise TypeError("sumsq must be a float64 CUDA tensor")
        sq = sumsq.data_ptr()
    L.call("sg_compute_residual", dt_code, H, W, p, ldp, d, ldd, mode, pf, ldf, pu, lu, pv, lv, float(alpha),
           float(reciprocal_beta), o, ldo, sq, L.stream_ptr())
    return residual_out


def apply_pressure_gradient(velocity_u, velocity_v, pressure, face_mask_u, face_mask_v, fluid_density, cell_size, dt,
                            **_ignored):
    """pressure_gradient.py:4-37."""
    dt_code = _same_dtype(velocity_u, velocity_v, pressure)
    H, W = pressure.shape
    mode, pu, lu, pv, lv = _face_pair(face_mask_u, face_mask_v, H, W)
    u, ldu = L.field(velocity_u, "velocity_u")
    v, ldv = L.field(velocity_v, "velocity_v")
    p, ldp = L.field(pressure, "pressure")
    L.call("sg_apply_pressure_gradient", dt_code, H, W, u, ldu, v, ldv, p, ldp, mode, pu, lu, pv, lv,
           float(fluid_density), float(cell_size), float(dt), L.stream_ptr())


def _solid_arg(solid_mask, H, W):
    if solid_mask is None:
        return L.SG_MASK_NONE, None, 0
    if isinstance(solid_mask, AnalyticMask):
        if solid_mask.mode != L.SG_MASK_RING:
            return L.SG_MASK_NONE, None, 0
        return L.SG_MASK_RING, None, 0
    p, ld = L.mask_plane(solid_mask, "solid_mask", (H, W))
    return L.SG_MASK_PLANES, p, ld


def enforce_boundary_conditions(velocity_u, velocity_v, solid_mask, **_ignored):
    """boundaries.py:7-39. ``solid_mask``: (H, W) plane, RING_BOX, or None."""
    dt_code = _same_dtype(velocity_u, velocity_v)
    H, W = velocity_u.shape[0], velocity_u.shape[1] - 1
    smode, ps, lds = _solid_arg(solid_mask, H, W)
    u, ldu = L.field(velocity_u, "velocity_u")
    v, ldv = L.field(velocity_v, "velocity_v")
    L.call("sg_enforce_boundary_conditions", dt_code, H, W, u, ldu, v, ldv, smode, ps, lds, L.stream_ptr())


def project(velocity_u, velocity_v, pressure, face_mask_u, face_mask_v, solid_mask, fluid_density, cell_size, dt):
    """apply_pressure_gradient then enforce_boundary_conditions in one pass (simulation.py:244-249)."""
    dt_code = _same_dtype(velocity_u, velocity_v, pressure)
    H, W = pressure.shape
    mode, pu, lu, pv, lv = _face_pair(face_mask_u, face_mask_v, H, W)
    smode, ps, lds = _solid_arg(solid_mask, H, W)
    u, ldu = L.field(velocity_u, "velocity_u")
    v, ldv = L.field(velocity_v, "velocity_v")
    p, ldp = L.field(pressure, "pressure")
    L.call("sg_project", dt_code, H, W, u, ldu, v, ldv, p, ldp, mode, pu, lu, pv, lv, smode, ps, lds,
           float(fluid_density), float(cell_size), float(dt), L.stream_ptr())


APPROACH_CODES = {"hard_cutoff": 0, "linear": 1, "quadratic": 2, "gaussian": 3}


def project_metrics(u_in, v_in, u_out, v_out, pressure, face_mask_u, face_mask_v, is_fluid, solid_mask, fluid_density,
                    cell_size, dt, alpha, reciprocal_beta, divergence_out, residual_out, arithmetic="reference"):
    """The substep's tail in one pass (simulation.py:244-265): project (u_in, v_in) into
    (u_out, v_out) (apply_pressure_gradient + enforce_boundary_conditions, out of place),
    then the divergence of the projected field into ``divergence_out`` and the reference
    residual of ``pressure`` with it into ``residual_out`` -- the values the four separate
    operators give."""
    dt_code = _same_dtype(u_in, v_in, u_out, v_out, pressure, divergence_out, residual_out)
    H, W = pressure.shape
    mode, pu, lu, pv, lv = _face_pair(face_mask_u, face_mask_v, H, W)
    fmode, pf, ldf = _masks(is_fluid, "is_fluid", (H, W))
    if fmode != mode:
        raise ValueError("is_fluid and the face masks must both be planes or the same analytic mask")
    smode, ps, lds = _solid_arg(solid_mask, H, W)
    a = [L.field(x, n) for x, n in ((u_in, "u_in"), (v_in, "v_in"), (u_out, "u_out"), (v_out, "v_out"),
                                    (pressure, "pressure"), (divergence_out, "divergence_out"),
                                    (residual_out, "residual_out"))]
    if _arithmetic(arithmetic, dt_code):  # float32 fields in float32 arithmetic
        L.call("sg_project_metrics_f32", H, W, a[0][0], a[0][1], a[1][0], a[1][1], a[2][0], a[2][1], a[3][0],
               a[3][1], a[4][0], a[4][1], mode, pu, lu, pv, lv, pf, ldf, smode, ps, lds, float(fluid_density),
               float(cell_size), float(dt), float(alpha), float(reciprocal_beta), a[5][0], a[5][1], a[6][0],
               a[6][1], L.stream_ptr())
        return
    L.call("sg_project_metrics", dt_code, H, W, a[0][0], a[0][1], a[1][0], a[1][1], a[2][0], a[2][1], a[3][0],
           a[3][1], a[4][0], a[4][1], mode, pu, lu, pv, lv, pf, ldf, smode, ps, lds, float(fluid_density),
           float(cell_size), float(dt), float(alpha), float(reciprocal_beta), a[5][0], a[5][1], a[6][0], a[6][1],
           L.stream_ptr())


def emit_scalar(field, value, dt, pos_x, pos_y, radius, approach):
    """emitters.py:37-66: field += value * falloff(dist) * dt inside the radius."""
    if approach not in APPROACH_CODES:
        raise ValueError(f"Unknown emission approach: {approach}")
    H, W = field.shape
    f, ld = L.field(field, "field")
    L.call("sg_emit_scalar", L.dtype_code(field), H, W, f, ld, float(value), float(dt), float(pos_x), float(pos_y),
           float(radius), APPROACH_CODES[approach], L.stream_ptr())


def plume_sources(density, velocity_u, velocity_v, sources, seed, step):
    """Overwriting disc sources (benchmark scenes). ``sources``: host table of shape (n, 6)
    (numpy array, CPU tensor or nested list) of (cx, cy, r, density, v, noise_amp) rows;
    it travels in the kernel's launch parameters."""
    dt_code = _same_dtype(density, velocity_u, velocity_v)
    H, W = density.shape
    if isinstance(sources, torch.Tensor):
        if sources.is_cuda:
            raise ValueError("sources must be a host table (it is passed in the launch parameters)")
        sources = sources.numpy()
    src = np.ascontiguousarray(np.asarray(sources, dtype=np.float64).reshape(-1, 6))
    d, ldd = L.field(density, "density")
    u, ldu = L.field(velocity_u, "velocity_u")
    v, ldv = L.field(velocity_v, "velocity_v")
    L.call("sg_plume_sources", dt_code, H, W, d, ldd, u, ldu, v, ldv, src.shape[0],
           src.ctypes.data_as(ctypes.c_void_p), int(seed) & (2**64 - 1), int(step), L.stream_ptr())


def build_masks(solid_mask):
    """Face masks and is_fluid from a solid plane (simulation.py:103-108); returns uint8 tensors."""
    H, W = solid_mask.shape
    s = solid_mask.to(torch.uint8).contiguous()
    fmu = torch.empty((H, W + 1), dtype=torch.uint8, device=s.device)
    fmv = torch.empty((H + 1, W), dtype=torch.uint8, device=s.device)
    fl = torch.empty((H, W), dtype=torch.uint8, device=s.device)
    L.call("sg_build_masks", H, W, s.data_ptr(), W, fmu.data_ptr(), W + 1, fmv.data_ptr(), W, fl.data_ptr(), W,
           L.stream_ptr())
    return fmu.bool(), fmv.bool(), fl.bool()


# registry names of src/cfd/operators/registrations.py:21-29
_REGISTRATIONS = {
    "advection_scalar": advect_scalar_field,
    "advection_velocity_u": advect_velocity_u,
    "advection_velocity_v": advect_velocity_v,
    "enforce_boundary_conditions": enforce_boundary_conditions,
    "compute_divergence": compute_divergence,
    "apply_forces": apply_forces,
    "cool_temperature": cool_temperature,
    "apply_pressure_gradient": apply_pressure_gradient,
    "compute_residual": compute_residual,
}

_registered = False


def register_operators():
    """Register the CUDA operators under backend "cuda" (idempotent)."""
    global _registered
    if _registered:
        return
    for name, fn in _REGISTRATIONS.items():
        register_operator(name, "cuda", fn)
    _registered = True


def dispatch(operation: str, *args, backend: str = "cuda", **kwargs):
    """Per-op dispatch as the reference's dispatchers do (e.g. operators/advection.py:13-38)."""
    return get_operator(operation, backend)(*args, **kwargs)
