"""CPU oracle for the smoke-simulation step.

TEST INFRASTRUCTURE ONLY. This package is the checker for the CUDA library
(``tests/``, ``__graft_entry__.smoke()``) and the CPU baseline that ``bench.py``
times beside it. The product path never imports it.

Layout:
  * ``smoke_oracle.c`` / ``smoke_oracle_impl.h`` -- a plain-C restatement of the
    reference's Numba kernels (LCEBurton/python-game-engine, ``src/cfd/backends/numba``),
    float32 and float64, OpenMP over rows. Built by ``oracle/Makefile``.
  * this module -- ctypes bindings plus the Python drivers the reference keeps in
    Python (solver loops, the multigrid recursion, the substep order), and the
    project's own FP64 restatement of the convergent multigrid / iterative
    refinement, which has no reference counterpart.

Parity pin: ``tests/test_oracle_golden.py`` checks every function here against
fixtures produced by running the reference itself (``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libsmoke_oracle.so")
_lib = None

_P = ctypes.c_void_p
_L = ctypes.c_long
_D = ctypes.c_double
_I = ctypes.c_int

_SIGS = {
    "or_advect_scalar": [_P, _P, _L, _L, _P, _L, _L, _P, _L, _L, _P, _D, _D],
    "or_advect_u": [_P, _P, _L, _L, _P, _L, _L, _P, _D, _D],
    "or_advect_v": [_P, _P, _L, _L, _P, _L, _L, _P, _D, _D],
    "or_apply_forces": [_P, _L, _L, _P, _P, _D, _D, _D, _D, _D, _I],
    "or_cool_temperature": [_P, _L, _L, _D, _D, _D],
    "or_divergence": [_P, _P, _P, _P, _P, _L, _L, _D],
    "or_jacobi_sweep": [_P, _P, _P, _P, _P, _P, _L, _L, _D, _D],
    "or_rbsor": [_P, _P, _P, _P, _P, _L, _L, _D, _D, _D, _L],
    "or_gauss_seidel": [_P, _P, _P, _P, _P, _L, _L, _D, _D, _L],
    "or_residual": [_P, _P, _P, _P, _P, _L, _L, _D, _D, _P],
    "or_pressure_gradient": [_P, _P, _P, _P, _P, _L, _L, _D, _D, _D],
    "or_enforce_bc": [_P, _P, _P, _L, _L],
    "or_restrict_avg": [_P, _P, _L, _L, _P, _L, _L],
    "or_prolong": [_P, _L, _L, _P, _L, _L, _P],
    "or_emit_scalar": [_P, _L, _L, _D, _D, _D, _D, _D, _I],
    "or_plume_source": [_P, _P, _P, _L, _L, _D, _D, _D, _D, _D, _D, ctypes.c_ulonglong, _L],
    "or_gmg_residual": [_P, _P, _P, _P, _P, _L, _L, _P],
    "or_gmg_rbgs": [_P, _P, _P, _P, _P, _L, _L, _D, _L],
    "or_gmg_prolong_add": [_P, _P, _L, _L, _P, _P, _L, _L],
    "or_gmg_restrict_fw": [_P, _P, _L, _L, _P, _P, _L, _L],
}

APPROACHES = {"hard_cutoff": 0, "linear": 1, "quadratic": 2, "gaussian": 3}


def build() -> str:
    """Compile the oracle library with its Makefile; returns the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        for base, argtypes in _SIGS.items():
            for sfx in ("_f32", "_f64"):
                fn = getattr(L, base + sfx)
                fn.argtypes = argtypes
                fn.restype = None
        L.sg_noise.argtypes = [ctypes.c_ulonglong, _L, _I, _L, _L, _D]
        L.sg_noise.restype = _D
        _lib = L
    return _lib


def _fn(name, dtype):
    return getattr(lib(), name + ("_f32" if np.dtype(dtype) == np.float32 else "_f64"))


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return a.ctypes.data_as(ctypes.c_void_p)


def _mask(m: np.ndarray) -> np.ndarray:
    m = np.ascontiguousarray(m)
    if m.dtype != np.uint8:
        m = m.astype(np.uint8)
    return m


def _real(*arrays):
    dt = arrays[0].dtype
    assert dt in (np.float32, np.float64), dt
    for a in arrays:
        assert a.dtype == dt, (a.dtype, dt)
    return dt


def noise(seed, step, comp, j, i, amp):
    return lib().sg_noise(seed, step, comp, j, i, amp)


# ---------------------------------------------------------------- operators
def advect_scalar_field(src, dst, u, v, is_fluid, dt, cell_size):
    """advection.py:112-128."""
    _real(src, dst, u, v)
    H, W = src.shape
    m = _mask(is_fluid)
    _fn("or_advect_scalar", src.dtype)(_ptr(src), _ptr(dst), H, W, _ptr(u), u.shape[0], u.shape[1],
                                        _ptr(v), v.shape[0], v.shape[1], _ptr(m), dt, cell_size)


def advect_velocity_u(u_src, u_dst, v, face_mask_u, dt, cell_size):
    """advection.py:130-154."""
    _real(u_src, u_dst, v)
    m = _mask(face_mask_u)
    _fn("or_advect_u", u_src.dtype)(_ptr(u_src), _ptr(u_dst), u_src.shape[0], u_src.shape[1],
                                     _ptr(v), v.shape[0], v.shape[1], _ptr(m), dt, cell_size)


def advect_velocity_v(v_src, v_dst, u, face_mask_v, dt, cell_size):
    """advection.py:156-180."""
    _real(v_src, v_dst, u)
    m = _mask(face_mask_v)
    _fn("or_advect_v", v_src.dtype)(_ptr(v_src), _ptr(v_dst), v_src.shape[0], v_src.shape[1],
                                     _ptr(u), u.shape[0], u.shape[1], _ptr(m), dt, cell_size)


def apply_forces(v, density, temperature, dt, gravity, buoyancy_coefficient,
                 density_coefficient, ambient_temperature, f32_temporaries=True):
    """forces.py:78-105 (v is (H+1, W))."""
    _real(v, density, temperature)
    H, W = density.shape
    assert v.shape == (H + 1, W)
    _fn("or_apply_forces", v.dtype)(_ptr(v), H, W, _ptr(density), _ptr(temperature), dt, gravity,
                                     buoyancy_coefficient, density_coefficient, ambient_temperature,
                                     1 if f32_temporaries else 0)


def cool_temperature(temperature, ambient_temperature, cooling_rate, dt):
    """forces.py:108-123."""
    H, W = temperature.shape
    _fn("or_cool_temperature", temperature.dtype)(_ptr(temperature), H, W, ambient_temperature,
                                                  cooling_rate, dt)


def compute_divergence(u, v, div, fmu, fmv, cell_size):
    """divergence.py:4-25."""
    _real(u, v, div)
    H, W = div.shape
    _fn("or_divergence", div.dtype)(_ptr(u), _ptr(v), _ptr(div), _ptr(_mask(fmu)), _ptr(_mask(fmv)),
                                     H, W, cell_size)


def compute_residual(p, div, is_fluid, fmu, fmv, alpha, reciprocal_beta, out):
    """residual.py:6-42."""
    _real(p, div, out)
    H, W = p.shape
    _fn("or_residual", p.dtype)(_ptr(p), _ptr(div), _ptr(_mask(is_fluid)), _ptr(_mask(fmu)),
                                 _ptr(_mask(fmv)), H, W, alpha, reciprocal_beta, _ptr(out))
    return out


def apply_pressure_gradient(u, v, p, fmu, fmv, rho, cell_size, dt):
    """pressure_gradient.py:4-37 (outer faces must be closed, as the reference builds them)."""
    _real(u, v, p)
    fmu = _mask(fmu)
    fmv = _mask(fmv)
    assert not fmu[:, 0].any() and not fmu[:, -1].any(), "outer u faces must be closed"
    assert not fmv[0].any() and not fmv[-1].any(), "outer v faces must be closed"
    H, W = p.shape
    _fn("or_pressure_gradient", p.dtype)(_ptr(u), _ptr(v), _ptr(p), _ptr(fmu), _ptr(fmv), H, W,
                                          rho, cell_size, dt)


def enforce_boundary_conditions(u, v, solid):
    """boundaries.py:7-39."""
    H, W = solid.shape
    _fn("or_enforce_bc", u.dtype)(_ptr(u), _ptr(v), _ptr(_mask(solid)), H, W)


# ---------------------------------------------------------------- coefficients
def alpha_coeff(cell_size, density, dt):
    """solvers/common.py:6-18 (calculateAlpha)."""
    return (-(cell_size * cell_size) * density) / dt


def reciprocal_beta():
    """solvers/common.py:20-28."""
    return 0.25


def optimal_omega(size):
    """solvers/common.py:30-39."""
    return min(2.0 / (1.0 + math.sin(math.pi / size)), 1.95)


def is_fluid_from_faces(fmu, fmv):
    """common/simulation.py:108."""
    return fmu[:, :-1] | fmu[:, 1:] | fmv[:-1, :] | fmv[1:, :]


def face_masks_from_solid(solid):
    """common/simulation.py:103-107 / multigrid/masks.py:30-49."""
    H, W = solid.shape
    fmu = np.zeros((H, W + 1), bool)
    fmv = np.zeros((H + 1, W), bool)
    fmu[:, 1:-1] = ~(solid[:, :-1] | solid[:, 1:])
    fmv[1:-1, :] = ~(solid[:-1, :] | solid[1:, :])
    return fmu, fmv


def box_solid(H, W):
    """common/simulation.py:126-131 (1-cell solid ring)."""
    s = np.zeros((H, W), bool)
    s[0, :] = s[-1, :] = True
    s[:, 0] = s[:, -1] = True
    return s


# ---------------------------------------------------------------- solvers
def jacobi_sweep(p, out, div, is_fluid, fmu, fmv, alpha, rb):
    H, W = p.shape
    _fn("or_jacobi_sweep", p.dtype)(_ptr(p), _ptr(out), _ptr(div), _ptr(_mask(is_fluid)),
                                     _ptr(_mask(fmu)), _ptr(_mask(fmv)), H, W, alpha, rb)


def jacobi_pressure_solver(p, div, fmu, fmv, fluid_density, cell_size, dt, iterations, **_ignored):
    """jacobi.py:27-52."""
    alpha = alpha_coeff(cell_size, fluid_density, dt)
    rb = reciprocal_beta()
    tmp = np.empty_like(p)
    fl = is_fluid_from_faces(fmu, fmv)
    src, dst = p, tmp
    for _ in range(iterations):
        jacobi_sweep(src, dst, div, fl, fmu, fmv, alpha, rb)
        src, dst = dst, src
    if src is not p:
        p[:] = src


def rb_sor_pressure_solver(p, div, fmu, fmv, fluid_density, cell_size, dt, iterations, omega=0.0,
                           **_ignored):
    """red_black_sor_gauss_seidel.py:30-42."""
    H, W = p.shape
    alpha = alpha_coeff(cell_size, fluid_density, dt)
    fl = is_fluid_from_faces(fmu, fmv)
    if omega <= 0.0 or omega > 2.0:
        omega = optimal_omega(max(H, W))
    _fn("or_rbsor", p.dtype)(_ptr(p), _ptr(div), _ptr(_mask(fl)), _ptr(_mask(fmu)), _ptr(_mask(fmv)),
                              H, W, alpha, reciprocal_beta(), omega, iterations)


def gauss_seidel_pressure_solver(p, div, fmu, fmv, fluid_density, cell_size, dt, iterations,
                                 **_ignored):
    """gauss_seidel.py:29-48."""
    H, W = p.shape
    alpha = alpha_coeff(cell_size, fluid_density, dt)
    fl = is_fluid_from_faces(fmu, fmv)
    _fn("or_gauss_seidel", p.dtype)(_ptr(p), _ptr(div), _ptr(_mask(fl)), _ptr(_mask(fmu)),
                                     _ptr(_mask(fmv)), H, W, alpha, reciprocal_beta(), iterations)


def rb_sor_tolerance(p, div, fmu, fmv, fluid_density, cell_size, dt, omega=1.9, tol=1e-6, max_iterations=200000,
                     check_every=100):
    """The CUDA SORToleranceSolver's loop (no reference counterpart; the reference runs a
    fixed sweep count): red_black_sor_gauss_seidel.py:8-27 sweeps in chunks of `check_every`
    until ||r(p)|| <= tol ||r(0)|| over fluid cells, r the reference residual
    (residual.py:39-40) rounded to the field's dtype, squares summed in float64.
    Returns (sweeps, relative residual)."""
    alpha = alpha_coeff(cell_size, fluid_density, dt)
    fl = is_fluid_from_faces(fmu, fmv)
    out = np.empty_like(p)

    def norm(q):
        compute_residual(q, div, fl, fmu, fmv, alpha, reciprocal_beta(), out)
        return float(np.sqrt(np.sum(out.astype(np.float64) ** 2)))

    r0 = norm(np.zeros_like(p))
    rel = norm(p) / r0 if r0 > 0 else 0.0
    it = 0
    while rel > tol and it < max_iterations:
        n = min(check_every, max_iterations - it)
        _fn("or_rbsor", p.dtype)(_ptr(p), _ptr(div), _ptr(_mask(fl)), _ptr(_mask(fmu)), _ptr(_mask(fmv)),
                                  p.shape[0], p.shape[1], alpha, reciprocal_beta(), omega, n)
        it += n
        rel = norm(p) / r0 if r0 > 0 else 0.0
    return it, rel


def rb_sor_mixed(p, div, fmu, fmv, fluid_density, cell_size, dt, omega=1.9, tol=1e-6, max_iterations=200000,
                 check_every=100):
    """The CUDA mixed-precision SOR (no reference counterpart): float64 iterative refinement
    around float32 red-black SOR sweeps (red_black_sor_gauss_seidel.py:8-27). The pressure
    is accumulated in float64; each refinement forms the float64 reference residual r
    (residual.py:39-40) and solves A e = float32(r) from e = 0 with float32 sweeps (alpha = 1)
    in chunks of `check_every`, until the correction's relative residual reaches
    max(1e-3, tol / (2 ||r|| / ||r0||)) (at most 0.5) or three chunks in a row gain less than
    1 %; then p += e. Stops when ||r(p)|| <= tol ||r(0)||. `p` and `div` are float32.
    Returns (sweeps, relative residual, refinements)."""
    alpha = alpha_coeff(cell_size, fluid_density, dt)
    fl = is_fluid_from_faces(fmu, fmv)
    H, W = p.shape
    p64 = p.astype(np.float64)
    d64 = div.astype(np.float64)
    out64 = np.empty_like(p64)
    out32 = np.empty((H, W), np.float32)

    def res64(q):
        return compute_residual(q, d64, fl, fmu, fmv, alpha, reciprocal_beta(), out64)

    r0 = float(np.sqrt(np.sum(res64(np.zeros_like(p64)) ** 2)))
    it = outer = 0
    while True:
        r = res64(p64)
        rel = float(np.sqrt(np.sum(r ** 2))) / r0 if r0 > 0 else 0.0
        if not np.isfinite(rel) or rel <= tol or it >= max_iterations:
            break
        inner_tol = min(0.5, max(1e-3, 0.5 * tol / rel))
        r32 = r.astype(np.float32)
        e = np.zeros((H, W), np.float32)

        def inorm(q):
            compute_residual(q, r32, fl, fmu, fmv, 1.0, reciprocal_beta(), out32)
            return float(np.sqrt(np.sum(out32.astype(np.float64) ** 2)))

        ir0 = inorm(np.zeros_like(e))
        irel = best = 1.0
        stalls = 0
        while irel > inner_tol and it < max_iterations:
            n = min(check_every, max_iterations - it)
            _fn("or_rbsor", np.float32)(_ptr(e), _ptr(r32), _ptr(_mask(fl)), _ptr(_mask(fmu)), _ptr(_mask(fmv)),
                                         H, W, 1.0, reciprocal_beta(), omega, n)
            it += n
            irel = inorm(e) / ir0 if ir0 > 0 else 0.0
            if not np.isfinite(irel):
                break
            if irel < 0.99 * best:
                best, stalls = irel, 0
            else:
                stalls += 1
                if stalls >= 3:
                    break
        p64 += e.astype(np.float64)
        outer += 1
        if not np.isfinite(irel):
            rel = irel
            break
    p[:] = p64.astype(np.float32)
    return it, rel, outer


SMOOTHERS = {
    "jacobi": jacobi_pressure_solver,
    "rb_sor_gauss_seidel": rb_sor_pressure_solver,
    "gauss_seidel": gauss_seidel_pressure_solver,
}


def restrict_avg(fine, is_fluid, coarse):
    """multigrid/transfer.py:5-36."""
    H, W = fine.shape
    Hc, Wc = coarse.shape
    _fn("or_restrict_avg", fine.dtype)(_ptr(fine), _ptr(_mask(is_fluid)), H, W, _ptr(coarse), Hc, Wc)
    return coarse


def prolong(coarse, is_fluid, fine):
    """multigrid/transfer.py:38-72."""
    Hc, Wc = coarse.shape
    H, W = fine.shape
    _fn("or_prolong", fine.dtype)(_ptr(coarse), Hc, Wc, _ptr(_mask(is_fluid)), H, W, _ptr(fine))
    return fine


def coarsen_solid_mask(solid):
    """multigrid/masks.py:3-27 (any solid child -> solid)."""
    H, W = solid.shape
    Hc, Wc = H // 2, W // 2
    s = solid[: 2 * Hc, : 2 * Wc]
    return s[0::2, 0::2] | s[0::2, 1::2] | s[1::2, 0::2] | s[1::2, 1::2]


class MultigridReference:
    """Restatement of ``MultigridSolver`` (multigrid/solver.py:16-176).

    The hierarchy (``_build_levels`` :34-73) starts from ``solid = ~is_fluid`` and
    coarsens with the any-solid rule while both dimensions are even; each level
    keeps pressure/residual/rhs/correction buffers; the V-cycle (:94-139) smooths,
    restricts the residual, divides the coarse rhs by alpha(2h), recurses from a
    zero guess, prolongs and adds, and smooths again. Like the reference it caches
    on the face-mask shape only; use one instance per dtype.
    """

    def __init__(self):
        self._shape = None
        self.levels = []
        self.buffers = []

    def _ensure(self, fmu, fmv, num_levels, dtype, rebuild):
        if rebuild or self._shape != fmu.shape or len(self.levels) != num_levels:
            fl = is_fluid_from_faces(fmu, fmv)
            solid = ~fl
            levels = [dict(is_fluid=fl, fmu=fmu, fmv=fmv, solid=solid)]
            for _ in range(1, num_levels):
                h, w = solid.shape
                if h % 2 or w % 2:
                    break
                sc = coarsen_solid_mask(solid)
                cu, cv = face_masks_from_solid(sc)
                levels.append(dict(is_fluid=is_fluid_from_faces(cu, cv), fmu=cu, fmv=cv, solid=sc))
                solid = sc
            self.levels = levels
            self.buffers = [
                {k: np.zeros(L["is_fluid"].shape, dtype) for k in ("pressure", "residual", "rhs", "correction")}
                for L in levels
            ]
            self._shape = fmu.shape

    def _v_cycle(self, k, p, rhs, rho, h, dt, smoother, nu, nu_c):
        L = self.levels[k]
        buf = self.buffers[k]
        coarsest = k == len(self.levels) - 1
        smoother(p, rhs, L["fmu"], L["fmv"], rho, h, dt, nu_c if coarsest else nu)
        if coarsest:
            return p
        alpha = alpha_coeff(h, rho, dt)
        compute_residual(p, rhs, L["is_fluid"], L["fmu"], L["fmv"], alpha, reciprocal_beta(),
                         buf["residual"])
        cb = self.buffers[k + 1]
        restrict_avg(buf["residual"], L["is_fluid"], cb["rhs"])
        cb["rhs"] /= alpha_coeff(h * 2.0, rho, dt)
        cb["pressure"].fill(0.0)
        self._v_cycle(k + 1, cb["pressure"], cb["rhs"], rho, h * 2.0, dt, smoother, nu, nu_c)
        prolong(cb["pressure"], L["is_fluid"], buf["correction"])
        p += buf["correction"]
        smoother(p, rhs, L["fmu"], L["fmv"], rho, h, dt, nu)
        return p

    def __call__(self, p, div, fmu, fmv, fluid_density, cell_size, dt, v_cycles=2,
                 smoother_type="jacobi", smoother_backend="numba", num_levels=4,
                 smoother_iterations=2, coarsest_iterations=50, rebuild_masks=False, **_ignored):
        self._ensure(fmu, fmv, num_levels, p.dtype, rebuild_masks)
        smoother = SMOOTHERS[smoother_type]
        fb = self.buffers[0]
        fb["pressure"][:] = p
        fb["rhs"][:] = div
        for _ in range(v_cycles):
            self._v_cycle(0, fb["pressure"], fb["rhs"], fluid_density, cell_size, dt, smoother,
                          smoother_iterations, coarsest_iterations)
        p[:] = fb["pressure"]


# ---------------------------------------------------------------- emitters
def emit_scalar(field, value, dt, px, py, radius, approach):
    """common/emitters.py:37-66 (Numba path)."""
    H, W = field.shape
    _fn("or_emit_scalar", field.dtype)(_ptr(field), H, W, value, dt, px, py, radius,
                                        APPROACHES[approach])


@dataclass
class EmitterSpec:
    """Fields of ``Emitter2D`` (common/emitters.py:106-137) that ``emit`` uses."""
    position: tuple
    radius: float
    density_value: float = 1.0
    temperature_value: float = 0.0
    velocity_value: tuple = (0.0, 0.0)
    approach: str = "linear"

    def emit(self, density, u, v, temperature, dt):
        """emitters.py:202-221: additive injection into each non-zero channel."""
        px, py = self.position
        if self.density_value != 0.0:
            emit_scalar(density, self.density_value, dt, px, py, self.radius, self.approach)
        if self.temperature_value != 0.0:
            emit_scalar(temperature, self.temperature_value, dt, px, py, self.radius, self.approach)
        if self.velocity_value[0] != 0.0:
            emit_scalar(u, self.velocity_value[0], dt, px, py, self.radius, self.approach)
        if self.velocity_value[1] != 0.0:
            emit_scalar(v, self.velocity_value[1], dt, px, py, self.radius, self.approach)


@dataclass
class PlumeSpec:
    """Overwriting disc source of the benchmark scenes (no reference counterpart)."""
    cx: float
    cy: float
    radius: float
    density_value: float = 1.0
    v_value: float = 1.0
    noise_amp: float = 0.0
    seed: int = 0

    def apply(self, density, u, v, step):
        H, W = density.shape
        _fn("or_plume_source", density.dtype)(_ptr(density), _ptr(u), _ptr(v), H, W, self.cx, self.cy,
                                               self.radius, self.density_value, self.v_value,
                                               self.noise_amp, self.seed, step)


# ---------------------------------------------------------------- substep
@dataclass
class OracleSim:
    """Restatement of ``SmokeSimulation2D`` state and ``substep`` (common/simulation.py:186-265).

    ``dtype`` may be float32 (what the reference allocates) or float64 (the
    reference kernels called directly on float64 arrays). ``solver`` is a
    callable with the ``PressureSolver`` signature. The solve uses ``self.dt``
    (simulation.py:311-312) while the other phases use the ``dt`` argument.
    """
    H: int
    W: int
    cell_size: float
    solver: object
    solver_kwargs: dict = field(default_factory=dict)
    dtype: object = np.float32
    dt: float = 0.016
    gravity: float = -0.5
    buoyancy: float = 5.0
    density_coefficient: float = 1.0
    fluid_density: float = 1.0
    density_dissipation: float = 0.999
    ambient_temperature: float = 0.0
    cooling_rate: float = 0.5
    f32_force_temporaries: bool = True

    def __post_init__(self):
        H, W, d = self.H, self.W, self.dtype
        z = lambda *s: np.zeros(s, d)
        self.density, self.density_temp = z(H, W), z(H, W)
        self.velocity_u, self.velocity_u_temp = z(H, W + 1), z(H, W + 1)
        self.velocity_v, self.velocity_v_temp = z(H + 1, W), z(H + 1, W)
        self.pressure = z(H, W)
        self.temperature, self.temperature_temp = z(H, W), z(H, W)
        self.divergence = z(H, W)
        self.pressure_residual = z(H, W)
        # simulation.py:102-113 builds the face masks from an all-fluid solid mask,
        # then _init_boundaries (:126-131) paints the 1-cell solid ring into the solid
        # mask only: until set_solid_mask() is called the solve sees every interior
        # face open and the ring acts only through enforce_boundary_conditions.
        self.fmu, self.fmv = face_masks_from_solid(np.zeros((H, W), bool))
        self.is_fluid = is_fluid_from_faces(self.fmu, self.fmv)
        self.solid = box_solid(H, W)
        self.emitters = []
        self.plumes = []
        self.step_index = 0

    def set_solid_mask(self, solid):
        """simulation.py:133-143 plus the rebuild at the next substep (:198-204)."""
        self.solid = np.ascontiguousarray(solid.astype(bool))
        self.fmu, self.fmv = face_masks_from_solid(self.solid)
        self.is_fluid = is_fluid_from_faces(self.fmu, self.fmv)

    def substep(self, dt):
        for e in self.emitters:
            e.emit(self.density, self.velocity_u, self.velocity_v, self.temperature, dt)
        for s in self.plumes:
            s.apply(self.density, self.velocity_u, self.velocity_v, self.step_index)
        apply_forces(self.velocity_v, self.density, self.temperature, dt, self.gravity, self.buoyancy,
                     self.density_coefficient, self.ambient_temperature, self.f32_force_temporaries)
        advect_velocity_u(self.velocity_u, self.velocity_u_temp, self.velocity_v, self.fmu, dt,
                          self.cell_size)
        advect_velocity_v(self.velocity_v, self.velocity_v_temp, self.velocity_u, self.fmv, dt,
                          self.cell_size)
        self.velocity_u, self.velocity_u_temp = self.velocity_u_temp, self.velocity_u
        self.velocity_v, self.velocity_v_temp = self.velocity_v_temp, self.velocity_v
        advect_scalar_field(self.density, self.density_temp, self.velocity_u, self.velocity_v,
                            self.is_fluid, dt, self.cell_size)
        self.density, self.density_temp = self.density_temp, self.density
        advect_scalar_field(self.temperature, self.temperature_temp, self.velocity_u, self.velocity_v,
                            self.is_fluid, dt, self.cell_size)
        self.temperature, self.temperature_temp = self.temperature_temp, self.temperature
        cool_temperature(self.temperature, self.ambient_temperature, self.cooling_rate, dt)
        self.density *= self.density_dissipation
        compute_divergence(self.velocity_u, self.velocity_v, self.divergence, self.fmu, self.fmv,
                           self.cell_size)
        self.pressure.fill(0.0)
        self.solver(self.pressure, self.divergence, self.fmu, self.fmv, self.fluid_density,
                    self.cell_size, self.dt, **self.solver_kwargs)
        apply_pressure_gradient(self.velocity_u, self.velocity_v, self.pressure, self.fmu, self.fmv,
                                self.fluid_density, self.cell_size, dt)
        enforce_boundary_conditions(self.velocity_u, self.velocity_v, self.solid)
        compute_divergence(self.velocity_u, self.velocity_v, self.divergence, self.fmu, self.fmv,
                           self.cell_size)
        compute_residual(self.pressure, self.divergence, self.is_fluid, self.fmu, self.fmv,
                         alpha_coeff(self.cell_size, self.fluid_density, dt), reciprocal_beta(),
                         self.pressure_residual)
        self.step_index += 1


# ---------------------------------------------------------------- convergent multigrid
def gmg_coarsen_fluid(fluid):
    """Any-fluid 2x2 coarsening; odd extents round up (the missing child is not fluid)."""
    H, W = fluid.shape
    Hc, Wc = (H + 1) // 2, (W + 1) // 2
    f = np.zeros((2 * Hc, 2 * Wc), bool)
    f[:H, :W] = fluid
    return f.reshape(Hc, 2, Wc, 2).any(axis=(1, 3))


def gmg_faces(fluid):
    """A face is open when both neighbouring cells are fluid; outer faces are closed."""
    H, W = fluid.shape
    fmu = np.zeros((H, W + 1), bool)
    fmv = np.zeros((H + 1, W), bool)
    fmu[:, 1:-1] = fluid[:, :-1] & fluid[:, 1:]
    fmv[1:-1, :] = fluid[:-1, :] & fluid[1:, :]
    return fmu, fmv


def gmg_apply(p, fluid, fmu, fmv):
    """A p = sum over open faces of (p - p_nb), on fluid cells."""
    out = np.zeros_like(p)
    out[:, 1:] += fmu[:, 1:-1] * (p[:, 1:] - p[:, :-1])
    out[:, :-1] += fmu[:, 1:-1] * (p[:, :-1] - p[:, 1:])
    out[1:, :] += fmv[1:-1, :] * (p[1:, :] - p[:-1, :])
    out[:-1, :] += fmv[1:-1, :] * (p[:-1, :] - p[1:, :])
    return out * fluid


class GMGOracle:
    """FP64 restatement of the project's convergent geometric multigrid.

    Level 0 uses the fine fluid/face masks of the simulation; coarser levels use
    any-fluid coarsening and faces open between two fluid cells. Smoother:
    red-black Gauss-Seidel with the exact diagonal (number of open faces) and
    over-relaxation ``omega``. Restriction is the transpose of bilinear
    prolongation (full weighting). The coarsest level is solved exactly with the
    pseudo-inverse of its operator after removing the rhs mean.
    """

    def __init__(self, fmu, fmv, fluid, coarsest=8, omega=1.3, pre=2, post=2, cycle="V"):
        self.levels = []
        f, cu, cv = fluid.astype(bool), fmu.astype(bool), fmv.astype(bool)
        while True:
            self.levels.append(dict(fluid=f, fmu=cu, fmv=cv))
            if max(f.shape) <= coarsest:
                break
            f = gmg_coarsen_fluid(f)
            cu, cv = gmg_faces(f)
        self.omega, self.pre, self.post, self.cycle = omega, pre, post, cycle
        L = self.levels[-1]
        H, W = L["fluid"].shape
        n = H * W
        # an open-box coarsest level above 64 x 64 cells: exact solve by the orthonormal
        # cosine transform (the operator's eigenbasis) instead of a dense pseudo-inverse
        self.coarse_dct = n > 4096 and bool(L["fluid"].all() and L["fmu"][:, 1:-1].all() and
                                             L["fmv"][1:-1, :].all() and not L["fmu"][:, [0, -1]].any() and
                                             not L["fmv"][[0, -1], :].any())
        if self.coarse_dct:
            lam = lambda m: 4.0 * np.sin(np.pi * np.arange(m) / (2.0 * m)) ** 2  # noqa: E731
            self.coarsest_lambda = lam(H)[:, None] + lam(W)[None, :]
            self.coarsest_lambda[0, 0] = np.inf  # the constant mode: zero, as the pseudo-inverse gives
            return
        A = np.zeros((n, n))
        for k in range(n):
            e = np.zeros(n)
            e[k] = 1.0
            A[:, k] = gmg_apply(e.reshape(H, W), L["fluid"], L["fmu"], L["fmv"]).ravel()
        self.coarsest_pinv = np.linalg.pinv(A)

    def _call(self, name, dtype, *args):
        return _fn(name, dtype)(*args)

    def residual(self, k, p, b, out):
        L = self.levels[k]
        H, W = p.shape
        _fn("or_gmg_residual", p.dtype)(_ptr(p), _ptr(b), _ptr(_mask(L["fluid"])), _ptr(_mask(L["fmu"])),
                                         _ptr(_mask(L["fmv"])), H, W, _ptr(out))
        return out

    def smooth(self, k, p, b, sweeps):
        L = self.levels[k]
        H, W = p.shape
        _fn("or_gmg_rbgs", p.dtype)(_ptr(p), _ptr(b), _ptr(_mask(L["fluid"])), _ptr(_mask(L["fmu"])),
                                     _ptr(_mask(L["fmv"])), H, W, self.omega, sweeps)

    def coarse_solve(self, b):
        L = self.levels[-1]
        if self.coarse_dct:
            from scipy.fft import dctn, idctn

            bh = dctn(b.astype(np.float64), type=2, norm="ortho")
            return idctn(bh / self.coarsest_lambda, type=2, norm="ortho")
        m = L["fluid"]
        bb = b.astype(np.float64).copy()
        if m.any():
            bb[m] -= bb[m].mean()
        bb[~m] = 0.0
        return (self.coarsest_pinv @ bb.ravel()).reshape(b.shape)

    def vcycle(self, k, e, b):
        """One cycle on A_k e = b from the guess e (in place)."""
        if k == len(self.levels) - 1:
            e[:] = self.coarse_solve(b).astype(e.dtype)
            return e
        L, C = self.levels[k], self.levels[k + 1]
        self.smooth(k, e, b, self.pre)
        r = self.residual(k, e, b, np.empty_like(e))
        Hc, Wc = C["fluid"].shape
        bc = np.empty((Hc, Wc), e.dtype)
        H, W = e.shape
        _fn("or_gmg_restrict_fw", e.dtype)(_ptr(r), _ptr(_mask(L["fluid"])), H, W, _ptr(bc),
                                            _ptr(_mask(C["fluid"])), Hc, Wc)
        ec = np.zeros_like(bc)
        self.vcycle(k + 1, ec, bc)
        if self.cycle == "W" and k + 1 < len(self.levels) - 1:
            self.vcycle(k + 1, ec, bc)
        _fn("or_gmg_prolong_add", e.dtype)(_ptr(ec), _ptr(_mask(C["fluid"])), Hc, Wc, _ptr(e),
                                            _ptr(_mask(L["fluid"])), H, W)
        self.smooth(k, e, b, self.post)
        return e

    def relres(self, p, b):
        r = self.residual(0, p, b, np.empty_like(p))
        nb = np.linalg.norm(b)
        return np.linalg.norm(r) / nb if nb > 0 else 0.0

    def solve(self, p, b, tol=1e-8, max_cycles=50, precision="fp64"):
        """Solve A p = b in place. precision: 'fp64' (cycles in FP64) or 'mixed'
        (FP64 residual and accumulation, FP32 cycles, FP64 coarsest solve).
        Returns (cycles, history of relative residuals)."""
        hist = [self.relres(p, b)]
        cycles = 0
        while hist[-1] > tol and cycles < max_cycles:
            if precision == "fp64":
                self.vcycle(0, p, b)
            else:
                r = self.residual(0, p, b, np.empty_like(p)).astype(np.float32)
                e = np.zeros_like(r)
                self.vcycle(0, e, r)
                p += e.astype(np.float64)
            cycles += 1
            hist.append(self.relres(p, b))
        return cycles, hist
