"""CUDA pressure solvers behind the reference's PressureSolver protocol.

Signature (src/cfd/solvers/base.py:5-19): ``fn(pressure, divergence, face_mask_u,
face_mask_v, fluid_density, cell_size, dt, **solver_kwargs)``; ``pressure`` is
updated in place and extra keyword arguments are ignored (jacobi.py:30).

Registered under backend "cuda": the reference's four methods (jacobi, gauss_seidel,
rb_sor_gauss_seidel, multigrid -- same arguments and iterates) and two methods the
reference lacks: rb_sor_tolerance and geometric_multigrid (convergent, FP32 / FP64 /
mixed precision).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import asdict

import numpy as np
import torch

from . import _lib as L
from .operators import AnalyticMask, OPEN_BOX, RING_BOX, _face_pair, _masks, build_masks, compute_residual
from .registry import get_solver, register_solver


# ---------------------------------------------------------------- coefficients (solvers/common.py)
def calculate_alpha(cell_size: float, density: float, dt: float) -> float:
    """solvers/common.py:6-18."""
    return (-(cell_size * cell_size) * density) / dt


def calculate_reciprocal_beta() -> float:
    """solvers/common.py:20-28."""
    return 0.25


def calculate_optimal_omega(size: int) -> float:
    """solvers/common.py:30-39."""
    return min(2.0 / (1.0 + math.sin(math.pi / size)), 1.95)


def is_fluid_from_faces(fmu, fmv):
    """common/simulation.py:108 (device tensors)."""
    return fmu[:, :-1] | fmu[:, 1:] | fmv[:-1, :] | fmv[1:, :]


def materialize_mask(m, H, W, which, device):
    """Turn an analytic mask sentinel into a bool plane (for code that needs planes)."""
    if not isinstance(m, AnalyticMask):
        return m
    solid = torch.zeros((H, W), dtype=torch.bool, device=device)
    if m is RING_BOX:
        solid[0, :] = solid[-1, :] = True
        solid[:, 0] = solid[:, -1] = True
    fmu, fmv, fl = build_masks(solid)
    return {"u": fmu, "v": fmv, "fluid": fl}[which]


# ---------------------------------------------------------------- reference methods
def jacobi_pressure_solver(pressure, divergence, face_mask_u, face_mask_v, fluid_density, cell_size, dt,
                           iterations, scratch=None, **_ignored):
    """jacobi.py:27-52: ``iterations`` ping-pong sweeps; the result ends in ``pressure``."""
    H, W = pressure.shape
    dtc = L.dtype_code(pressure)
    mode, pu, lu, pv, lv = _face_pair(face_mask_u, face_mask_v, H, W)
    if scratch is None:
        scratch = torch.empty((H, W), dtype=pressure.dtype, device=pressure.device)
    p, ldp = L.field(pressure, "pressure")
    d, ldd = L.field(divergence, "divergence", dtype=pressure.dtype)
    L.call("sg_jacobi_solve", dtc, H, W, p, ldp, d, ldd, mode, pu, lu, pv, lv,
           calculate_alpha(cell_size, fluid_density, dt), calculate_reciprocal_beta(), int(iterations),
           scratch.data_ptr(), L.stream_ptr())


def red_black_sor_gauss_seidel_pressure_solver(pressure, divergence, face_mask_u, face_mask_v, fluid_density,
                                               cell_size, dt, iterations, omega: float = 0.0, **_ignored):
    """red_black_sor_gauss_seidel.py:30-42 (omega <= 0 or > 2 selects the optimal omega)."""
    H, W = pressure.shape
    if omega <= 0.0 or omega > 2.0:
        omega = calculate_optimal_omega(max(H, W))
    mode, pu, lu, pv, lv = _face_pair(face_mask_u, face_mask_v, H, W)
    p, ldp = L.field(pressure, "pressure")
    d, ldd = L.field(divergence, "divergence", dtype=pressure.dtype)
    L.call("sg_rbsor_solve", L.dtype_code(pressure), H, W, p, ldp, d, ldd, mode, pu, lu, pv, lv,
           calculate_alpha(cell_size, fluid_density, dt), calculate_reciprocal_beta(), float(omega), int(iterations),
           L.stream_ptr())


def gauss_seidel_pressure_solver(pressure, divergence, face_mask_u, face_mask_v, fluid_density, cell_size, dt,
                                 iterations, **_ignored):
    """gauss_seidel.py:29-48 (lexicographic order, as anti-diagonal wavefronts in one block)."""
    H, W = pressure.shape
    mode, pu, lu, pv, lv = _face_pair(face_mask_u, face_mask_v, H, W)
    p, ldp = L.field(pressure, "pressure")
    d, ldd = L.field(divergence, "divergence", dtype=pressure.dtype)
    L.call("sg_gauss_seidel_solve", L.dtype_code(pressure), H, W, p, ldp, d, ldd, mode, pu, lu, pv, lv,
           calculate_alpha(cell_size, fluid_density, dt), calculate_reciprocal_beta(), int(iterations),
           L.stream_ptr())


class MultigridSolver:
    """The reference's V-cycle (multigrid/solver.py:16-176) on CUDA kernels.

    Same hierarchy (any-solid coarsening from ``solid = ~is_fluid`` while both extents
    are even, :34-73), same cycle (smooth, residual, mean-of-fluid-children
    restriction, rhs / alpha(2h), zero-guess recursion, clamped bilinear
    prolongation added to the pressure, smooth; :94-139) and same smoother lookup
    through the registry. The cache is keyed on shape, level count and dtype.
    A smoother backend of "numba" maps to the CUDA smoother of the same name.
    """

    def __init__(self):
        self._key = None
        self.levels = []
        self.buffers = []

    def _ensure(self, H, W, fmu, fmv, num_levels, dtype, device, rebuild):
        kind = fmu.name if isinstance(fmu, AnalyticMask) else "planes"
        key = ((H, W + 1), num_levels, dtype, kind)
        if not rebuild and key == self._key:
            return
        fmu = materialize_mask(fmu, H, W, "u", device)
        fmv = materialize_mask(fmv, H, W, "v", device)
        fl = is_fluid_from_faces(fmu.bool(), fmv.bool())
        solid = ~fl
        levels = [dict(is_fluid=fl, fmu=fmu, fmv=fmv, solid=solid)]
        for _ in range(1, num_levels):
            h, w = solid.shape
            if h % 2 or w % 2:
                break
            sc = torch.empty((h // 2, w // 2), dtype=torch.uint8, device=device)
            s8 = solid.to(torch.uint8).contiguous()
            L.call("sg_mg_coarsen_solid", h, w, s8.data_ptr(), w, sc.data_ptr(), w // 2, L.stream_ptr())
            cu, cv, cf = build_masks(sc.bool())
            levels.append(dict(is_fluid=cf, fmu=cu, fmv=cv, solid=sc.bool()))
            solid = sc.bool()
        self.levels = levels
        self.buffers = [{k: torch.zeros(lv["is_fluid"].shape, dtype=dtype, device=device)
                         for k in ("pressure", "residual", "rhs")} for lv in levels]
        self._key = key

    def _v_cycle(self, k, p, rhs, rho, h, dt, smoother, nu, nu_c):
        lv = self.levels[k]
        buf = self.buffers[k]
        coarsest = k == len(self.levels) - 1
        smoother(p, rhs, lv["fmu"], lv["fmv"], rho, h, dt, nu_c if coarsest else nu)
        if coarsest:
            return p
        H, W = p.shape
        alpha = calculate_alpha(h, rho, dt)
        compute_residual(p, rhs, lv["is_fluid"], lv["fmu"], lv["fmv"], alpha, calculate_reciprocal_beta(),
                         buf["residual"])
        cb = self.buffers[k + 1]
        Hc, Wc = cb["rhs"].shape
        fpl, fld = L.mask_plane(lv["is_fluid"], "is_fluid", (H, W))
        L.call("sg_mg_restrict_average", L.dtype_code(p), H, W, buf["residual"].data_ptr(), W, L.SG_MASK_PLANES, fpl,
               fld, cb["rhs"].data_ptr(), Wc, Hc, Wc, calculate_alpha(h * 2.0, rho, dt), L.stream_ptr())
        cb["pressure"].zero_()
        self._v_cycle(k + 1, cb["pressure"], cb["rhs"], rho, h * 2.0, dt, smoother, nu, nu_c)
        pp, ldp = L.field(p, "pressure")
        L.call("sg_mg_prolong", L.dtype_code(p), Hc, Wc, cb["pressure"].data_ptr(), Wc, H, W, L.SG_MASK_PLANES, fpl, fld,
               pp, ldp, 1, L.stream_ptr())
        smoother(p, rhs, lv["fmu"], lv["fmv"], rho, h, dt, nu)
        return p

    def __call__(self, pressure, divergence, face_mask_u, face_mask_v, fluid_density, cell_size, dt, v_cycles=2,
                 smoother_type="jacobi", smoother_backend="cuda", num_levels=4, smoother_iterations=2,
                 coarsest_iterations=50, rebuild_masks=False, profiler=None, **_ignored):
        H, W = pressure.shape
        self._ensure(H, W, face_mask_u, face_mask_v, num_levels, pressure.dtype, pressure.device, rebuild_masks)
        backend = smoother_backend if smoother_backend == "cuda" else "cuda"
        smoother = get_solver(smoother_type, backend)
        fb = self.buffers[0]
        fb["pressure"].copy_(pressure)
        fb["rhs"].copy_(divergence)
        for _ in range(v_cycles):
            self._v_cycle(0, fb["pressure"], fb["rhs"], fluid_density, cell_size, dt, smoother, smoother_iterations,
                          coarsest_iterations)
        pressure.copy_(fb["pressure"])


# ---------------------------------------------------------------- new methods
class SORToleranceSolver:
    """Red-black SOR until ||r(p)|| / ||r(0)|| <= tol over fluid cells, with r the
    reference residual (residual.py:39-40), on the checkerboard-split layout: red and
    black cells in separate contiguous planes, the residual norm checked every
    ``check_every`` sweeps. The iterates are the reference kernel's
    (red_black_sor_gauss_seidel.py:8-27) bit for bit; the tolerance loop has no reference
    counterpart (the reference runs a fixed sweep count). ``variant``: 1 sweeps
    shared-memory tiles up to four sweeps per launch, 0 launches one streaming kernel per
    half sweep, -1 (default) picks the tiles for grids that sit in L2 and the streaming
    kernel above.

    ``precision="mixed"`` (float32 fields): float64 iterative refinement around float32
    sweeps (``sg_rbsor_mixed_solve``), which reaches tolerances below float32's residual
    floor; ``last_refinements`` counts the refinements."""

    def __init__(self):
        self.last_iterations = 0
        self.last_relres = None
        self.last_refinements = 0
        self.converged = None
        self._ws = None

    def workspace(self, nbytes, device):
        if self._ws is None or self._ws.numel() < nbytes + 256 or self._ws.device != torch.device(device):
            self._ws = torch.empty(nbytes + 256, dtype=torch.uint8, device=device)
        base = self._ws.data_ptr()
        off = (-base) % 256
        return ctypes.c_void_p(base + off), self._ws.numel() - off

    def __call__(self, pressure, divergence, face_mask_u, face_mask_v, fluid_density, cell_size, dt, omega=1.9,
                 tol=1e-6, max_iterations=200000, check_every=100, strict=False, variant=-1, precision="native",
                 **_ignored):
        H, W = pressure.shape
        alpha = calculate_alpha(cell_size, fluid_density, dt)
        mode, pu, lu, pv, lv = _face_pair(face_mask_u, face_mask_v, H, W)
        p, ldp = L.field(pressure, "pressure")
        d, ldd = L.field(divergence, "divergence", dtype=pressure.dtype)
        lib = L.load()
        its = ctypes.c_int64(0)
        refs = ctypes.c_int64(0)
        rel = ctypes.c_double(0.0)
        if precision == "mixed":
            if pressure.dtype != torch.float32:
                raise TypeError("precision='mixed' refines a float32 pressure; a float64 one needs no refinement")
            ws, nbytes = self.workspace(int(lib.sg_rbsor_mixed_workspace_bytes(H, W)), pressure.device)
            rc = lib.sg_rbsor_mixed_solve(H, W, p, ldp, d, ldd, mode, pu, lu, pv, lv, alpha,
                                          calculate_reciprocal_beta(), float(omega), float(tol), int(max_iterations),
                                          int(check_every), int(variant), ws, nbytes, ctypes.byref(its),
                                          ctypes.byref(rel), ctypes.byref(refs), L.stream_ptr())
            name = "sg_rbsor_mixed_solve"
        elif precision == "native":
            code = L.dtype_code(pressure)
            ws, nbytes = self.workspace(int(lib.sg_rbsor_split_workspace_bytes(code, H, W)), pressure.device)
            rc = lib.sg_rbsor_tol_solve(code, H, W, p, ldp, d, ldd, mode, pu, lu, pv, lv, alpha,
                                        calculate_reciprocal_beta(), float(omega), float(tol), int(max_iterations),
                                        int(check_every), int(variant), ws, nbytes, ctypes.byref(its),
                                        ctypes.byref(rel), L.stream_ptr())
            name = "sg_rbsor_tol_solve"
        else:
            raise ValueError(f"precision must be 'native' or 'mixed', got {precision!r}")
        self.last_iterations, self.last_relres = int(its.value), float(rel.value)
        self.last_refinements = int(refs.value)
        self.converged = rc == L.SG_OK
        if rc == L.SG_ERR_NOT_CONVERGED:
            if strict:
                raise L.NotConverged(f"SOR relative residual {self.last_relres:.3e} > {tol:.3e} after "
                                     f"{self.last_iterations} sweeps", self.last_iterations, self.last_relres)
            return
        L.check(rc, name)


_PRECISION = {"fp32": L.SG_GMG_FP32, "fp64": L.SG_GMG_FP64, "mixed": L.SG_GMG_MIXED}


class GMGPlan:
    """A bound multigrid plan (host plan + device workspace) for one grid and mask."""

    def __init__(self, H, W, fmu, fmv, device, coarsest=8, omega=1.3, pre=2, post=2, cycle="V", precision="fp64",
                 remove_mean=False, inner_cycles=1):
        lib = L.load()
        self.H, self.W, self.precision = H, W, precision
        handle = ctypes.c_void_p()
        if isinstance(fmu, AnalyticMask):
            mode, a, b, c = fmu.mode, None, None, None
            self._host = None
        else:
            fu = fmu.to(torch.uint8).cpu().numpy()
            fv = fmv.to(torch.uint8).cpu().numpy()
            fl = (fu[:, :-1] | fu[:, 1:] | fv[:-1, :] | fv[1:, :]).astype(np.uint8)
            self._host = [np.ascontiguousarray(x) for x in (fl, fu, fv)]
            mode = L.SG_MASK_PLANES
            a, b, c = (x.ctypes.data_as(ctypes.c_void_p) for x in self._host)
        L.check(lib.sg_gmg_plan_create(ctypes.byref(handle), H, W, mode, a, b, c, int(coarsest), float(omega), int(pre),
                                       int(post), 0 if cycle.upper() == "V" else 1, _PRECISION[precision]),
                "sg_gmg_plan_create")
        self.handle = handle
        L.check(lib.sg_gmg_set_remove_mean(handle, 1 if remove_mean else 0), "sg_gmg_set_remove_mean")
        L.check(lib.sg_gmg_set_inner_cycles(handle, int(inner_cycles)), "sg_gmg_set_inner_cycles")
        nbytes = lib.sg_gmg_workspace_bytes(handle)
        self.workspace = torch.empty(int(nbytes), dtype=torch.uint8, device=device)
        L.check(lib.sg_gmg_bind(handle, self.workspace.data_ptr(), L.stream_ptr()), "sg_gmg_bind")
        self.num_levels = lib.sg_gmg_num_levels(handle)
        self.workspace_bytes = int(nbytes)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value and L._lib is not None:
            L._lib.sg_gmg_plan_destroy(h)
            self.handle = None

    def solve_async(self, pressure, divergence, alpha, tol, max_cycles, zero_guess=False):
        """Graph solve without host synchronisation (outcome: stats()). zero_guess: start
        from p = 0 without reading `pressure` (it is only written)."""
        p, ldp = L.field(pressure, "pressure")
        d, ldd = L.field(divergence, "divergence")
        L.call("sg_gmg_solve_from_zero_async" if zero_guess else "sg_gmg_solve_async", self.handle, p, ldp, d, ldd,
               L.dtype_code(divergence), float(alpha), float(tol), int(max_cycles), L.stream_ptr())

    def stats(self):
        """(cycles, relres, status, total_cycles) of the last solve; synchronises the stream."""
        c, s = ctypes.c_int(0), ctypes.c_int(0)
        r = ctypes.c_double(0.0)
        t = ctypes.c_longlong(0)
        L.call("sg_gmg_stats", self.handle, ctypes.byref(c), ctypes.byref(r), ctypes.byref(s), ctypes.byref(t),
               L.stream_ptr())
        return c.value, r.value, s.value, t.value

    def counters(self):
        """(solves, cycles, failures) since the plan was bound; synchronises the stream."""
        a, b, c = ctypes.c_longlong(0), ctypes.c_longlong(0), ctypes.c_longlong(0)
        L.call("sg_gmg_counters", self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), L.stream_ptr())
        return a.value, b.value, c.value

    def graph_nodes(self):
        a, b = ctypes.c_int(0), ctypes.c_int(0)
        L.call("sg_gmg_graph_nodes", self.handle, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def tail_start(self):
        return L.load().sg_gmg_tail_start(self.handle)

    def level_shape(self, level):
        """(H, W) of one level of the hierarchy (0 is the fine grid)."""
        h, w = ctypes.c_int(0), ctypes.c_int(0)
        L.call("sg_gmg_level_shape", self.handle, int(level), ctypes.byref(h), ctypes.byref(w))
        return h.value, w.value

    def relres_async(self, dst, stream=None):
        """Enqueue a copy of the last solve's relative residual into `dst` (one float64,
        pinned host or CUDA tensor) on `stream`; no synchronisation."""
        L.call("sg_gmg_relres_async", self.handle, ctypes.c_void_p(dst.data_ptr()), L.stream_ptr(stream))

    def fine_fused(self):
        """True when the fine level runs the fused register-tiled pre/post kernels."""
        return bool(L.load().sg_gmg_fine_fused(self.handle))

    COARSE_SOLVE_KINDS = ("pseudo-inverse", "cosine transform (one block)", "cosine transform (four products)",
                          "cosine transform (two streaming launches)",
                          "cosine transform (two streaming launches on 4-CTA clusters)")

    def set_post_events(self, events):
        """Record the torch.cuda.Events (timing enabled, each already recorded once so that it
        exists) in pairs around the next len(events) // 2 fused fine-level post launches of
        kernel-by-kernel solves; an empty list clears it."""
        n = len(events) // 2
        arr = (ctypes.c_void_p * max(2 * n, 1))(*[ctypes.c_void_p(e.cuda_event) for e in events[:2 * n]])
        L.call("sg_gmg_set_post_events", self.handle, arr, n)

    def coarse_solve_kind(self):
        """How the coarsest level is solved (one of COARSE_SOLVE_KINDS)."""
        return self.COARSE_SOLVE_KINDS[L.load().sg_gmg_coarse_solve_kind(self.handle)]

    def fine_kernel_async(self, which, pressure=None):
        """Launch the fused fine-level pre (0) or post (1) kernel once on the workspace as it
        stands (for timing the dominant kernels alone; the post kernel adds to `pressure`)."""
        p, ldp = L.field(pressure, "pressure") if pressure is not None else (None, 0)
        L.call("sg_gmg_fine_kernel_async", self.handle, int(which), p, ldp, L.stream_ptr())

    def cycles_async(self, pressure, divergence, alpha, n_cycles, relres_out):
        p, ldp = L.field(pressure, "pressure")
        d, ldd = L.field(divergence, "divergence")
        L.call("sg_gmg_cycles_async", self.handle, p, ldp, d, ldd, L.dtype_code(divergence), float(alpha), int(n_cycles),
               ctypes.cast(relres_out.data_ptr(), L.PD), L.stream_ptr())


class GeometricMultigridSolver:
    """Convergent geometric multigrid; see ``sg_gmg_*`` in include/smoke_b200.h.

    ``precision``: "fp32" (pressure float32), "fp64" or "mixed" (pressure float64; the
    mixed path runs FP32 cycles inside FP64 iterative refinement). A pressure tensor
    of another dtype is solved through an internal buffer kept across calls. A solve is
    one CUDA graph launch (tolerance loop on the device); the outcome (``last_cycles``,
    ``last_relres``, ``converged``) is read from the device only when asked for, and
    ``strict=True`` reads it at once and raises NotConverged / SmokeCudaError. With
    ``fixed_cycles > 0`` exactly that many cycles run kernel by kernel (capturable);
    per-cycle relative residuals then stay on the device in ``last_relres_dev``.
    ``inner_cycles`` k >= 2 (mixed precision): classical iterative refinement, k FP32 cycles
    on the correction from zero between two FP64 passes (p += e, residual), instead of the
    fused fine level that corrects p and updates the FP64 residual every cycle; the cycle
    counts then grow in steps of k.
    """

    def __init__(self):
        self._plans = {}
        self._pending = None
        self._last = (0, None, None)
        self.last_relres_dev = None
        self._buffers = {}

    def _outcome(self):
        if self._pending is not None:
            cycles, rel, status, _ = self._pending.stats()
            self._pending = None
            if status == 3:
                self._last = (cycles, rel, False)
                raise L.SmokeCudaError(f"multigrid: non-finite residual after {cycles} cycles")
            if status == 4:
                self._last = (cycles, rel, False)
                raise L.SmokeCudaError("multigrid: a bounded device wait gave up (a bulk copy never landed)")
            self._last = (cycles, rel, status == 1)
        return self._last

    @property
    def last_cycles(self):
        return self._outcome()[0]

    @property
    def last_relres(self):
        return self._outcome()[1]

    @property
    def converged(self):
        return self._outcome()[2]

    def current_plan(self):
        return next(iter(self._plans.values()), None)

    def plan_for(self, H, W, fmu, fmv, device, coarsest, omega, pre, post, cycle, precision, rebuild=False,
                 remove_mean=False, inner_cycles=1):
        if isinstance(fmu, AnalyticMask):
            mkey = ("analytic", fmu.mode)
        else:
            mkey = (fmu.data_ptr(), fmu._version, fmv.data_ptr(), fmv._version)
        key = (H, W, mkey, coarsest, omega, pre, post, cycle, precision, str(device), bool(remove_mean),
               int(inner_cycles))
        plan = self._plans.get(key)
        if plan is None or rebuild:
            plan = GMGPlan(H, W, fmu, fmv, device, coarsest, omega, pre, post, cycle, precision, remove_mean,
                           inner_cycles)
            self._plans = {key: plan}
        return plan

    def __call__(self, pressure, divergence, face_mask_u, face_mask_v, fluid_density, cell_size, dt, tol=1e-6,
                 max_cycles=50, cycle="V", pre_sweeps=2, post_sweeps=2, omega=1.3, coarsest=8, precision="fp64",
                 check_every=1, fixed_cycles=0, rebuild_masks=False, strict=False, zero_initial_guess=False,
                 remove_mean=False, inner_cycles=1, **_ignored):
        H, W = pressure.shape
        plan = self.plan_for(H, W, face_mask_u, face_mask_v, pressure.device, coarsest, omega, pre_sweeps, post_sweeps,
                             cycle, precision, rebuild_masks, remove_mean, inner_cycles)
        want = torch.float32 if precision == "fp32" else torch.float64
        if pressure.dtype == want:
            p = pressure
        else:
            key = (H, W, want, str(pressure.device))
            p = self._buffers.get(key)
            if p is None:
                p = torch.empty((H, W), dtype=want, device=pressure.device)
                self._buffers = {key: p}
            if not zero_initial_guess or fixed_cycles:
                p.copy_(pressure)
        alpha = calculate_alpha(cell_size, fluid_density, dt)
        self._pending = None
        if fixed_cycles and fixed_cycles > 0:
            if self.last_relres_dev is None or self.last_relres_dev.numel() != fixed_cycles + 1:
                self.last_relres_dev = torch.zeros(fixed_cycles + 1, dtype=torch.float64, device=pressure.device)
            plan.cycles_async(p, divergence, alpha, fixed_cycles, self.last_relres_dev)
            self._last = (fixed_cycles, None, None)
        else:
            plan.solve_async(p, divergence, alpha, tol, max_cycles, zero_guess=bool(zero_initial_guess))
            self._pending = plan
            if strict:
                cycles, rel, ok = self._outcome()
                if not ok:
                    raise L.NotConverged(f"multigrid relative residual {rel:.3e} > {tol:.3e} after {cycles} cycles",
                                         cycles, rel)
        if p is not pressure:
            pressure.copy_(p)


# ---------------------------------------------------------------- dispatch + registration
def solve_pressure(pressure, divergence, face_mask_u, face_mask_v, fluid_density, cell_size, dt, params, **hints):
    """solvers/dispatch.py:5-12: look up (method, backend) and call with the params as kwargs.
    ``hints`` (e.g. zero_initial_guess=True from a caller that just zeroed the pressure) are
    passed along; solvers that do not use them ignore them."""
    fn = get_solver(params.pressure_solver_method, params.pressure_solver_backend)
    kwargs = asdict(params.solver_params)
    kwargs.update(hints)
    fn(pressure, divergence, face_mask_u, face_mask_v, fluid_density, cell_size, dt,
       profiler=getattr(params, "profiler", None), **kwargs)


_registered = False


def register_solvers():
    """Register the CUDA solvers under backend "cuda" (idempotent)."""
    global _registered
    if _registered:
        return
    register_solver("jacobi", "cuda", jacobi_pressure_solver)
    register_solver("gauss_seidel", "cuda", gauss_seidel_pressure_solver)
    register_solver("rb_sor_gauss_seidel", "cuda", red_black_sor_gauss_seidel_pressure_solver)
    register_solver("multigrid", "cuda", MultigridSolver())
    register_solver("rb_sor_tolerance", "cuda", SORToleranceSolver())
    register_solver("geometric_multigrid", "cuda", GeometricMultigridSolver())
    _registered = True
