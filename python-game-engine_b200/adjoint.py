"""Differentiable smoke rollouts with hand-written adjoint kernels.

The step is SmokeSimulation2D.substep (common/simulation.py:186-265) on the default scene
(kernel masks of the open box, a solid ring for the boundary zeroing) with overwriting plume
sources and a per-step control force (fu, fv), H x W each, added to the left / lower face
of every cell right after the buoyancy force:

    plume -> buoyancy + dt * control -> velocity self-advection -> density advection with the
    advected velocity (and dissipation) -> divergence -> pressure solve -> projection.

``SmokeStep`` is a torch.autograd.Function over one step whose backward runs the adjoint
kernels of libsmoke_b200 (sg_adjoint_*) and the same multigrid solve for the pressure's
adjoint; ``rollout`` chains steps with a checkpoint every k steps (torch.utils.checkpoint,
which recomputes each segment's steps during the backward pass), so a rollout holds k
steps' intermediates at a time. The reference has no differentiation; gradients are checked
against central finite differences of the forward and against an FP64 PyTorch-autodiff
restatement of the step (tests).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch
from torch.utils.checkpoint import checkpoint

from . import _lib as L
from . import operators as ops
from .operators import OPEN_BOX, RING_BOX
from .solvers import GeometricMultigridSolver

_GATHER = {"scatter": 0, "gather": 1}


@dataclass
class ControlledSmoke:
    """A fixed scene for differentiable rollouts.

    plumes: (n, 6) host rows (cx, cy, r, density, v, noise) in cell units, overwritten every
    step; dtype float32 or float64; precision / tol of the multigrid pressure solves (the
    forward and the adjoint use the same); adjoint_advection "scatter" (atomicAdd) or
    "gather" (deterministic). exact_forces: evaluate the buoyancy in the field precision
    rather than through the reference's float32 temporaries (keeps FP64 runs smooth enough
    for finite differences). fixed_cycles > 0: every solve runs exactly that many cycles (a
    fixed linear map; with enough cycles, the exact solve to rounding)."""

    H: int
    W: int
    cell_size: float
    dt: float
    gravity: float = -1.0
    plumes: np.ndarray = None
    seed: int = 0
    dtype: torch.dtype = torch.float32
    device: torch.device = None
    precision: str = "fp32"
    tol: float = 1e-6
    max_cycles: int = 60
    fixed_cycles: int = 0
    fluid_density: float = 1.0
    buoyancy: float = 0.0
    density_coefficient: float = 1.0
    dissipation: float = 0.999
    adjoint_advection: str = "scatter"
    exact_forces: bool = False

    def __post_init__(self):
        if self.device is None:
            self.device = torch.device("cuda")
        if self.adjoint_advection not in _GATHER:
            raise ValueError("adjoint_advection must be 'scatter' or 'gather'")
        self.plumes = np.ascontiguousarray(np.asarray(self.plumes if self.plumes is not None else np.zeros((0, 6)),
                                                      dtype=np.float64).reshape(-1, 6))
        # the adjoint of an overwriting source zeroes the adjoint where it wrote
        self._zero_plumes = self.plumes.copy()
        self._zero_plumes[:, 3:6] = 0.0
        self.solver = GeometricMultigridSolver()
        self._ws = None

    # ------------------------------------------------------------------ helpers
    def zeros_state(self):
        z = lambda *s: torch.zeros(s, dtype=self.dtype, device=self.device)  # noqa: E731
        return z(self.H, self.W), z(self.H, self.W + 1), z(self.H + 1, self.W)

    def _solve(self, out, rhs):
        out.zero_()
        self.solver(out, rhs, OPEN_BOX, OPEN_BOX, self.fluid_density, self.cell_size, self.dt, tol=self.tol,
                    max_cycles=self.max_cycles, precision=self.precision, fixed_cycles=self.fixed_cycles)

    def _workspace(self):
        gather = _GATHER[self.adjoint_advection]
        n = L.load().sg_adjoint_advect_scalar_workspace(L.dtype_code(torch.empty(0, dtype=self.dtype)), self.H, self.W,
                                                        gather)
        if self._ws is None or self._ws.numel() < n:
            self._ws = torch.empty(n, dtype=torch.uint8, device=self.device)
        return self._ws

    # ------------------------------------------------------------------ forward
    @torch.no_grad()
    def forward_step(self, d, u, v, fu, fv, t):
        """One step from (d, u, v) under control (fu, fv) at step index t; returns the new
        state and the intermediates the adjoint needs."""
        H, W, h, dt = self.H, self.W, self.cell_size, self.dt
        code = L.dtype_code(d)
        d1, u1, v1 = d.clone(), u.clone(), v.clone()
        if len(self.plumes):
            ops.plume_sources(d1, u1, v1, self.plumes, self.seed, t)
        ops.apply_forces(v1, d1, None, dt, self.gravity, self.buoyancy, self.density_coefficient, 0.0,
                         f32_temporaries=not self.exact_forces)
        pu, lu = L.field(u1, "u")
        pv, lv = L.field(v1, "v")
        pfu, lfu = L.field(fu.contiguous(), "fu")
        pfv, lfv = L.field(fv.contiguous(), "fv")
        L.call("sg_add_control", code, H, W, pu, lu, pv, lv, pfu, lfu, pfv, lfv, float(dt), L.stream_ptr())
        u2, v2 = torch.empty_like(u1), torch.empty_like(v1)
        ops.advect_velocity(u1, u2, v1, v2, OPEN_BOX, OPEN_BOX, dt, h)
        d2 = torch.empty_like(d1)
        ops.advect_scalar_field(d1, d2, u2, v2, OPEN_BOX, dt, h, dissipation=self.dissipation)
        div = torch.empty_like(d1)
        ops.compute_divergence(u2, v2, div, OPEN_BOX, OPEN_BOX, h)
        p = torch.empty((H, W), dtype=torch.float32 if self.precision == "fp32" else torch.float64,
                        device=self.device)
        self._solve(p, div)
        u3, v3 = u2.clone(), v2.clone()
        ops.project(u3, v3, p.to(self.dtype), OPEN_BOX, OPEN_BOX, RING_BOX, self.fluid_density, h, dt)
        return (d2, u3, v3), (d1, u1, v1, u2, v2)

    # ------------------------------------------------------------------ adjoint
    @torch.no_grad()
    def adjoint_step(self, saved, t, lam_d2, lam_u3, lam_v3):
        """Adjoints of the step's input state and control from those of its output."""
        d1, u1, v1, u2, v2 = saved
        H, W, h, dt = self.H, self.W, self.cell_size, self.dt
        code = L.dtype_code(d1)
        sp = L.stream_ptr()
        lam_d2, lam_u3, lam_v3 = lam_d2.contiguous(), lam_u3.contiguous(), lam_v3.contiguous()
        # projection: identity part and the pressure's adjoint, then the same solve
        lam_u2, lam_v2 = torch.empty_like(u2), torch.empty_like(v2)
        lam_p = torch.empty_like(d1)
        a = [L.field(x, "lam")[0] for x in (lam_u3, lam_v3, lam_u2, lam_v2, lam_p)]
        L.call("sg_adjoint_project", code, H, W, a[0], W + 1, a[1], W, a[2], W + 1, a[3], W, a[4], W, L.SG_MASK_OPEN,
               None, 0, None, 0, L.SG_MASK_RING, None, 0, float(self.fluid_density), float(h), float(dt), sp)
        lam_div = torch.empty((H, W), dtype=torch.float32 if self.precision == "fp32" else torch.float64,
                              device=self.device)
        self._solve(lam_div, lam_p)
        lam_div = lam_div.to(self.dtype)
        L.call("sg_adjoint_divergence", code, H, W, L.field(lam_div)[0], W, a[2], W + 1, a[3], W, L.SG_MASK_OPEN,
               None, 0, None, 0, float(h), sp)
        # density advection (with the advected velocity)
        lam_d1 = torch.zeros_like(d1)
        ws = self._workspace()
        L.call("sg_adjoint_advect_scalar", code, H, W, L.field(lam_d2)[0], W, L.field(d1)[0], W, L.field(u2)[0], W + 1,
               L.field(v2)[0], W, L.SG_MASK_OPEN, None, 0, float(dt), float(h), float(self.dissipation),
               L.field(lam_d1)[0], W, a[2], W + 1, a[3], W, _GATHER[self.adjoint_advection],
               ws.data_ptr(), ws.numel(), sp)
        # velocity self-advection
        lam_u1, lam_v1 = torch.zeros_like(u1), torch.zeros_like(v1)
        L.call("sg_adjoint_advect_velocity", code, H, W, a[2], W + 1, a[3], W, L.field(u1)[0], W + 1,
               L.field(v1)[0], W, L.SG_MASK_OPEN, None, 0, None, 0, float(dt), float(h), L.field(lam_u1)[0], W + 1,
               L.field(lam_v1)[0], W, sp)
        # control and buoyancy
        gfu, gfv = torch.empty_like(d1), torch.empty_like(d1)
        L.call("sg_adjoint_forces", code, H, W, L.field(lam_u1)[0], W + 1, L.field(lam_v1)[0], W, L.field(lam_d1)[0],
               W, L.field(gfu)[0], W, L.field(gfv)[0], W, float(dt), float(self.gravity),
               float(self.density_coefficient), sp)
        # overwriting sources: nothing before the step reaches the cells they wrote
        if len(self.plumes):
            ops.plume_sources(lam_d1, lam_u1, lam_v1, self._zero_plumes, self.seed, t)
        return lam_d1, lam_u1, lam_v1, gfu, gfv


class SmokeStep(torch.autograd.Function):
    """(d, u, v, fu, fv) -> (d', u', v') for one step of ``model`` at step index t."""

    @staticmethod
    def forward(ctx, d, u, v, fu, fv, model, t):
        (d2, u3, v3), saved = model.forward_step(d, u, v, fu, fv, t)
        ctx.model, ctx.t = model, t
        ctx.save_for_backward(*saved)
        return d2, u3, v3

    @staticmethod
    def backward(ctx, gd, gu, gv):
        model = ctx.model
        saved = ctx.saved_tensors
        d1, u1, v1 = saved[0], saved[1], saved[2]
        gd = torch.zeros_like(d1) if gd is None else gd
        gu = torch.zeros_like(u1) if gu is None else gu
        gv = torch.zeros_like(v1) if gv is None else gv
        ld, lu, lv, gfu, gfv = model.adjoint_step(saved, ctx.t, gd, gu, gv)
        return ld, lu, lv, gfu, gfv, None, None


def rollout(model: ControlledSmoke, d0, u0, v0, force, checkpoint_every: int = 8, t0: int = 0):
    """Run force.shape[0] steps (force: (T, 2, H, W), channel 0 on u faces, 1 on v faces);
    differentiable w.r.t. force and the initial state. One state in every
    ``checkpoint_every`` steps is kept; the steps in between are recomputed in backward."""
    T = force.shape[0]
    k = max(1, int(checkpoint_every))

    def segment(d, u, v, f, start):
        for s in range(f.shape[0]):
            d, u, v = SmokeStep.apply(d, u, v, f[s, 0], f[s, 1], model, start + s)
        return d, u, v

    state = (d0, u0, v0)
    for s0 in range(0, T, k):
        fs = force[s0:s0 + k]
        if torch.is_grad_enabled() and (fs.requires_grad or any(x.requires_grad for x in state)):
            state = checkpoint(segment, *state, fs, t0 + s0, use_reentrant=False)
        else:
            state = segment(*state, fs, t0 + s0)
    return state


def density_loss(d_final, target):
    """Sum of squared differences between the final density and the target."""
    return ((d_final - target) ** 2).sum()


def loss_and_grad(model, force, target, checkpoint_every=8):
    """(loss, d loss / d force) of a rollout from rest."""
    f = force.detach().requires_grad_(True)
    d0, u0, v0 = model.zeros_state()
    d, _, _ = rollout(model, d0, u0, v0, f, checkpoint_every)
    loss = density_loss(d, target)
    (g,) = torch.autograd.grad(loss, f)
    return float(loss.detach()), g


def loss_only(model, force, target):
    with torch.no_grad():
        d0, u0, v0 = model.zeros_state()
        d, _, _ = rollout(model, d0, u0, v0, force)
        return float(density_loss(d, target))


def optimize(model, force, target, iters=100, step=None, checkpoint_every=8, log=None):
    """Gradient descent on the control: f <- f - step * g / max|g| (a fixed step in the max
    norm); returns the final control and the loss history."""
    f = force.detach().clone()
    history = []
    for it in range(iters):
        loss, g = loss_and_grad(model, f, target, checkpoint_every)
        history.append(loss)
        if log:
            log(it, loss)
        gmax = float(g.abs().max())
        if gmax == 0.0:
            break
        f -= (step if step is not None else 0.05) * g / gmax
    history.append(loss_only(model, f, target))
    return f, history


def inverse_problem(n=256, steps=64, dtype=torch.float32, device=None, **kw):
    """The 256^2 inverse scene: rest start, one seeded source, control ~ N(0, 0.01^2), target
    a Gaussian blob (sigma 20 cells) in the upper half. Returns (model, force, target)."""
    from .scenes import inverse_256, target_blob

    sc = inverse_256(steps)
    scale = n / sc.W
    plumes = np.asarray(sc.plumes, dtype=np.float64)
    plumes[:, :3] *= scale
    model = ControlledSmoke(n, n, 1.0 / n, 0.5 / n, gravity=sc.gravity, plumes=plumes, seed=sc.seed, dtype=dtype,
                            device=device, **kw)
    gen = torch.Generator(device="cpu").manual_seed(sc.seed)
    force = (0.01 * torch.randn((steps, 2, n, n), generator=gen, dtype=torch.float64)).to(dtype).to(model.device)
    target = torch.from_numpy(target_blob(n, 20.0 * scale, sc.seed)).to(dtype).to(model.device)
    return model, force, target
