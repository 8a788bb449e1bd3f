"""Generate golden fixtures by running the reference's own Numba kernels.

Run in a container that holds the reference source (it is not needed anywhere
else):  python tests/golden/make_golden.py path/to/reference/src [generator ...]
(or with REFERENCE_SRC set to that path; generator names select a subset, default all)

The reference (LCEBurton/python-game-engine, src/cfd) is imported read-only; numba's
on-disk cache is redirected to tests/golden/_numba_cache (git-ignored) because the
reference tree may be read-only. Outputs: tests/golden/*.npz, small seeded cases
(16x16 .. 48x40) in float32 and float64, consumed by tests/test_oracle_golden.py
(oracle pin) and tests/test_cuda_parity.py (CUDA parity).
"""
from __future__ import annotations

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SRC = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE_SRC")
if not REF_SRC:
    sys.exit("usage: python tests/golden/make_golden.py path/to/reference/src (or set REFERENCE_SRC)")
os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(HERE, "_numba_cache"))
sys.path.insert(0, REF_SRC)

import numpy as np  # noqa: E402

import cfd.solvers  # noqa: E402,F401  (import order: registries first, see multigrid/solver.py:5)
import cfd.operators  # noqa: E402,F401
from cfd.backends.numba.operators import advection as ref_adv  # noqa: E402
from cfd.backends.numba.operators import forces as ref_forces  # noqa: E402
from cfd.backends.numba.operators.boundaries import enforce_boundary_conditions  # noqa: E402
from cfd.backends.numba.operators.divergence import compute_divergence  # noqa: E402
from cfd.backends.numba.operators.pressure_gradient import apply_pressure_gradient  # noqa: E402
from cfd.backends.numba.operators.residual import compute_residual  # noqa: E402
from cfd.backends.numba.solvers.jacobi import jacobi_pressure_solver  # noqa: E402
from cfd.backends.numba.solvers.red_black_sor_gauss_seidel import (  # noqa: E402
    red_black_sor_gauss_seidel_pressure_solver,
)
from cfd.backends.numba.solvers.gauss_seidel import gauss_seidel_pressure_solver  # noqa: E402
from cfd.backends.numba.solvers.multigrid.solver import MultigridSolver  # noqa: E402
from cfd.backends.numba.solvers.multigrid.transfer import restrict, prolong  # noqa: E402
from cfd.backends.numba.solvers.multigrid.masks import coarsen_solid_mask  # noqa: E402
from cfd.common.emitters import Emitter2D  # noqa: E402
from cfd.common.config import SimulationConfig, GridConfig, PressureSolverConfig  # noqa: E402
from cfd.common.simulation import SmokeSimulation2D  # noqa: E402
from cfd.solvers.params import JacobiParams, SORParams, MultigridParams, GaussSeidelParams  # noqa: E402
from cfd.profiling.session import ProfileSession  # noqa: E402


def masks(H, W, rng=None, obstacles=0):
    solid = np.zeros((H, W), bool)
    solid[0, :] = solid[-1, :] = True
    solid[:, 0] = solid[:, -1] = True
    if rng is not None and obstacles:
        for _ in range(obstacles):
            j, i = rng.integers(2, H - 3), rng.integers(2, W - 3)
            solid[j:j + 2, i:i + 3] = True
    fmu = np.zeros((H, W + 1), bool)
    fmv = np.zeros((H + 1, W), bool)
    fmu[:, 1:-1] = ~(solid[:, :-1] | solid[:, 1:])
    fmv[1:-1, :] = ~(solid[:-1, :] | solid[1:, :])
    fl = fmu[:, :-1] | fmu[:, 1:] | fmv[:-1] | fmv[1:]
    return solid, fmu, fmv, fl


def save(name, **arrays):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
    print("wrote", name, sum(a.nbytes for a in arrays.values() if hasattr(a, "nbytes")))


def gen_operators():
    out = {}
    for dt_name, dtype in (("f32", np.float32), ("f64", np.float64)):
        for (H, W, obst, seed) in ((16, 16, 0, 1), (20, 28, 3, 2), (17, 13, 1, 3)):
            rng = np.random.default_rng(seed)
            tag = f"{dt_name}_{H}x{W}"
            solid, fmu, fmv, fl = masks(H, W, rng, obst)
            h = 1.0 / max(H, W)
            dt = 1.7 * h  # backtraces up to ~2.5 cells: exercises clamping at the walls
            rnd = lambda *s: rng.uniform(-1.0, 1.0, s).astype(dtype)
            dens = rng.uniform(0.0, 1.0, (H, W)).astype(dtype)
            temp = rnd(H, W)
            u = rnd(H, W + 1)
            v = rnd(H + 1, W)
            p = rnd(H, W)
            div = rnd(H, W)
            d = dict(solid=solid, fmu=fmu, fmv=fmv, fl=fl, dens=dens, temp=temp, u=u, v=v, p=p,
                     div=div, h=np.float64(h), dt=np.float64(dt))
            # advection (MAC shapes)
            o = np.zeros_like(dens)
            ref_adv.advect_scalar_field(dens, o, u, v, fl, dt, h)
            d["adv_scalar"] = o
            o = np.zeros_like(u)
            ref_adv.advect_velocity_u(u, o, v, fmu, dt, h)
            d["adv_u"] = o
            o = np.zeros_like(v)
            ref_adv.advect_velocity_v(v, o, u, fmv, dt, h)
            d["adv_v"] = o
            # forces / cooling
            vv = v.copy()
            ref_forces.apply_forces(vv, dens, temp, dt, -0.5, 5.0, 1.0, 0.1)
            d["forces_v"] = vv
            tt = temp.copy()
            ref_forces.cool_temperature(tt, 0.1, 0.5, dt)
            d["cool_t"] = tt
            # divergence / residual / gradient / boundaries
            o = np.zeros_like(dens)
            compute_divergence(u, v, o, fmu, fmv, h)
            d["divergence"] = o
            alpha = (-(h * h) * 1.0) / dt
            o = np.zeros_like(dens)
            compute_residual(p, div, fl, fmu, fmv, alpha, 0.25, o)
            d["residual"] = o
            uu, vv = u.copy(), v.copy()
            apply_pressure_gradient(uu, vv, p, fmu, fmv, 1.3, h, dt)
            d["grad_u"], d["grad_v"] = uu, vv
            uu, vv = u.copy(), v.copy()
            enforce_boundary_conditions(uu, vv, solid.astype(np.uint8))
            d["bc_u"], d["bc_v"] = uu, vv
            # solvers
            pp = np.zeros_like(p)
            jacobi_pressure_solver(pp, div, fmu, fmv, 1.0, h, dt, iterations=23)
            d["jacobi"] = pp
            pp = p.copy()
            red_black_sor_gauss_seidel_pressure_solver(pp, div, fmu, fmv, 1.0, h, dt, iterations=9, omega=1.7)
            d["rbsor"] = pp
            pp = p.copy()
            red_black_sor_gauss_seidel_pressure_solver(pp, div, fmu, fmv, 1.0, h, dt, iterations=5, omega=0.0)
            d["rbsor_auto"] = pp
            pp = p.copy()
            gauss_seidel_pressure_solver(pp, div, fmu, fmv, 1.0, h, dt, iterations=4)
            d["gauss_seidel"] = pp
            # transfer operators on even shapes
            if H % 2 == 0 and W % 2 == 0:
                c = np.zeros((H // 2, W // 2), dtype)
                restrict(p, fl, c)
                d["restrict"] = c
                f = np.zeros_like(p)
                prolong(c, fl, f)
                d["prolong"] = f
                sc = np.zeros((H // 2, W // 2), np.bool_)
                coarsen_solid_mask(~fl, sc)
                d["coarsen"] = sc
            out[tag] = d
    for tag, d in out.items():
        save("ops_" + tag, **d)


def gen_kat_shapes():
    """The reference advection KATs pass (H, W)-shaped u and v (test_advection.py:16-138)."""
    H = W = 16
    _, fmu, fmv, fl = masks(H, W)
    rng = np.random.default_rng(11)
    d = {}
    for dt_name, dtype in (("f32", np.float32), ("f64", np.float64)):
        s = rng.uniform(0, 5, (H, W)).astype(dtype)
        u = rng.uniform(-1.5, 1.5, (H, W)).astype(dtype)
        v = rng.uniform(-1.5, 1.5, (H, W)).astype(dtype)
        o = np.zeros_like(s)
        ref_adv.advect_scalar_field(s, o, u, v, fl, 1.0, 1.0)
        d[f"{dt_name}_src"], d[f"{dt_name}_u"], d[f"{dt_name}_v"], d[f"{dt_name}_out"] = s, u, v, o
    d["fl"] = fl
    save("kat_square_uv", **d)


def gen_multigrid():
    d = {}
    for dt_name, dtype in (("f32", np.float32), ("f64", np.float64)):
        H = W = 32
        rng = np.random.default_rng(5)
        _, fmu, fmv, fl = masks(H, W)
        h = 1.0 / H
        dt = 0.5 * h
        div = (rng.uniform(-1, 1, (H, W)) * fl).astype(dtype)
        d["div_" + dt_name] = div
        for name, kw in (
            ("jac", dict(smoother_type="jacobi", v_cycles=1, num_levels=4, smoother_iterations=2,
                         coarsest_iterations=30)),
            ("sor", dict(smoother_type="rb_sor_gauss_seidel", v_cycles=2, num_levels=3, smoother_iterations=2,
                         coarsest_iterations=20)),
            ("jac5", dict(smoother_type="jacobi", v_cycles=2, num_levels=5, smoother_iterations=3,
                          coarsest_iterations=40)),
        ):
            mg = MultigridSolver()
            p = np.zeros((H, W), dtype)
            mg(p, div, fmu, fmv, 1.0, h, dt, smoother_backend="numba", profiler=ProfileSession.disabled(),
               **kw)
            d[f"mg_{name}_{dt_name}"] = p
    save("multigrid", **d)


def gen_emitters():
    d = {}
    H, W = 24, 20
    for k, approach in enumerate(("linear", "gaussian", "quadratic", "hard_cutoff")):
        for numba_opt in (True, False):
            f = np.zeros((H, W), np.float32)
            e = Emitter2D(position=(8.5, 10.25), radius=5.5, density_value=1.7, approach=approach,
                          numba_optimized=numba_opt)
            e._apply_scalar_field(f, 1.7, 0.016)
            e._apply_scalar_field(f, 1.7, 0.016)
            d[f"{approach}_{'numba' if numba_opt else 'python'}"] = f
    save("emitters", **d)


def gen_sim():
    """Full SmokeSimulation2D substeps (float32, the reference's only dtype)."""
    d = {}
    H = W = 32
    for name, method, params in (
        ("jacobi", "jacobi", JacobiParams(iterations=30)),
        ("rbsor", "rb_sor_gauss_seidel", SORParams(iterations=20, omega=1.8)),
        ("mg", "multigrid", MultigridParams(smoother_type="jacobi", num_levels=3, v_cycles=2,
                                            smoother_iterations=2, coarsest_iterations=20)),
        ("gs", "gauss_seidel", GaussSeidelParams(iterations=10)),
    ):
        cfg = SimulationConfig(grid=GridConfig(size=(W, H), cell_size=1.0 / H),
                               pressure_solver=PressureSolverConfig(method=method, params=params))
        sim = SmokeSimulation2D(cfg, profiler=ProfileSession.disabled((H, W)))
        sim.add_emitter(Emitter2D(position=(16, 6), radius=4.0, density_value=3.0, temperature_value=2.0,
                                  velocity_value=(0.3, 2.0), approach="linear", numba_optimized=True))
        for step in range(8):
            sim.substep(sim.dt)
            if step in (0, 7):
                d[f"{name}_s{step}_density"] = sim.density.copy()
                d[f"{name}_s{step}_u"] = sim.velocity_u.copy()
                d[f"{name}_s{step}_v"] = sim.velocity_v.copy()
                d[f"{name}_s{step}_p"] = sim.pressure.copy()
                d[f"{name}_s{step}_t"] = sim.temperature.copy()
                d[f"{name}_s{step}_div"] = sim.divergence.copy()
                d[f"{name}_s{step}_res"] = sim.pressure_residual.copy()
    save("sim", **d)


def obstacle_solid(H, W):
    """The 1-cell wall ring plus a rectangle and a disc inside (set_solid_mask replaces the
    whole solid mask, so the ring is part of it, as a caller of the reference would pass)."""
    j, i = np.indices((H, W))
    solid = np.zeros((H, W), bool)
    solid[0, :] = solid[-1, :] = True
    solid[:, 0] = solid[:, -1] = True
    solid[14:18, 6:13] = True
    solid |= (i + 0.5 - 22.0) ** 2 + (j + 0.5 - 20.0) ** 2 < 3.2 ** 2
    return solid


def gen_sim_obstacles():
    """SmokeSimulation2D substeps after set_solid_mask with interior obstacles (the masks are
    rebuilt at the next substep, simulation.py:133-143, :198-204; the reference multigrid
    rebuilds its hierarchy with rebuild_masks=True)."""
    d = {}
    H = W = 32
    solid = obstacle_solid(H, W)
    d["solid"] = solid
    for name, method, params in (
        ("jacobi", "jacobi", JacobiParams(iterations=30)),
        ("mg", "multigrid", MultigridParams(smoother_type="jacobi", num_levels=3, v_cycles=2,
                                            smoother_iterations=2, coarsest_iterations=20, rebuild_masks=True)),
    ):
        cfg = SimulationConfig(grid=GridConfig(size=(W, H), cell_size=1.0 / H),
                               pressure_solver=PressureSolverConfig(method=method, params=params))
        sim = SmokeSimulation2D(cfg, profiler=ProfileSession.disabled((H, W)))
        sim.add_emitter(Emitter2D(position=(16, 6), radius=4.0, density_value=3.0, temperature_value=2.0,
                                  velocity_value=(0.3, 2.0), approach="linear", numba_optimized=True))
        for step in range(8):
            if step == 2:
                sim.set_solid_mask(solid.astype(np.uint8))
            sim.substep(sim.dt)
            if step in (1, 2, 7):
                d[f"{name}_s{step}_density"] = sim.density.copy()
                d[f"{name}_s{step}_u"] = sim.velocity_u.copy()
                d[f"{name}_s{step}_v"] = sim.velocity_v.copy()
                d[f"{name}_s{step}_p"] = sim.pressure.copy()
                d[f"{name}_s{step}_t"] = sim.temperature.copy()
                d[f"{name}_s{step}_div"] = sim.divergence.copy()
                d[f"{name}_s{step}_res"] = sim.pressure_residual.copy()
    save("sim_obstacles", **d)


GENERATORS = {"operators": gen_operators, "kat_shapes": gen_kat_shapes, "multigrid": gen_multigrid,
              "emitters": gen_emitters, "sim": gen_sim, "sim_obstacles": gen_sim_obstacles}

if __name__ == "__main__":
    # optional generator names after the reference path select a subset (default: all)
    for name in (sys.argv[2:] or list(GENERATORS)):
        GENERATORS[name]()
