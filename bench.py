"""Benchmark: cell-steps/s of the smoke step at 2048^2 with the mixed-precision solve.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload ``mixed_2048``: one SmokeSimulation2D substep of the 2048^2 four-source
scene (float32 state), pressure solved by the convergent multigrid (V(2,2),
red-black Gauss-Seidel omega 1.3, full weighting, bilinear prolongation, the 128^2
coarsest level solved exactly by the cosine transform) with FP32 cycles inside FP64
iterative refinement to a relative residual of 1e-8 (and, in a short second run, 1e-10), then projection and the reference's metrics tail. The same scene is also
timed with a float64 state and an all-FP64 solve to the same residual ("fp64_gpu").

A step runs on data resident in HBM (``value``); ``e2e`` repeats it through the
public API with a pinned-host -> device copy of the step's source table and a
device -> pinned-host read of the density field and solve residual every step. The
working set (~190 MB) exceeds the 126 MB L2, so no explicit flush runs between
steps. Multi-GPU (torchrun): the scene does not shard, so each rank advances its own
replica (weak scaling) and ``value`` counts every rank's cells over the slowest
rank's time.

--impl reference times the CPU oracle (a C/OpenMP restatement of the reference's
kernels plus the same multigrid) on the host cores: each step is one substep of the
same scene; rank 0 alone runs it.
"""
from __future__ import annotations

import argparse
import dataclasses
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-steps/s at 2048² mixed vs FP64 GPU at equal resid 1e-8; % HBM roofline"
UNIT = "cell-steps/s"
TOL = 1e-8
TOL_TIGHT = 1e-10  # the workload's second residual target
COARSEST = 128  # exact coarsest level (open box: cosine transform); the hierarchy is 2048^2 .. 128^2
# (measured per 2048^2 mixed step: coarsest 32 0.880 ms, 64 1.004, 128 0.856, 256 0.910)
OMEGA = 1.3  # red-black Gauss-Seidel over-relaxation of the multigrid (GPU arms and the oracle)
BATCH_METRIC = "cell-steps/s, 256 batched scenes {64..256}^2, mixed-precision multigrid to 1e-6 per scene"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 8:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[4 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def mixed_config(mean_cycles, converged, parallelism):
    """The `config` object of the mixed_2048 line, the same keys in both arms."""
    return {"workload": "mixed_2048", "grid": [2048, 2048], "sources": 4,
            "solver": f"multigrid V(2,2) RBGS w={OMEGA}, full weighting, bilinear, {COARSEST}x{COARSEST} exact "
                      f"coarsest (cosine transform); FP32 cycles in FP64 iterative refinement",
            "tol": TOL, "mean_cycles_per_step": mean_cycles, "converged": bool(converged),
            "l2": "working set > 126 MB L2; no flush", "parallelism": parallelism}


# ----------------------------------------------------------------------------- reference arm
def cpu_oracle_steps(n_steps, warmup, fields=None):
    """Time the CPU oracle on the same scene: returns (seconds per step list, cycles, threads).
    `fields` (a dict), when given, receives the oracle's density, u, v and pressure after
    all warmup + n_steps substeps."""
    import numpy as np

    import oracle as O

    sg = importlib.import_module("python-game-engine_b200")
    sc = sg.scenes.mixed_2048(steps=n_steps + warmup)
    fmu, fmv = O.face_masks_from_solid(np.zeros((sc.H, sc.W), bool))
    fl = O.is_fluid_from_faces(fmu, fmv)
    gmg = O.GMGOracle(fmu, fmv, fl, coarsest=COARSEST, omega=OMEGA)  # the GPU arm's hierarchy
    cycles = []

    def solver(p, div, fmu_, fmv_, rho, h, dt, **_):
        alpha = O.alpha_coeff(h, rho, dt)
        b = alpha * div.astype(np.float64) * fl
        p64 = np.zeros(p.shape)
        c, _hist = gmg.solve(p64, b, tol=TOL, max_cycles=40, precision="mixed")
        cycles.append(c)
        p[:] = p64.astype(p.dtype)

    sim = O.OracleSim(sc.H, sc.W, sc.cell_size, solver, {}, dtype=np.float32)
    sim.dt, sim.gravity = sc.dt, sc.gravity
    sim.plumes = [O.PlumeSpec(*row, seed=sc.seed) for row in sc.plumes]
    times = []
    for k in range(n_steps + warmup):
        t0 = time.perf_counter()
        sim.substep(sc.dt)
        if k >= warmup:
            times.append(time.perf_counter() - t0)
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    if fields is not None:
        fields.update(steps=n_steps + warmup, density=sim.density.copy(), velocity_u=sim.velocity_u.copy(),
                      velocity_v=sim.velocity_v.copy(), pressure=sim.pressure.copy())
    return times, cycles[warmup:], threads


def batch_sample(scenes, per_size=1):
    """A sample of the batch stratified by grid size: the first `per_size` scenes of each size."""
    picked, seen = [], {}
    for sc in scenes:
        if seen.get(sc.W, 0) < per_size:
            picked.append(sc)
            seen[sc.W] = seen.get(sc.W, 0) + 1
    return picked


def cpu_oracle_batch(scenes, sample, steps, warmup=1):
    """The CPU oracle on a size-stratified `sample` of the batch `scenes`: each sampled scene
    is stepped `warmup` untimed then `steps` timed substeps with the oracle's multigrid in mixed
    precision to 1e-6. The time per cell-step measured for each grid size is weighted by that
    size's share of the whole batch's cells, so the figure estimates the whole batch's rate."""
    import numpy as np

    import oracle as O

    per_size = {}
    for sc in sample:
        fmu, fmv = O.face_masks_from_solid(np.zeros((sc.H, sc.W), bool))
        fl = O.is_fluid_from_faces(fmu, fmv)
        gmg = O.GMGOracle(fmu, fmv, fl, coarsest=8, omega=OMEGA)

        def solver(p, div, fmu_, fmv_, rho, h, dt, gmg=gmg, fl=fl, **_):
            b = O.alpha_coeff(h, rho, dt) * div.astype(np.float64) * fl
            p64 = np.zeros(p.shape)
            gmg.solve(p64, b, tol=1e-6, max_cycles=50, precision="mixed")
            p[:] = p64.astype(p.dtype)

        sim = O.OracleSim(sc.H, sc.W, sc.cell_size, solver, {}, dtype=np.float32)
        sim.dt, sim.gravity = sc.dt, sc.gravity
        sim.plumes = [O.PlumeSpec(*row, seed=sc.seed) for row in sc.plumes]
        for _ in range(warmup):
            sim.substep(sc.dt)
        t0 = time.perf_counter()
        for _ in range(steps):
            sim.substep(sc.dt)
        dt_s = time.perf_counter() - t0
        acc = per_size.setdefault(sc.W, [0.0, 0])
        acc[0] += dt_s
        acc[1] += sc.H * sc.W * steps
    batch_cells = {}
    for sc in scenes:
        batch_cells[sc.W] = batch_cells.get(sc.W, 0) + sc.H * sc.W
    est_s = sum(batch_cells[w] * per_size[w][0] / per_size[w][1] for w in batch_cells)
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    sizes = sorted(per_size)
    return {"value": sum(batch_cells.values()) / est_s, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{len(sample)} scenes of the batch (the first of each size {sizes}) x {steps} substeps each "
                      f"on the CPU oracle (C/OpenMP restatement of the reference kernels + the same multigrid to "
                      f"1e-6), after {warmup} warm-up substep(s); time per cell-step per size weighted by that "
                      f"size's share of the batch's {sum(batch_cells.values())} cells"}


def reference_numba(n=2048, steps=2, warmup=2, cycles=5):
    """The reference's own Numba code on the host cores, as context beside the oracle port
    (the reference cannot reach the 1e-8 target: its multigrid stalls near 0.1). Imports
    the reference installed under baseline/_ref (or REFERENCE_SRC). Measures
    (a) SmokeSimulation2D substeps (float32, the reference's only dtype) at n^2 with its
        multigrid (Jacobi smoother, log2(n / 8) + 1 levels, 2 V(2,2) cycles), the 4 sources
        of the scene as the reference's additive emitters, after `warmup` substeps (JIT);
    (b) float64 calls of its kernels on the scene's first divergence: one multigrid V(2,2)
        cycle (Jacobi smoother) repeated `cycles` times with the relative residual after each,
        and one Jacobi sweep."""
    ref = os.environ.get("REFERENCE_SRC") or os.path.join(ROOT, "baseline", "_ref")
    if not os.path.isdir(os.path.join(ref, "cfd")):
        return {"unavailable": "the reference package is not installed under baseline/_ref"}
    try:
        import numba
    except ImportError:
        return {"unavailable": "numba is not installed"}
    import numpy as np

    os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(tempfile.gettempdir(), "sg_reference_numba_cache"))
    if ref not in sys.path:
        sys.path.insert(0, ref)
    import cfd.solvers  # noqa: F401  (registries first: the reference's import order)
    import cfd.operators  # noqa: F401
    from cfd.backends.numba.operators.divergence import compute_divergence
    from cfd.backends.numba.operators.residual import compute_residual
    from cfd.backends.numba.solvers.jacobi import jacobi_pressure_solver
    from cfd.backends.numba.solvers.multigrid.solver import MultigridSolver
    from cfd.common.config import GridConfig, PressureSolverConfig, SimulationConfig
    from cfd.common.emitters import Emitter2D
    from cfd.common.simulation import SmokeSimulation2D
    from cfd.profiling import ProfileSession
    from cfd.solvers.params import MultigridParams

    sg = importlib.import_module("python-game-engine_b200")
    sc = sg.scenes.mixed_2048(steps=steps + warmup)
    levels = int(np.log2(n // 8)) + 1
    mgp = MultigridParams(smoother_type="jacobi", num_levels=levels, v_cycles=2, smoother_iterations=2,
                          coarsest_iterations=30)
    cfg = SimulationConfig(grid=GridConfig(size=(n, n), cell_size=1.0 / n),
                           pressure_solver=PressureSolverConfig(method="multigrid", params=mgp))
    import contextlib

    with contextlib.redirect_stdout(sys.stderr):  # the reference prints a banner; stdout carries the JSON line
        sim = SmokeSimulation2D(cfg, profiler=ProfileSession.disabled((n, n)))
    sim.dt, sim.gravity = 0.5 / n, sc.gravity
    k = n / sc.W
    for cx, cy, r, dens, vin, _ in sc.plumes:
        sim.add_emitter(Emitter2D(position=(cx * k, cy * k), radius=r * k, density_value=dens / sim.dt,
                                  velocity_value=(0.0, vin / sim.dt), approach="hard_cutoff", numba_optimized=True))
    t_jit = time.perf_counter()
    for _ in range(warmup):
        sim.substep(sim.dt)
    t_jit = time.perf_counter() - t_jit
    t0 = time.perf_counter()
    for _ in range(steps):
        sim.substep(sim.dt)
    t_step = (time.perf_counter() - t0) / steps
    # float64 kernels on the current divergence (recomputed from the state)
    u = sim.velocity_u.astype(np.float64)
    v = sim.velocity_v.astype(np.float64)
    fmu, fmv = sim._face_mask_u, sim._face_mask_v
    fl = sim.is_fluid
    div = np.zeros((n, n))
    compute_divergence(u, v, div, fmu, fmv, sim.cell_size)
    alpha = -(sim.cell_size ** 2) * sim.fluid_density / sim.dt
    res = np.zeros((n, n))

    def relres(p):
        compute_residual(p, div, fl, fmu, fmv, alpha, 0.25, res)
        return float(np.linalg.norm(res))

    r0 = relres(np.zeros((n, n)))
    mg = MultigridSolver()
    p = np.zeros((n, n))
    mg(p, div, fmu, fmv, sim.fluid_density, sim.cell_size, sim.dt, v_cycles=1, smoother_type="jacobi",
       smoother_backend="numba", num_levels=levels, smoother_iterations=2, coarsest_iterations=30,
       profiler=ProfileSession.disabled((n, n)))  # JIT and hierarchy
    p[:] = 0.0
    hist, t_cyc = [], 0.0
    for _ in range(cycles):
        t0 = time.perf_counter()
        mg(p, div, fmu, fmv, sim.fluid_density, sim.cell_size, sim.dt, v_cycles=1, smoother_type="jacobi",
           smoother_backend="numba", num_levels=levels, smoother_iterations=2, coarsest_iterations=30,
           profiler=ProfileSession.disabled((n, n)))
        t_cyc += time.perf_counter() - t0
        hist.append(relres(p) / r0 if r0 > 0 else 0.0)
    q = np.zeros((n, n))
    jacobi_pressure_solver(q, div, fmu, fmv, sim.fluid_density, sim.cell_size, sim.dt, iterations=1)
    t0 = time.perf_counter()
    jacobi_pressure_solver(q, div, fmu, fmv, sim.fluid_density, sim.cell_size, sim.dt, iterations=10)
    t_jac = (time.perf_counter() - t0) / 10
    return {"threads": int(numba.get_num_threads()), "numba": numba.__version__,
            "substep_fp32": {"ms_per_step": 1e3 * t_step, "cell_steps_per_s": n * n / t_step, "steps": steps,
                             "solver": f"reference multigrid, {levels} levels, Jacobi smoother, 2 x V(2,2) "
                                       "(fixed cycles: it has no tolerance loop)",
                             "warmup_s_with_jit": t_jit},
            "vcycle_fp64": {"ms_per_cycle": 1e3 * t_cyc / cycles, "relres_after_each_cycle": hist},
            "jacobi_sweep_fp64_ms": 1e3 * t_jac,
            "sources": "the scene's 4 sources as additive hard-cutoff emitters (the reference has no overwriting "
                       "source)"}


def run_reference(args):
    world, rank, _ = _dist()
    if rank != 0:
        return 0
    if args.workload == "batch_256":
        return run_reference_batch(args)
    steps = max(1, args.steps)
    times, cycles, threads = cpu_oracle_steps(steps, args.warmup)
    cells = 2048 * 2048
    value = cells * len(times) / sum(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": len(times),
        "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 state, f64/f32 mixed solve", "data": "synthetic",
        "config": mixed_config(sum(cycles) / max(len(cycles), 1), len(cycles) == len(times),
                               f"replicas x{args.gpus} (host cores of rank 0)"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{len(times)} substeps of mixed_2048 on the CPU oracle (C/OpenMP restatement of "
                                   f"the reference kernels + the same multigrid), after {args.warmup} warm-up"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_reference_numba:
        try:
            line["reference_numba"] = reference_numba()
        except Exception as e:  # context only: the timed arm above stands on its own
            line["reference_numba"] = {"unavailable": f"{type(e).__name__}: {e}"}
    print(json.dumps(line), flush=True)
    return 0


def run_reference_batch(args):
    """The batch workload's reference arm: the CPU oracle steps a size-stratified sample of the
    batch (one scene of each grid size, `warmup` untimed and `steps` timed substeps each) on the
    host cores, and the per-size rates are weighted by the batch's size mix."""
    sg = importlib.import_module("python-game-engine_b200")
    scenes = sg.scenes.batch_256(256, steps=args.steps)
    steps = max(1, args.steps)
    cpu = cpu_oracle_batch(scenes, batch_sample(scenes), steps, warmup=max(0, args.warmup))
    total_cells = sum(sc.H * sc.W for sc in scenes)
    value = cpu["value"]
    line = {
        "impl": "reference", "metric": BATCH_METRIC, "workload": "batch_256", "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * total_cells / value,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32 state, f64/f32 mixed solve",
        "data": "synthetic",
        "config": {"workload": "batch_256", "scenes": len(scenes), "cells": total_cells, "tol": 1e-6,
                   "sample": cpu["sample"]},
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _measured_traffic(kernel):
    """DRAM bytes (read + write) of one launch of `kernel` from the committed ncu summary, or
    None when no summary lists it."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles", "traffic_mixed_2048.json")
    try:
        with open(path) as f:
            return json.load(f).get(kernel, {}).get("dram_bytes")
    except (OSError, ValueError):
        return None


def compare_fp64(sg, sc, make, steps):
    """Run the mixed-precision and the all-FP64 GPU paths side by side from the same initial
    state for `steps` substeps; errors of the mixed path's fields relative to the FP64 ones."""
    import torch

    mixed = make(torch.float32, "mixed")
    full = make(torch.float64, "fp64")
    for _ in range(steps):
        mixed.substep(sc.dt)
        full.substep(sc.dt)
    torch.cuda.synchronize()

    def rel(a, b):
        a, b = a.double(), b.double()
        return float((a - b).norm() / max(float(b.norm()), 1e-300))

    out = {"steps": steps,
           "pressure_rel_l2": rel(mixed.pressure - mixed.pressure.mean(), full.pressure - full.pressure.mean()),
           "density_rel_l2": rel(mixed.density, full.density),
           "velocity_u_rel_l2": rel(mixed.velocity_u, full.velocity_u),
           "divergence_l2_mixed": float(mixed.divergence.double().norm()),
           "divergence_l2_fp64": float(full.divergence.double().norm())}
    del mixed, full
    torch.cuda.empty_cache()
    return out


def compare_oracle(sg, sc, make, ofields):
    """The mixed GPU path run for the CPU oracle's substeps from the same initial state:
    relative L2 errors of its fields against the oracle's (the reference's kernels restated
    in C, the same multigrid to 1e-8 in mixed precision on the CPU; pressures compared with
    their means removed, the pressure being defined up to a constant)."""
    import numpy as np
    import torch

    sim = make(torch.float32, "mixed")
    for _ in range(ofields["steps"]):
        sim.substep(sc.dt)
    torch.cuda.synchronize()

    def rel(a, b):
        a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    p_gpu = sim.pressure.double().cpu().numpy()
    p_cpu = np.asarray(ofields["pressure"], np.float64)
    out = {"steps": ofields["steps"],
           "density_rel_l2": rel(sim.density.cpu().numpy(), ofields["density"]),
           "velocity_u_rel_l2": rel(sim.velocity_u.cpu().numpy(), ofields["velocity_u"]),
           "velocity_v_rel_l2": rel(sim.velocity_v.cpu().numpy(), ofields["velocity_v"]),
           "pressure_rel_l2": rel(p_gpu - p_gpu.mean(), p_cpu - p_cpu.mean()),
           "oracle": f"CPU restatement of the reference kernels + the same multigrid ({COARSEST}x{COARSEST} exact "
                     f"coarsest, solved by the cosine transform in float64) to 1e-8"}
    del sim
    torch.cuda.empty_cache()
    return out


# ----------------------------------------------------------------------------- our arm
def run_ours(args):
    import torch
    import torch.distributed as dist

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    sg = importlib.import_module("python-game-engine_b200")
    lib = sg._lib.load()
    dev = torch.device("cuda", local)
    sc = sg.scenes.mixed_2048(steps=args.steps)
    cells = sc.cells

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def make(dtype, precision, tol=TOL, remove_mean=False, inner=1):
        params = sg.GeometricMultigridParams(tol=tol, max_cycles=40, precision=precision, omega=OMEGA,
                                             coarsest=args.coarsest, fixed_cycles=args.fixed_cycles,
                                             remove_mean=remove_mean, inner_cycles=inner)
        sim = sg.scenes.make_sim(sc, "geometric_multigrid", params, dtype=dtype, device=dev)
        # float32 states advect in the arithmetic chosen for the run; float64 states in the
        # reference's float64 arithmetic
        sim.advection_arithmetic = args.advection if dtype == torch.float32 else "reference"
        # forces and the projection tail follow the same choice
        sim.operator_arithmetic = sim.advection_arithmetic
        return sim

    solver = sg.get_solver("geometric_multigrid", "cuda")

    def timed(sim, steps, warmup, e2e=False, sample_clocks=False):
        stream = torch.cuda.current_stream()
        host_table = None
        if e2e:
            # the step's input: the source table, rewritten on the host and sent with the
            # source kernel's launch parameters every step; its result: the density field
            # and the solve's relative residual, copied to pinned host memory every step on a
            # copy stream that overlaps the next step (the density goes through a device
            # staging slot, since the next step's sources write the field in place; two
            # slots, a step waits for the copy of the slot it is about to refill)
            host_table = torch.tensor([p.row() for p in sim.plumes], dtype=torch.float64).pin_memory()
            rows = host_table.numpy().copy()
            sim.set_plume_table(host_table.numpy())
            readback = sg.FieldReadback(sim, "density", slots=2)
            host_res = torch.zeros(2, dtype=torch.float64).pin_memory()
        for _ in range(warmup):
            sim.substep(sc.dt)
        barrier()
        sampler = ClockSampler(local) if sample_clocks else None
        if sampler:
            sampler.start()
            time.sleep(0.3)
        plan = solver.current_plan()
        solves0, cycles0, fails0 = plan.counters()
        l0 = lib.sg_launch_count()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        start.record(stream)
        for k in range(steps):
            if e2e:
                host_table.numpy()[:] = rows
            sim.substep(sc.dt)
            if e2e:
                slot = readback.submit()
                # the solve's relative residual rides on the same copy stream
                plan.relres_async(host_res[slot:slot + 1], readback.copy_stream)
        if e2e:
            readback.wait(stream)
        end.record(stream)
        barrier()
        ms = start.elapsed_time(end)
        launches = lib.sg_launch_count() - l0
        clocks = sampler.stop() if sampler else None
        solves1, cycles1, fails1 = plan.counters()
        prologue_nodes, body_nodes = plan.graph_nodes()
        # eager launches counted by the library + kernel nodes run by the solve graphs
        launches += prologue_nodes * (solves1 - solves0) + body_nodes * (cycles1 - cycles0)
        info = {"cycles": cycles1 - cycles0, "solves": solves1 - solves0, "failures": fails1 - fails0}
        if e2e:
            sim.set_plume_table(None)
            sim._plume_table = None
            last = (steps - 1) % 2
            assert torch.equal(readback.result(last), sim.density.cpu()) and 0.0 <= float(host_res[last]) <= TOL
        return ms, info, launches, clocks

    # ---- mixed precision (headline)
    if args.only == "sor":  # profiler runs: the split-layout SOR sweep kernel alone
        if rank == 0:
            print(json.dumps({"only": "sor", "sor_split_kernel": sor_split_kernel(sg, dev, lib, _peaks()[0],
                                                                                 sweeps_per_launch=2, reps=1)}))
        if world > 1:
            dist.destroy_process_group()
        return 0
    only_fp64 = args.only == "fp64"
    sim = make(torch.float64, "fp64") if only_fp64 else make(torch.float32, "mixed")
    ms, info, launches, clocks = timed(sim, args.steps, args.warmup, sample_clocks=True)
    ms_max = max_over_ranks(ms)
    value = world * cells * args.steps / (ms_max / 1e3)
    relres_ok = info["failures"] == 0 and info["solves"] == args.steps
    if args.only:  # profiler runs: one timed region only
        if rank == 0:
            print(json.dumps({"metric": METRIC, "only": args.only, "value": value, "unit": UNIT,
                              "ms_per_step": ms_max / args.steps, "cycles": info["cycles"], "converged": relres_ok,
                              "gpu_launches": int(launches)}))
        if world > 1:
            dist.destroy_process_group()
        return 0
    # ---- end to end through the public API with host buffers
    ms_e2e, _, _, _ = timed(sim, args.steps, args.warmup, e2e=True)
    ms_e2e = max_over_ranks(ms_e2e)
    e2e_value = world * cells * args.steps / (ms_e2e / 1e3)
    h2d = 6 * 8 * len(sim.plumes)
    d2h = sim.density.numel() * sim.density.element_size()
    # ---- dominant kernel roofline. The solve's kernels run inside its CUDA graph, where
    # events cannot bracket one kernel, so the two fused fine-level kernels (which take most
    # of a cycle) are launched alone on the same plan and inputs right after the timed
    # region and timed with events on the launching stream.
    plan = solver.current_plan()
    peak, peak_kind = _peaks()
    H0, W0 = sc.H, sc.W
    n_rep = 20
    stream = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    p_scratch = torch.zeros((H0, W0), dtype=torch.float64, device=dev)

    def kernel_ms(which):
        plan.fine_kernel_async(which, p_scratch)
        torch.cuda.synchronize()
        ev[0].record(stream)
        for _ in range(n_rep):
            plan.fine_kernel_async(which, p_scratch)
        ev[1].record(stream)
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / n_rep

    post_ms, pre_ms = kernel_ms(1), kernel_ms(0)
    del p_scratch
    # the same kernel inside the solve graph, where it follows the kernels that leave part
    # of its inputs in L2: device durations of two more substeps from the CUDA activity
    # trace (events cannot be placed inside the graph's loop)
    in_graph_ms = None
    try:
        from torch.profiler import ProfilerActivity, profile

        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            for _ in range(2):
                sim.substep(sc.dt)
            torch.cuda.synchronize()
        d = [e.device_time_total for e in prof.key_averages() if "k_gmg_post_final" in e.key]
        n = [e.count for e in prof.key_averages() if "k_gmg_post_final" in e.key]
        if d and sum(n):
            in_graph_ms = sum(d) / sum(n) / 1e3
    except Exception:  # the trace is a cross-check; the events above are the figure
        in_graph_ms = None
    # algorithmic bytes per fine cell (mixed: cycle values TC = 4 B, fine values TP = 8 B)
    #   post: reads e_pre, rhs, p, r64 and a quarter cell of the coarse correction; writes
    #         p, r64 and the next rhs: 3 TC + 4 TP + TC / 4 = 45 B
    #   pre:  reads rhs; writes e and a quarter cell of the coarse rhs: 2.25 TC = 9 B
    post_bytes = 45 * H0 * W0
    pre_bytes = 9 * H0 * W0
    # the same kernel inside real substeps, timed with CUDA events on the solve's stream: the
    # solve runs its 5 cycles (the tolerance solve's count at 1e-8) kernel by kernel, and the
    # plan records an event pair around every fused fine-level post launch, so each duration
    # is that launch's on the device, after the kernels that precede it in a cycle
    n_step_k = 3
    simk = make(torch.float32, "mixed")
    simk.solver_params = dataclasses.replace(simk.solver_params, fixed_cycles=5)
    for _ in range(2):
        simk.substep(sc.dt)
    plan_k = solver.current_plan()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(2 * 5 * n_step_k)]
    for e in evs:
        e.record(stream)
    torch.cuda.synchronize()
    plan_k.set_post_events(evs)
    for _ in range(n_step_k):
        simk.substep(sc.dt)
    torch.cuda.synchronize()
    plan_k.set_post_events([])
    in_step = [evs[2 * q].elapsed_time(evs[2 * q + 1]) for q in range(5 * n_step_k)]
    in_step_ms = sum(in_step) / len(in_step)
    del simk
    achieved = post_bytes / (in_step_ms / 1e3) / 1e9
    achieved_alone = post_bytes / (post_ms / 1e3) / 1e9
    traffic = _measured_traffic("k_gmg_post_final_stage")
    # ---- error of the mixed path against the all-FP64 GPU path, same scene and steps
    errors = compare_fp64(sg, sc, make, 5)
    # ---- all-FP64 GPU path at the same residual
    del sim
    torch.cuda.empty_cache()
    sim64 = make(torch.float64, "fp64")
    ms64, info64, _, _ = timed(sim64, args.steps, args.warmup)
    ms64 = max_over_ranks(ms64)
    value64 = world * cells * args.steps / (ms64 / 1e3)
    fp64_ok = info64["failures"] == 0 and info64["solves"] == args.steps
    del sim64
    # ---- the second tolerance of the workload: both paths to 1e-10 (a short timed run each).
    # The float32 state's divergence sums to zero only up to rounding, which leaves a constant
    # part of the rhs near 1e-10 relative that no pressure removes; both solves take the fluid
    # mean off the rhs first (remove_mean), so that the target is reachable.
    tight = {"tol": TOL_TIGHT, "rhs": "fluid mean removed (remove_mean)"}
    k_tight = min(args.steps, 5)
    for name, dtype, precision in (("mixed", torch.float32, "mixed"), ("fp64", torch.float64, "fp64")):
        st = make(dtype, precision, TOL_TIGHT, remove_mean=True)
        ms_t, info_t, _, _ = timed(st, k_tight, args.warmup)
        ms_t = max_over_ranks(ms_t)
        tight[name] = {"value": world * cells * k_tight / (ms_t / 1e3), "ms_per_step": ms_t / k_tight,
                       "mean_cycles_per_step": info_t["cycles"] / max(info_t["solves"], 1),
                       "converged": bool(info_t["failures"] == 0 and info_t["solves"] == k_tight)}
        del st
    tight["mixed_speedup"] = tight["mixed"]["value"] / tight["fp64"]["value"]
    # ---- classical iterative refinement: k FP32 cycles on the correction between two FP64
    # passes (p += e, residual), against the headline's per-cycle correction in the fused fine
    # kernel (k = 1); same scene, residual and cycle type
    refinement = {"fused_per_cycle (inner 1)": {"value": value, "ms_per_step": ms_max / args.steps,
                                                "mean_cycles_per_step": info["cycles"] / max(info["solves"], 1)}}
    for k in (2, 3, 4):
        st = make(torch.float32, "mixed", inner=k)
        ms_k, info_k, _, _ = timed(st, k_tight, args.warmup)
        ms_k = max_over_ranks(ms_k)
        refinement[f"inner {k}"] = {"value": world * cells * k_tight / (ms_k / 1e3), "ms_per_step": ms_k / k_tight,
                                    "mean_cycles_per_step": info_k["cycles"] / max(info_k["solves"], 1),
                                    "converged": bool(info_k["failures"] == 0 and info_k["solves"] == k_tight)}
        del st
    torch.cuda.empty_cache()
    extras = None
    if rank == 0 and world == 1 and not args.no_extras:
        extras = other_workloads(sg, dev, lib, peak_gbs=_peaks()[0])
    # ---- CPU baseline on a bounded sample (rank 0, one GPU only)
    cpu = None
    cpu_error = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ofields = {}
        times, ccyc, threads = cpu_oracle_steps(args.cpu_steps, 1, ofields)
        cpu_error = compare_oracle(sg, sc, make, ofields)
        cpu = {"value": cells * len(times) / sum(times), "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{len(times)} substeps of mixed_2048 on the CPU oracle (C/OpenMP restatement of the "
                         f"reference kernels + the same multigrid, {COARSEST}x{COARSEST} exact coarsest, to "
                         f"1e-8), after 1 warm-up substep; mean {sum(ccyc) / max(len(ccyc), 1):.1f} cycles/step"}
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 state + f64/f32 mixed solve", "data": "synthetic",
        "config": mixed_config(info["cycles"] / max(info["solves"], 1), bool(relres_ok), f"replicas x{world}"),
        "fp64_gpu": {"value": value64, "ms_per_step": ms64 / args.steps,
                     "mean_cycles_per_step": info64["cycles"] / max(info64["solves"], 1), "converged": bool(fp64_ok),
                     "mixed_speedup": value / value64},
        "tol_1e-10": tight,
        "advection_arithmetic": {"float32_state": args.advection, "float64_state": "reference"},
        "operator_arithmetic": {"float32_state": args.advection, "float64_state": "reference",
                                "covers": "forces and the projection tail"},
        "clocks": clocks,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h + 8},
        "gpu_launches": int(launches),
        "roofline": {"kernel": "k_gmg_post_final_stage<float,double> (fine level: post-smoothing + correction + "
                               "residual)", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                     "alg_bytes_per_launch": post_bytes, "avg_launch_ms": in_step_ms, "launches": len(in_step),
                     "timing": "CUDA events on the solve's stream around each launch inside 3 substeps of the "
                               "workload whose solves run their 5 cycles kernel by kernel (graph-body kernels "
                               "cannot be bracketed by events)",
                     "alone": {"avg_launch_ms": post_ms, "achieved": achieved_alone, "frac": achieved_alone / peak,
                               "timing": "20 back-to-back launches on the bound plan, CUDA events around them "
                                         "(each launch re-reads its 189 MB from DRAM)"},
                     "in_graph": None if in_graph_ms is None else {
                         "avg_launch_ms": in_graph_ms, "achieved": post_bytes / (in_graph_ms / 1e3) / 1e9,
                         "frac": post_bytes / (in_graph_ms / 1e3) / 1e9 / peak,
                         "how": "CUDA activity trace (torch.profiler) of two substeps after the timed region"},
                     "also": {"k_gmg_pre_reg<float> (fine level pre-smoothing + restriction)": {
                         "avg_launch_ms": pre_ms, "alg_bytes_per_launch": pre_bytes,
                         "achieved": pre_bytes / (pre_ms / 1e3) / 1e9,
                         "frac": pre_bytes / (pre_ms / 1e3) / 1e9 / peak}}},
        "error_vs_fp64": errors,
        "error_vs_cpu_oracle": cpu_error,
        "refinement_modes": refinement,
        "workloads": extras,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    return 0


def _time_steps(torch, fn, steps, warmup):
    """CUDA-event time of `steps` calls of fn() after `warmup` calls (ms per call)."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps


def sor_split_kernel(sg, dev, lib, peak_gbs, n=4096, sweeps_per_launch=10, reps=3):
    """The split-layout red-black SOR sweep kernel alone (streaming half sweeps) at n^2, float32
    and float64, on a grid well above L2: 4 S bytes per cell and sweep moved (each half sweep
    reads the other colour's plane, its own plane and divergence, writes its own)."""
    import torch

    kern = {}
    for dtype in (torch.float32, torch.float64):
        code = sg._lib.dtype_code(torch.empty((), dtype=dtype))
        nb = int(lib.sg_rbsor_split_workspace_bytes(code, n, n))
        ws = torch.zeros(nb, dtype=torch.uint8, device=dev)
        s = sg._lib.stream_ptr()

        def sweeps(k, code=code, nb=nb, ws=ws, s=s):
            rc = lib.sg_rbsor_split_sweeps(code, n, n, ws.data_ptr(), nb, sg._lib.SG_MASK_OPEN, None, 0, None, 0,
                                           -1e-3, 0.25, 1.9, k, 0, s)
            assert rc == 0, lib.sg_last_error()
        ms = _time_steps(torch, lambda: sweeps(sweeps_per_launch), reps, 1) / sweeps_per_launch
        S = dtype.itemsize
        gbs = 4 * S * n * n / (ms / 1e3) / 1e9
        kern[str(dtype).replace("torch.", "")] = {"grid": [n, n], "us_per_sweep": ms * 1e3,
                                                  "bytes_per_cell_sweep": 4 * S, "achieved_gbs": gbs,
                                                  "frac": gbs / peak_gbs}
        del ws
    torch.cuda.empty_cache()
    return kern


def other_workloads(sg, dev, lib, peak_gbs):
    """Bounded runs of the other configurations, as sub-objects of the line:
    plume_512  512^2 plume: red-black SOR omega 1.9 (float64; float32 state with float64
               refinement) and multigrid V(2,2) RBGS omega 1, 8^2 coarsest (float64; float32
               state with the mixed solve), each to 1e-6; plus the split-layout SOR sweep kernel
               alone at 4096^2 (streaming half sweeps, 4 S bytes per cell and sweep moved)
    plume_128  128^2 plume, Jacobi x 100 per step, float64 (the reference's iterates)
    batch_256  the 256 batched scenes, mixed multigrid to 1e-6, autotuned, graph step
    inverse_256  the differentiable 256^2 x 64-step rollout: adjoint gradient against FP64
               central differences (eps = 1e-6 with the scatter that measures their rounding
               floor, and eps = 1e-4), and gradient-descent iterations in FP32"""
    import torch

    out = {}
    # ---- 512^2
    sc = sg.scenes.plume_512(0, steps=20)
    p512 = {"grid": [512, 512], "tol": 1e-6}
    runs = (("sor_fp64", "rb_sor_tolerance", sg.SORToleranceParams(omega=1.9, tol=1e-6, check_every=200),
             torch.float64, 3),
            ("sor_fp32_mixed", "rb_sor_tolerance",
             sg.SORToleranceParams(omega=1.9, tol=1e-6, check_every=200, precision="mixed"), torch.float32, 3),
            ("mg_fp64", "geometric_multigrid",
             sg.GeometricMultigridParams(tol=1e-6, max_cycles=60, omega=1.0, coarsest=8, precision="fp64"),
             torch.float64, 10),
            ("mg_fp32_mixed", "geometric_multigrid",
             sg.GeometricMultigridParams(tol=1e-6, max_cycles=60, omega=1.0, coarsest=8, precision="mixed"),
             torch.float32, 10))
    for name, method, params, dtype, steps in runs:
        sim = sg.scenes.make_sim(sc, method, params, dtype=dtype, device=dev)
        solver = sg.get_solver(method, "cuda")
        work = []

        def step(sim=sim, solver=solver, work=work, method=method):
            sim.substep(sc.dt)
            if method == "rb_sor_tolerance":
                work.append(solver.last_iterations)
                assert solver.converged
        ms = _time_steps(torch, step, steps, 2)
        entry = {"value": sc.cells / (ms / 1e3), "unit": "cell-steps/s", "ms_per_step": ms, "steps": steps}
        if method == "rb_sor_tolerance":
            entry["mean_sweeps_per_step"] = sum(work[2:]) / max(len(work) - 2, 1)
            entry["timing"] = "host-synchronised tolerance loop (residual read every 200 sweeps)"
        else:
            cyc, rel, ok = solver.last_cycles, solver.last_relres, solver.converged
            entry["last_cycles"], entry["last_relres"], entry["converged"] = cyc, rel, bool(ok)
        p512[name] = entry
        del sim
    p512["sor_split_kernel"] = sor_split_kernel(sg, dev, lib, peak_gbs)
    out["plume_512"] = p512
    torch.cuda.empty_cache()
    # ---- 128^2, Jacobi x 100, float64
    sc = sg.scenes.plume_128(steps=40)
    sim = sg.scenes.make_sim(sc, "jacobi", sg.JacobiParams(iterations=100), dtype=torch.float64, device=dev)
    ms = _time_steps(torch, lambda: sim.substep(sc.dt), 20, 3)
    out["plume_128"] = {"value": sc.cells / (ms / 1e3), "unit": "cell-steps/s", "ms_per_step": ms, "steps": 20,
                        "solver": "Jacobi x 100 (reference iterates), float64",
                        "hbm_ceiling_cell_steps_per_s": peak_gbs * 1e9 / 2568,
                        "note": "ceiling at (21 + 100 x 3) x 8 B per cell-step; 16384 cells sit in L2 and the step "
                                "is launch-bound (one launch per sweep)"}
    del sim
    # ---- batch of 256 scenes
    scenes = sg.scenes.batch_256(256, steps=10)
    b = sg.batch.BatchedSmoke(scenes, tol=1e-6, max_cycles=50, seed=1000, device=dev)
    b.step(2)
    choice = b.autotune(steps=2)
    b.step(3)
    _, _, tot0 = b.stats()
    ms = _time_steps(torch, lambda: b.step(1), 10, 0)
    _, rel, tot1 = b.stats()
    out["batch_256"] = {"value": b.cells / (ms / 1e3), "unit": "cell-steps/s", "ms_per_step": ms, "steps": 10,
                        "scenes": len(scenes), "cells": b.cells, "autotuned": choice,
                        "mean_cycles_per_scene_step": float((tot1 - tot0).sum()) / (len(scenes) * 10),
                        "scenes_not_converged_last_step": int((rel > 1e-6).sum())}
    del b
    torch.cuda.empty_cache()
    # ---- differentiable inverse problem, 256^2 x 64 steps, checkpoints every 8 steps
    inv = importlib.import_module("python-game-engine_b200.inverse")
    t0 = time.perf_counter()
    fdc = inv.fd_floor_check(256, 64, n_entries=8)
    fdc["seconds"] = time.perf_counter() - t0
    fdc.pop("rows")
    A = sg.adjoint
    model, force, target = A.inverse_problem(n=256, steps=64, dtype=torch.float32, precision="fp32", tol=1e-6,
                                             device=dev)
    iters = 10
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, hist = A.optimize(model, force, target, iters=iters, step=5.0)
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    out["inverse_256"] = {"fd_check_fp64": fdc, "checkpoint_every": 8,
                          "gradient_descent_fp32": {"iters": iters, "ms_per_iteration": 1e3 * sec / iters,
                                                    "loss_first": hist[0], "loss_last": hist[-1],
                                                    "loss_ratio": hist[-1] / hist[0]}}
    del model, force, target
    torch.cuda.empty_cache()
    return out


def run_batch(args):
    """The batch workload: 256 independent scenes of sizes drawn from {64, 96, 128, 192, 256},
    one plume each (seeded position, radius 4-16 % of the width, buoyancy 0.5-2), mixed-precision
    multigrid to 1e-6 per scene, one graph launch per step, autotuned configuration. Scenes
    are sharded across ranks by cell count (strong scaling: the batch is fixed)."""
    import torch
    import torch.distributed as dist

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    sg = importlib.import_module("python-game-engine_b200")
    lib = sg._lib.load()
    dev = torch.device("cuda", local)
    scenes = sg.scenes.batch_256(256, steps=args.steps)
    mine = sg.batch.shard_scenes(scenes, world, rank)
    b = sg.batch.BatchedSmoke([scenes[k] for k in mine], tol=1e-6, max_cycles=50, seed=1000, device=dev)
    b.step(2)  # leave the rest state so the autotuner sees moving smoke
    choice = b.autotune(steps=2)
    b.step(args.warmup)
    torch.cuda.synchronize()
    _, _, tot0 = b.stats()
    loops0 = b.loops()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    stream = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    l0 = lib.sg_launch_count()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev[0].record(stream)
    b.step(args.steps)
    ev[1].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = ev[0].elapsed_time(ev[1])
    clocks = sampler.stop()
    cyc, rel, tot1 = b.stats()
    cycles = int((tot1 - tot0).sum())
    cell_cycles = int(sum(int(dc) * s.H * s.W for dc, s in zip(tot1 - tot0, b.scenes)))
    step_nodes, cycle_nodes = b.graph_nodes()
    loops = b.loops() - loops0
    launches = step_nodes * args.steps + cycle_nodes * loops + (lib.sg_launch_count() - l0)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        c = torch.tensor([b.cells, cycles, int((rel > 1e-6).sum()), cell_cycles], dtype=torch.float64, device=dev)
        dist.all_reduce(c)
        total_cells, cycles, failed, cell_cycles = int(c[0]), int(c[1]), int(c[2]), int(c[3])
        dist.destroy_process_group()
    else:
        total_cells, failed = b.cells, int((rel > 1e-6).sum())
    if rank != 0:
        return 0
    value = total_cells * args.steps / (ms / 1e3)
    peak, peak_kind = _peaks()
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = cpu_oracle_batch(scenes, batch_sample(scenes), 2)
    # algorithmic bytes per cell and step outside the solver (float32): forces 12, advect u/v
    # 12 + 12, advect density + dissipation 16, divergence 12, projection 20, metrics
    # divergence 12 + residual 12 = 108 B; per cycle the solver moves >= the fine level's
    # ~110 B (mixed refinement: float32 V-cycle plus the float64 correction and residual)
    alg_bytes = total_cells * 108 * args.steps + 110 * cell_cycles
    line = {
        "metric": BATCH_METRIC,
        "workload": "batch_256", "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32 state + f64/f32 mixed solve", "data": "synthetic",
        "config": {"workload": "batch_256", "scenes": len(scenes), "cells": total_cells, "tol": 1e-6,
                   "autotuned": choice, "mean_cycles_per_scene_step": cycles / (len(scenes) * args.steps),
                   "cycle_loops_per_step": loops / args.steps,
                   "scenes_not_converged_last_step": failed, "parallelism": f"scene shards x{world}"},
        "clocks": clocks, "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "peak": peak, "unit": "GB/s", "peak_kind": peak_kind,
                     "non_solver_alg_bytes_per_step": total_cells * 108,
                     "note": "whole-step figure: algorithmic bytes of the non-solver operators and of the "
                             "solver's fine level per cycle (~110 B / cell) over the step time",
                     "achieved": alg_bytes / (ms / 1e3) / 1e9},
    }
    line["roofline"]["frac"] = line["roofline"]["achieved"] / peak
    line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fixed-cycles", type=int, default=0,
                    help="profiling: run this many cycles per solve kernel by kernel instead of the graph loop")
    ap.add_argument("--workload", choices=["mixed_2048", "batch_256"], default="mixed_2048")
    ap.add_argument("--advection", choices=["float32", "reference"], default="float32",
                    help="arithmetic of the float32 state's advection: float32 (relative to the cell) or the "
                         "reference's float64 positions and weights (bit for bit)")
    ap.add_argument("--no-extras", action="store_true", help="skip the other workloads' sub-objects")
    ap.add_argument("--coarsest", type=int, default=COARSEST,
                    help="exact coarsest level side of the 2048^2 multigrid (cosine transform; 17..256)")
    ap.add_argument("--no-reference-numba", action="store_true",
                    help="reference arm: skip timing the reference's own Numba code beside the oracle port")
    ap.add_argument("--only", choices=["mixed", "fp64", "sor"], default=None,
                    help="time one path only, without e2e / roofline / CPU parts (for profiler runs)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        sys.exit(run_reference(args))
    sys.exit(run_batch(args) if args.workload == "batch_256" else run_ours(args))


if __name__ == "__main__":
    main()
