"""CUDA path vs the reference (golden fixtures) and the CPU oracle.

Tolerances: the operators restate the reference's arithmetic, so the non-fastmath
ones are checked bit for bit; the bar of the project is 1e-6 relative (float64) and
1e-5 relative (float32) per operator, which every test below also states. Red-black
SOR and Gauss-Seidel are compiled with fastmath=True by the reference and compared at
that bar only.
"""
import glob
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN, golden, package

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # collected on CPU-only hosts, run on the GPU box
    pytest.skip("CUDA device required", allow_module_level=True)

import kats  # noqa: E402
import oracle as O  # noqa: E402
from cuda_adapter import CudaOps, dev  # noqa: E402
from test_oracle_golden import oracle_ops  # noqa: E402

sg = package()
OPS_FILES = sorted(os.path.basename(f)[:-4] for f in glob.glob(os.path.join(GOLDEN, "ops_*.npz")))
FASTMATH = {"rbsor", "rbsor_auto", "gauss_seidel"}


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30))


def tol(dtype):
    return 1e-5 if dtype == np.float32 else 1e-6


def cuda_ops(d):
    """The oracle_ops() set of outputs, computed by the CUDA library."""
    h, dt = float(d["h"]), float(d["dt"])
    fl, fmu, fmv, solid = d["fl"], d["fmu"], d["fmv"], d["solid"]
    C = CudaOps
    out = {}
    o = np.zeros_like(d["dens"]); C.advect_scalar_field(d["dens"], o, d["u"], d["v"], fl, dt, h); out["adv_scalar"] = o
    o = np.zeros_like(d["u"]); C.advect_velocity_u(d["u"], o, d["v"], fmu, dt, h); out["adv_u"] = o
    o = np.zeros_like(d["v"]); C.advect_velocity_v(d["v"], o, d["u"], fmv, dt, h); out["adv_v"] = o
    vv = d["v"].copy(); C.apply_forces(vv, d["dens"], d["temp"], dt, -0.5, 5.0, 1.0, 0.1); out["forces_v"] = vv
    tt = d["temp"].copy(); C.cool_temperature(tt, 0.1, 0.5, dt); out["cool_t"] = tt
    o = np.zeros_like(d["dens"]); C.compute_divergence(d["u"], d["v"], o, fmu, fmv, h); out["divergence"] = o
    alpha = O.alpha_coeff(h, 1.0, dt)
    o = np.zeros_like(d["dens"]); C.compute_residual(d["p"], d["div"], fl, fmu, fmv, alpha, 0.25, o); out["residual"] = o
    uu, vv = d["u"].copy(), d["v"].copy(); C.apply_pressure_gradient(uu, vv, d["p"], fmu, fmv, 1.3, h, dt)
    out["grad_u"], out["grad_v"] = uu, vv
    uu, vv = d["u"].copy(), d["v"].copy(); C.enforce_boundary_conditions(uu, vv, solid)
    out["bc_u"], out["bc_v"] = uu, vv
    pp = np.zeros_like(d["p"]); C.jacobi_pressure_solver(pp, d["div"], fmu, fmv, 1.0, h, dt, iterations=23)
    out["jacobi"] = pp
    pp = d["p"].copy(); C.rb_sor_pressure_solver(pp, d["div"], fmu, fmv, 1.0, h, dt, iterations=9, omega=1.7)
    out["rbsor"] = pp
    pp = d["p"].copy(); C.rb_sor_pressure_solver(pp, d["div"], fmu, fmv, 1.0, h, dt, iterations=5, omega=0.0)
    out["rbsor_auto"] = pp
    pp = d["p"].copy(); C.gauss_seidel_pressure_solver(pp, d["div"], fmu, fmv, 1.0, h, dt, iterations=4)
    out["gauss_seidel"] = pp
    if "restrict" in d:
        H, W = d["p"].shape
        t = dev(np.zeros((H // 2, W // 2), d["p"].dtype))
        sgl = sg._lib
        flt = dev(fl)
        sgl.call("sg_mg_restrict_average", sgl.dtype_code(t), H, W, dev(d["p"]).data_ptr(), W, sgl.SG_MASK_PLANES,
                 flt.data_ptr(), W, t.data_ptr(), W // 2, H // 2, W // 2, 1.0, sgl.stream_ptr())
        out["restrict"] = t.cpu().numpy()
        f = dev(np.zeros_like(d["p"]))
        sgl.call("sg_mg_prolong", sgl.dtype_code(f), H // 2, W // 2, dev(d["restrict"]).data_ptr(), W // 2, H, W,
                 sgl.SG_MASK_PLANES, flt.data_ptr(), W, f.data_ptr(), W, 0, sgl.stream_ptr())
        out["prolong"] = f.cpu().numpy()
        s = dev((~fl).astype(np.uint8))
        c = torch.zeros((H // 2, W // 2), dtype=torch.uint8, device="cuda")
        sgl.call("sg_mg_coarsen_solid", H, W, s.data_ptr(), W, c.data_ptr(), W // 2, sgl.stream_ptr())
        out["coarsen"] = c.cpu().numpy().astype(bool)
    return out


@pytest.mark.parametrize("name", OPS_FILES)
def test_operators_vs_reference_within_tolerance(name):
    d = golden(name)
    dtype = d["dens"].dtype
    for key, val in cuda_ops(d).items():
        assert rel(val, d[key]) <= tol(dtype), (key, rel(val, d[key]))


@pytest.mark.parametrize("name", OPS_FILES)
def test_operators_vs_reference_bit_exact(name):
    d = golden(name)
    for key, val in cuda_ops(d).items():
        if key in FASTMATH:
            continue
        assert np.array_equal(val, d[key]), (key, rel(val, d[key]))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape", [(96, 128), (61, 45)])
def test_operators_vs_oracle_random(shape, dtype):
    """Seeded inputs at sizes the golden set does not cover, against the live oracle."""
    H, W = shape
    rng = np.random.default_rng(H * 1000 + W)
    solid = O.box_solid(H, W)
    solid[H // 3:H // 3 + 4, W // 2:W // 2 + 5] = True
    fmu, fmv = O.face_masks_from_solid(solid)
    fl = O.is_fluid_from_faces(fmu, fmv)
    h = 1.0 / max(H, W)
    d = dict(solid=solid, fmu=fmu, fmv=fmv, fl=fl, h=np.float64(h), dt=np.float64(2.3 * h),
             dens=rng.uniform(0, 1, (H, W)).astype(dtype), temp=rng.uniform(-1, 1, (H, W)).astype(dtype),
             u=rng.uniform(-1, 1, (H, W + 1)).astype(dtype), v=rng.uniform(-1, 1, (H + 1, W)).astype(dtype),
             p=rng.uniform(-1, 1, (H, W)).astype(dtype), div=rng.uniform(-1, 1, (H, W)).astype(dtype))
    exp = oracle_ops(d)
    got = cuda_ops(d)
    for key in exp:
        assert rel(got[key], exp[key]) <= tol(dtype), (key, rel(got[key], exp[key]))
        if key not in FASTMATH:
            assert np.array_equal(got[key], exp[key]), key


def test_kat_square_uv_shapes():
    d = golden("kat_square_uv")
    for t in ("f32", "f64"):
        o = np.zeros_like(d[f"{t}_src"])
        CudaOps.advect_scalar_field(d[f"{t}_src"], o, d[f"{t}_u"], d[f"{t}_v"], d["fl"], 1.0, 1.0)
        assert np.array_equal(o, d[f"{t}_out"])


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("kat", kats.ALL_OPERATOR_KATS, ids=lambda f: f.__name__)
def test_reference_kats_on_cuda(kat, dtype, face_masks):
    kat(CudaOps, face_masks, dtype=dtype)


def test_div_grad_random_on_cuda(face_masks, small_random_grid):
    kats.kat_div_grad_random(CudaOps, face_masks, small_random_grid)


@pytest.mark.parametrize("solver", ["jacobi_pressure_solver", "rb_sor_pressure_solver", "gauss_seidel_pressure_solver"])
def test_zero_pipeline_noop_on_cuda(face_masks, solver):
    fn = getattr(CudaOps, solver)
    kats.kat_zero_pipeline_noop(CudaOps, face_masks, lambda *a: fn(*a, iterations=10))


@pytest.mark.parametrize("dt_name", ["f32", "f64"])
@pytest.mark.parametrize("case", ["jac", "sor", "jac5"])
def test_reference_multigrid_on_cuda(case, dt_name):
    d = golden("multigrid")
    kw = {
        "jac": dict(smoother_type="jacobi", v_cycles=1, num_levels=4, smoother_iterations=2, coarsest_iterations=30),
        "sor": dict(smoother_type="rb_sor_gauss_seidel", v_cycles=2, num_levels=3, smoother_iterations=2,
                    coarsest_iterations=20),
        "jac5": dict(smoother_type="jacobi", v_cycles=2, num_levels=5, smoother_iterations=3, coarsest_iterations=40),
    }[case]
    H = W = 32
    fmu, fmv = O.face_masks_from_solid(O.box_solid(H, W))
    div = d["div_" + dt_name]
    p = torch.zeros(div.shape, dtype=torch.float32 if dt_name == "f32" else torch.float64, device="cuda")
    sg.MultigridSolver()(p, dev(div), dev(fmu), dev(fmv), 1.0, 1.0 / H, 0.5 / H, **kw)
    ref = d[f"mg_{case}_{dt_name}"]
    got = p.cpu().numpy()
    assert rel(got, ref) <= tol(div.dtype)
    if case != "sor":
        assert np.array_equal(got, ref)


SIM_CASES = {
    "jacobi": ("jacobi", sg.JacobiParams(iterations=30)),
    "rbsor": ("rb_sor_gauss_seidel", sg.SORParams(iterations=20, omega=1.8)),
    "mg": ("multigrid", sg.MultigridParams(smoother_type="jacobi", num_levels=3, v_cycles=2, smoother_iterations=2,
                                           coarsest_iterations=20)),
    "gs": ("gauss_seidel", sg.GaussSeidelParams(iterations=10)),
}


@pytest.mark.parametrize("name", list(SIM_CASES))
def test_substeps_vs_reference(name):
    """Eight SmokeSimulation2D substeps (reference float32 simulator) on CUDA."""
    method, params = SIM_CASES[name]
    d = golden("sim")
    cfg = sg.SimulationConfig(grid=sg.GridConfig(size=(32, 32), cell_size=1.0 / 32),
                              pressure_solver=sg.PressureSolverConfig(method=method, params=params))
    sim = sg.SmokeSimulation2D(cfg)
    sim.add_emitter(sg.Emitter2D(position=(16, 6), radius=4.0, density_value=3.0, temperature_value=2.0,
                                 velocity_value=(0.3, 2.0), approach="linear", numba_optimized=True))
    for step in range(8):
        sim.substep(sim.dt)
        if step in (0, 7):
            for k, attr in (("density", "density"), ("u", "velocity_u"), ("v", "velocity_v"), ("p", "pressure"),
                            ("t", "temperature"), ("div", "divergence"), ("res", "pressure_residual")):
                got = getattr(sim, attr).cpu().numpy()
                ref = d[f"{name}_s{step}_{k}"]
                scale = max(np.max(np.abs(ref)), 1.0)
                assert np.max(np.abs(got - ref)) <= 1e-5 * scale, (step, k, np.max(np.abs(got - ref)))
                if name in ("jacobi", "mg"):
                    assert np.array_equal(got, ref), (step, k)


def test_plume_source_vs_oracle():
    H, W = 40, 36
    rng = np.random.default_rng(9)
    for dtype in (np.float32, np.float64):
        dens = rng.uniform(0, 1, (H, W)).astype(dtype)
        u = rng.uniform(-1, 1, (H, W + 1)).astype(dtype)
        v = rng.uniform(-1, 1, (H + 1, W)).astype(dtype)
        specs = [O.PlumeSpec(12.3, 7.7, 5.5, 1.0, 1.0, 0.05, seed=123), O.PlumeSpec(20.0, 9.0, 4.0, 0.7, 1.3, 0.02,
                                                                                    seed=123)]
        ed, eu, ev = dens.copy(), u.copy(), v.copy()
        for s in specs:
            s.apply(ed, eu, ev, 17)
        td, tu, tv = dev(dens), dev(u), dev(v)
        table = np.array([[s.cx, s.cy, s.radius, s.density_value, s.v_value, s.noise_amp] for s in specs])
        sg.operators.plume_sources(td, tu, tv, table, 123, 17)
        assert np.array_equal(td.cpu().numpy(), ed)
        assert np.array_equal(tu.cpu().numpy(), eu)
        assert np.array_equal(tv.cpu().numpy(), ev)


@pytest.mark.parametrize("approach", ["linear", "gaussian", "quadratic", "hard_cutoff"])
def test_emitters_vs_reference(approach):
    d = golden("emitters")
    f = torch.zeros((24, 20), dtype=torch.float32, device="cuda")
    for _ in range(2):
        sg.operators.emit_scalar(f, 1.7, 0.016, 8.5, 10.25, 5.5, approach)
    got = f.cpu().numpy()
    assert rel(got, d[approach + "_numba"]) <= 1e-6
    assert rel(got, d[approach + "_python"]) <= 1e-6


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("planes", [False, True])
@pytest.mark.parametrize("H, W", [(67, 90), (64, 31), (9, 33), (3, 65), (130, 64)])
def test_fused_tail_equals_separate_operators(dtype, planes, H, W):
    """project_metrics (projection out of place + divergence + residual in one pass) must
    give bit for bit what project, compute_divergence and compute_residual give (shapes
    with partial warps, partial row strips and warp-edge columns)."""
    g = torch.Generator().manual_seed(11)
    r = lambda *s: torch.randn(s, generator=g, dtype=torch.float64).to(dtype).cuda()  # noqa: E731
    u, v, p = r(H, W + 1), r(H + 1, W), r(H, W)
    if planes:
        solid = torch.zeros((H, W), dtype=torch.bool)
        solid[0, :] = solid[-1, :] = solid[:, 0] = solid[:, -1] = True
        solid[H // 3:H // 2 + 1, W // 3:W // 2 + 1] = True
        fmu, fmv, fl = sg.operators.build_masks(solid.cuda())
        solid_arg = solid.cuda()
    else:
        fmu = fmv = fl = sg.OPEN_BOX
        solid_arg = sg.RING_BOX
    h, dt, rho = 1.0 / W, 0.5 / W, 1.0
    alpha = sg.calculate_alpha(h, rho, dt)
    # separate passes
    u1, v1 = u.clone(), v.clone()
    sg.operators.project(u1, v1, p, fmu, fmv, solid_arg, rho, h, dt)
    d1 = torch.empty((H, W), dtype=dtype, device="cuda")
    sg.operators.compute_divergence(u1, v1, d1, fmu, fmv, h)
    r1 = torch.empty_like(d1)
    sg.operators.compute_residual(p, d1, fl, fmu, fmv, alpha, 0.25, r1)
    # fused
    u2, v2, d2, r2 = torch.empty_like(u), torch.empty_like(v), torch.empty_like(d1), torch.empty_like(d1)
    sg.operators.project_metrics(u, v, u2, v2, p, fmu, fmv, fl, solid_arg, rho, h, dt, alpha, 0.25, d2, r2)
    for a, b in ((u1, u2), (v1, v2), (d1, d2), (r1, r2)):
        assert torch.equal(a, b)


@pytest.mark.parametrize("name", ["jacobi", "mg"])
def test_substeps_with_obstacles_vs_reference(name):
    """set_solid_mask with interior obstacles (a rectangle and a disc inside the wall ring)
    before the third substep: masks rebuilt at the next substep (simulation.py:133-143,
    :198-204), the reference multigrid rebuilding its hierarchy (rebuild_masks=True). Bit for
    bit against the reference's own substeps."""
    method, params = SIM_CASES[name]
    if name == "mg":
        params = sg.MultigridParams(smoother_type="jacobi", num_levels=3, v_cycles=2, smoother_iterations=2,
                                    coarsest_iterations=20, rebuild_masks=True)
    d = golden("sim_obstacles")
    cfg = sg.SimulationConfig(grid=sg.GridConfig(size=(32, 32), cell_size=1.0 / 32),
                              pressure_solver=sg.PressureSolverConfig(method=method, params=params))
    sim = sg.SmokeSimulation2D(cfg)
    sim.add_emitter(sg.Emitter2D(position=(16, 6), radius=4.0, density_value=3.0, temperature_value=2.0,
                                 velocity_value=(0.3, 2.0), approach="linear", numba_optimized=True))
    for step in range(8):
        if step == 2:
            sim.set_solid_mask(d["solid"].astype(np.uint8))
        sim.substep(sim.dt)
        if step in (1, 2, 7):
            for k, attr in (("density", "density"), ("u", "velocity_u"), ("v", "velocity_v"), ("p", "pressure"),
                            ("t", "temperature"), ("div", "divergence"), ("res", "pressure_residual")):
                got = getattr(sim, attr).cpu().numpy()
                assert np.array_equal(got, d[f"{name}_s{step}_{k}"]), (step, k)
