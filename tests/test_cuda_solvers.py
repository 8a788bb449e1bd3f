"""CUDA solvers and multi-step scenes against the CPU oracle.

* plume_128 (128^2, Jacobi x100, float64): 200 CUDA steps vs 200 oracle steps; the
  stated tolerance is 1e-12 absolute on density (the operators are bit-exact).
* Convergent multigrid (no reference counterpart; oracle = the project's FP64 C
  restatement, GMGOracle): one cycle within 1e-10 relative of the oracle's cycle,
  the tolerance targets float64 1e-10, mixed 1e-8, float32 1e-5, and the converged
  pressure (mean removed) within 1e-6 / 1e-4 / 5e-2 relative of the oracle's.
* Failure detection without faulting the GPU: non-finite input and an unreachable
  tolerance come back as host exceptions.
"""
import numpy as np
import pytest
import torch

from conftest import package

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("CUDA device required", allow_module_level=True)

import oracle as O  # noqa: E402
from cuda_adapter import dev  # noqa: E402

sg = package()
scenes = sg.scenes
OMEGA = 1.3  # the red-black over-relaxation of both the CUDA multigrid and the oracle's


def _oracle_sim(scene, solver, kw, dtype):
    s = O.OracleSim(scene.H, scene.W, scene.cell_size, solver, kw, dtype=dtype)
    s.dt = scene.dt
    s.gravity = scene.gravity
    s.plumes = [O.PlumeSpec(*row, seed=scene.seed) for row in scene.plumes]
    return s


def test_plume_128_200_steps_fp64_vs_oracle():
    sc = scenes.plume_128(steps=200)
    cu = scenes.make_sim(sc, "jacobi", sg.JacobiParams(iterations=100), dtype=torch.float64)
    ora = _oracle_sim(sc, O.jacobi_pressure_solver, dict(iterations=100), np.float64)
    for _ in range(sc.steps):
        cu.substep(sc.dt)
        ora.substep(sc.dt)
    d_err = np.max(np.abs(cu.density.cpu().numpy() - ora.density))
    u_err = np.max(np.abs(cu.velocity_u.cpu().numpy() - ora.velocity_u))
    p_err = np.max(np.abs(cu.pressure.cpu().numpy() - ora.pressure))
    assert np.max(ora.density) > 0.5
    assert d_err <= 1e-12 and u_err <= 1e-12 and p_err <= 1e-12, (d_err, u_err, p_err)


def test_plume_128_fp32_20_steps_vs_oracle():
    sc = scenes.plume_128(steps=20)
    cu = scenes.make_sim(sc, "jacobi", sg.JacobiParams(iterations=100), dtype=torch.float32)
    ora = _oracle_sim(sc, O.jacobi_pressure_solver, dict(iterations=100), np.float32)
    for _ in range(sc.steps):
        cu.substep(sc.dt)
        ora.substep(sc.dt)
    assert np.array_equal(cu.density.cpu().numpy(), ora.density)
    assert np.array_equal(cu.velocity_v.cpu().numpy(), ora.velocity_v)


def _problem(H, W, obstacles, seed):
    rng = np.random.default_rng(seed)
    solid = np.zeros((H, W), bool)
    if obstacles:
        solid = O.box_solid(H, W)
        solid[H // 3:H // 3 + H // 8, W // 4:W // 2] = True
    fmu, fmv = O.face_masks_from_solid(solid)
    fl = O.is_fluid_from_faces(fmu, fmv)
    div = rng.standard_normal((H, W)) * fl
    div[fl] -= div[fl].mean()
    return fmu, fmv, fl, div


@pytest.mark.parametrize("shape,obstacles,cycle,precision", [
    ((64, 64), False, "V", "fp64"), ((96, 80), True, "V", "fp64"), ((37, 50), True, "V", "fp64"),
    ((256, 256), False, "V", "fp64"), ((300, 260), True, "V", "fp64"), ((200, 176), False, "W", "fp64"),
    ((96, 80), True, "W", "fp64"), ((1100, 1300), False, "V", "fp64"), ((1201, 1025), False, "V", "fp64"),
    ((1100, 1300), False, "W", "fp32"), ((1201, 1025), False, "V", "fp32"), ((1100, 1300), False, "V", "mixed")])
def test_gmg_one_cycle_vs_oracle(shape, obstacles, cycle, precision):
    """Coarse levels run in a single-block tail kernel, open-box levels in the tiled level
    kernels (register tiles on levels large enough to fill the GPU, the fine one fused with
    the correction and residual; 16 x 16 shared-memory tiles below), levels with obstacles
    in the grid-wide kernels."""
    H, W = shape
    fmu, fmv, fl, div = _problem(H, W, obstacles, 1)
    alpha = -0.7
    g = O.GMGOracle(fmu, fmv, fl, coarsest=8, omega=OMEGA, cycle=cycle)
    pe = np.zeros((H, W))
    g.vcycle(0, pe, alpha * div)
    solver = sg.GeometricMultigridSolver()
    masks = (sg.OPEN_BOX, sg.OPEN_BOX) if not obstacles else (dev(fmu), dev(fmv))
    p = torch.zeros((H, W), dtype=torch.float32 if precision == "fp32" else torch.float64, device="cuda")
    # cell_size, rho, dt chosen so that alpha = -(h^2) rho / dt = -0.7
    solver(p, dev(div.astype(np.float64 if precision == "fp64" else np.float32)), masks[0], masks[1], 0.7, 1.0, 1.0,
           precision=precision, fixed_cycles=1, cycle=cycle, omega=OMEGA)
    got = p.double().cpu().numpy()
    tol = 1e-10 if precision == "fp64" else 2e-5
    assert np.max(np.abs(got - pe)) <= tol * np.max(np.abs(pe))


@pytest.mark.parametrize("shape,cycle,precision", [
    ((64, 64), "V", "fp64"), ((200, 176), "V", "fp64"), ((200, 176), "W", "fp64"), ((20, 30), "V", "fp64"),
    ((1100, 1300), "V", "fp64"), ((1100, 1300), "V", "mixed"), ((1201, 1025), "W", "fp32")])
def test_gmg_one_cycle_cosine_coarsest_vs_oracle(shape, cycle, precision):
    """coarsest=32: the last level (<= 32 a side, open box) is solved exactly by the cosine
    transform instead of a dense pseudo-inverse; one cycle must equal the oracle's cycle with
    the pseudo-inverse of that level (a single-level grid is solved outright)."""
    H, W = shape
    fmu, fmv, fl, div = _problem(H, W, False, 3)
    alpha = -0.7
    g = O.GMGOracle(fmu, fmv, fl, coarsest=32, omega=OMEGA, cycle=cycle)
    pe = np.zeros((H, W))
    g.vcycle(0, pe, alpha * div)
    solver = sg.GeometricMultigridSolver()
    p = torch.zeros((H, W), dtype=torch.float32 if precision == "fp32" else torch.float64, device="cuda")
    solver(p, dev(div.astype(np.float64 if precision == "fp64" else np.float32)), sg.OPEN_BOX, sg.OPEN_BOX, 0.7,
           1.0, 1.0, precision=precision, fixed_cycles=1, cycle=cycle, coarsest=32, omega=OMEGA)
    got = p.double().cpu().numpy()
    tol = 1e-10 if precision == "fp64" else 2e-5
    assert np.max(np.abs(got - pe)) <= tol * np.max(np.abs(pe))


@pytest.mark.parametrize("shape,coarsest,cycle,precision", [
    ((512, 512), 128, "V", "fp64"), ((1024, 768), 256, "V", "fp64"), ((300, 260), 80, "V", "fp64"),
    ((300, 260), 80, "W", "fp64"), ((2048, 2048), 256, "V", "mixed"), ((2048, 2048), 128, "V", "mixed"),
    ((2048, 2048), 128, "V", "fp64"), ((1024, 768), 256, "V", "fp32"),
    ((200, 176), 256, "V", "fp64")])
def test_gmg_one_cycle_large_cosine_coarsest_vs_oracle(shape, coarsest, cycle, precision):
    """coarsest above 64 (up to 256): the last level is solved exactly by the cosine transform
    written as four tiled products over many blocks (k_dct_gemm); one cycle must equal the
    oracle's cycle, whose coarsest solve is the same transform in float64 (scipy's orthonormal
    DCT-II, checked against the dense pseudo-inverse in the oracle tests). Odd and rectangular
    coarsest levels (75 x 65, 256 x 192) and a grid that is its own coarsest level (200 x 176)
    included."""
    H, W = shape
    fmu, fmv, fl, div = _problem(H, W, False, 5)
    alpha = -0.7
    g = O.GMGOracle(fmu, fmv, fl, coarsest=coarsest, omega=OMEGA, cycle=cycle)
    assert g.coarse_dct
    pe = np.zeros((H, W))
    g.vcycle(0, pe, alpha * div)
    solver = sg.GeometricMultigridSolver()
    p = torch.zeros((H, W), dtype=torch.float32 if precision == "fp32" else torch.float64, device="cuda")
    solver(p, dev(div.astype(np.float64 if precision == "fp64" else np.float32)), sg.OPEN_BOX, sg.OPEN_BOX, 0.7,
           1.0, 1.0, precision=precision, fixed_cycles=1, cycle=cycle, coarsest=coarsest, omega=OMEGA)
    got = p.double().cpu().numpy()
    tol = 1e-10 if precision == "fp64" else 2e-5
    assert np.max(np.abs(got - pe)) <= tol * np.max(np.abs(pe))
    # rows of whole 16-byte units run the two streaming launches, the rest the four products
    plan = solver.current_plan()
    Wc = plan.level_shape(plan.num_levels - 1)[1]
    streams = (Wc * (8 if precision == "fp64" else 4)) % 16 == 0
    assert plan.coarse_solve_kind() in (plan.COARSE_SOLVE_KINDS[3:] if streams else plan.COARSE_SOLVE_KINDS[2:3])


def test_gmg_large_cosine_coarsest_reaches_1e8_in_no_more_cycles():
    """The 2048^2 scene's first solve to 1e-8 (mixed): an exact 256^2 coarsest level needs no
    more V(2,2) cycles than the exact 32^2 one."""
    sc = scenes.mixed_2048(steps=1)
    cycles = {}
    for coarsest in (32, 256):
        params = sg.GeometricMultigridParams(tol=1e-8, precision="mixed", max_cycles=30, coarsest=coarsest,
                                             omega=OMEGA)
        sim = scenes.make_sim(sc, "geometric_multigrid", params, dtype=torch.float32)
        sim.substep(sc.dt)
        solver = sg.get_solver("geometric_multigrid", "cuda")
        assert solver.converged and solver.last_relres <= 1e-8
        cycles[coarsest] = solver.last_cycles
    assert cycles[256] <= cycles[32], cycles


@pytest.mark.parametrize("precision,obstacles", [("fp64", False), ("mixed", False), ("mixed", True)])
def test_gmg_remove_mean_reaches_1e10(precision, obstacles):
    """An rhs whose sum is not zero (as float rounding leaves a divergence) has a constant part
    no pressure removes: the residual stalls above it. With remove_mean the fluid mean is
    taken off first and the solve reaches 1e-10; its pressure equals the oracle's solve of
    the mean-free rhs."""
    H = W = 256
    fmu, fmv, fl, div = _problem(H, W, obstacles, 4)
    div = (div + 1e-7 * np.abs(div).max()) * fl
    d = dev(div.astype(np.float64 if precision == "fp64" else np.float32))
    h, rho, dt = 1.0 / H, 1.0, 0.5 / H
    masks = (sg.OPEN_BOX, sg.OPEN_BOX) if not obstacles else (dev(fmu), dev(fmv))
    coarsest = 8 if obstacles else 32  # the cosine-transform coarsest level needs an open box
    solver = sg.GeometricMultigridSolver()
    p = torch.zeros((H, W), dtype=torch.float64, device="cuda")
    solver(p, d, *masks, rho, h, dt, tol=1e-10, max_cycles=40, precision=precision, coarsest=coarsest)
    assert not solver.converged and solver.last_relres > 1e-10
    p.zero_()
    solver(p, d, *masks, rho, h, dt, tol=1e-10, max_cycles=40, precision=precision, coarsest=coarsest,
           remove_mean=True, strict=True)
    assert solver.converged and solver.last_relres <= 1e-10 and solver.last_cycles <= (20 if obstacles else 12)
    alpha = O.alpha_coeff(h, rho, dt)
    b = alpha * d.double().cpu().numpy() * fl
    b[fl] -= b[fl].mean()  # the mean over the fluid cells
    g = O.GMGOracle(fmu, fmv, fl)
    pe = np.zeros((H, W))
    g.solve(pe, b, tol=1e-13, max_cycles=60)
    got = p.double().cpu().numpy()
    a, e = got[fl] - got[fl].mean(), pe[fl] - pe[fl].mean()
    assert np.max(np.abs(a - e)) <= 1e-5 * np.max(np.abs(e))  # two 1e-10 solves differ by <~ kappa * 1e-10


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-8), ("fp32", 1e-5)])
@pytest.mark.parametrize("obstacles", [False, True])
def test_gmg_reaches_tolerance(precision, tol, obstacles):
    H = W = 128
    fmu, fmv, fl, div = _problem(H, W, obstacles, 2)
    solver = sg.GeometricMultigridSolver()
    masks = (sg.OPEN_BOX, sg.OPEN_BOX) if not obstacles else (dev(fmu), dev(fmv))
    dtype = torch.float32 if precision == "fp32" else torch.float64
    p = torch.zeros((H, W), dtype=dtype, device="cuda")
    d = dev(div.astype(np.float32 if precision != "fp64" else np.float64))
    solver(p, d, masks[0], masks[1], 1.0, 1.0 / H, 0.5 / H, tol=tol, max_cycles=40, precision=precision, strict=True)
    assert solver.converged and solver.last_relres <= tol and solver.last_cycles <= 20
    # converged solution vs the oracle's FP64 solve of the same problem (mean removed)
    alpha = O.alpha_coeff(1.0 / H, 1.0, 0.5 / H)
    g = O.GMGOracle(fmu, fmv, fl)
    pe = np.zeros((H, W))
    g.solve(pe, alpha * d.double().cpu().numpy() * fl, tol=1e-12, max_cycles=60)
    got = p.double().cpu().numpy()
    a = got[fl] - got[fl].mean()
    b = pe[fl] - pe[fl].mean()
    # two solutions with relative residuals <= tol differ by at most ~ (lambda_max / lambda_min) * tol
    # relative (about 1.3e4 * tol at 128^2); the bounds below sit well inside that
    bound = {"fp64": 1e-6, "mixed": 1e-4, "fp32": 5e-2}[precision]
    assert np.max(np.abs(a - b)) <= bound * np.max(np.abs(b))


def _true_relres(p, b):
    """||b - A p|| / ||b|| on an open box, A p = sum over open faces of p - p_nb (float64)."""
    r = b.copy()
    r[:, 1:] += p[:, :-1] - p[:, 1:]
    r[:, :-1] += p[:, 1:] - p[:, :-1]
    r[1:, :] += p[:-1, :] - p[1:, :]
    r[:-1, :] += p[1:, :] - p[:-1, :]
    return np.linalg.norm(r) / np.linalg.norm(b)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-8), ("fp32", 1e-4)])
def test_gmg_large_grid_reported_residual_is_true(precision, tol):
    """On grids large enough for the fused fine-level kernel the residual is carried from
    cycle to cycle (r - A e) rather than recomputed; the relative residual the solver reports
    must still be the true one of the returned pressure, and the solve must get there."""
    H, W = 1100, 1300
    _, _, _, div = _problem(H, W, False, 4)
    solver = sg.GeometricMultigridSolver()
    p = torch.zeros((H, W), dtype=torch.float32 if precision == "fp32" else torch.float64, device="cuda")
    d = dev(div.astype(np.float64 if precision == "fp64" else np.float32))
    solver(p, d, sg.OPEN_BOX, sg.OPEN_BOX, 1.0, 1.0 / H, 0.5 / H, tol=tol, max_cycles=40, precision=precision,
           strict=True)
    assert solver.converged and solver.last_relres <= tol
    alpha = O.alpha_coeff(1.0 / H, 1.0, 0.5 / H)
    b = alpha * d.double().cpu().numpy()
    true = _true_relres(p.double().cpu().numpy(), b)
    # the reported value tracks the true one to rounding (FP32: to the rounding of p itself)
    slack = {"fp64": 1e-3, "mixed": 1e-3, "fp32": 0.5}[precision]
    assert abs(true - solver.last_relres) <= slack * tol + 1e-13


def test_gmg_fixed_cycles_residual_history():
    H = W = 256
    fmu, fmv, fl, div = _problem(H, W, False, 3)
    solver = sg.GeometricMultigridSolver()
    p = torch.zeros((H, W), dtype=torch.float64, device="cuda")
    solver(p, dev(div), sg.OPEN_BOX, sg.OPEN_BOX, 1.0, 1.0 / H, 0.5 / H, precision="mixed", fixed_cycles=8)
    hist = solver.last_relres_dev.cpu().numpy()
    assert hist[0] == pytest.approx(1.0)
    assert np.all(np.diff(hist) < 0) and hist[-1] < 1e-7


def test_sor_tolerance_reaches_1e6():
    H = W = 48
    fmu, fmv, fl, div = _problem(H, W, False, 4)
    s = sg.SORToleranceSolver()
    p = torch.zeros((H, W), dtype=torch.float64, device="cuda")
    s(p, dev(div), sg.OPEN_BOX, sg.OPEN_BOX, 1.0, 1.0 / H, 0.5 / H, omega=1.9, tol=1e-6, check_every=50, strict=True)
    assert s.converged and s.last_relres <= 1e-6


def test_nonfinite_input_is_reported():
    H = W = 32
    div = np.zeros((H, W))
    div[5, 5] = np.nan
    p = torch.zeros((H, W), dtype=torch.float64, device="cuda")
    with pytest.raises(sg.SmokeCudaError):
        sg.GeometricMultigridSolver()(p, dev(div), sg.OPEN_BOX, sg.OPEN_BOX, 1.0, 1.0, 1.0, precision="fp64", strict=True)
    # the context stays usable after the reported failure
    q = torch.ones(4, device="cuda")
    assert float(q.sum()) == 4.0


def test_unreachable_tolerance_is_reported():
    H = W = 64
    fmu, fmv, fl, div = _problem(H, W, False, 5)
    p = torch.zeros((H, W), dtype=torch.float64, device="cuda")
    s = sg.GeometricMultigridSolver()
    with pytest.raises(sg.NotConverged):
        s(p, dev(div), sg.OPEN_BOX, sg.OPEN_BOX, 1.0, 1.0, 1.0, precision="fp64", tol=1e-30, max_cycles=3, strict=True)
    assert s.last_cycles == 3


def test_bad_arguments_raise_before_launch():
    t = torch.zeros((8, 8), device="cuda")
    with pytest.raises(ValueError):
        sg.operators.compute_divergence(t, t, t, sg.OPEN_BOX, sg.OPEN_BOX, 1.0)  # wrong u/v shapes
    with pytest.raises(TypeError):
        sg.operators.cool_temperature(torch.zeros((4, 4), dtype=torch.int32, device="cuda"), 0.0, 0.5, 0.1)


def test_gmg_step_sim_mixed_2048_short():
    """Two steps of the 2048^2 scene: mixed precision reaches 1e-8 each step."""
    sc = scenes.mixed_2048(steps=2)
    params = sg.GeometricMultigridParams(tol=1e-8, precision="mixed", max_cycles=30)
    sim = scenes.make_sim(sc, "geometric_multigrid", params, dtype=torch.float32)
    solver = sg.get_solver("geometric_multigrid", "cuda")
    for _ in range(2):
        sim.substep(sc.dt)
        assert solver.converged and solver.last_relres <= 1e-8
    assert float(sim.density.max()) > 0.5


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape", [(37, 50), (100, 131), (1, 7), (130, 2)])
@pytest.mark.parametrize("iters", [1, 7, 8, 9, 17])
def test_jacobi_multi_sweep_tiles_vs_oracle(dtype, shape, iters):
    """jacobi.py:27-52 with up to 8 sweeps per launch (shared-memory tiles, used for grids in
    L2): bit for bit against the oracle's sweeps, on odd shapes, thin grids, obstacle planes
    and sweep counts that end inside a launch."""
    H, W = shape
    rng = np.random.default_rng(H * 31 + W + iters)
    solid = np.zeros((H, W), bool)
    if H > 8 and W > 8:
        solid = O.box_solid(H, W)
        solid[H // 3:H // 3 + 3, W // 4:W // 2] = True
    fmu, fmv = O.face_masks_from_solid(solid)
    div = rng.uniform(-1, 1, (H, W)).astype(dtype)
    p0 = rng.uniform(-1, 1, (H, W)).astype(dtype)
    exp = p0.copy()
    O.jacobi_pressure_solver(exp, div, fmu, fmv, 1.0, 1.0 / W, 0.5 / W, iterations=iters)
    got = dev(p0)
    sg.solvers.jacobi_pressure_solver(got, dev(div), dev(fmu), dev(fmv), 1.0, 1.0 / W, 0.5 / W, iterations=iters)
    assert np.array_equal(got.cpu().numpy(), exp)


@pytest.mark.parametrize("precision,pdtype", [("fp64", torch.float64), ("fp32", torch.float32),
                                              ("mixed", torch.float64)])
def test_gmg_fused_post_kernel_staged_and_unstaged_agree(precision, pdtype):
    """The fused fine-level post kernel stages the caller's pressure rows (and, in mixed
    precision, the carried float64 residual) in shared memory with bulk asynchronous copies
    when they start on 16-byte boundaries, and reads them from global memory otherwise. Both
    forms run the same arithmetic: a pressure array whose rows sit one element off a 16-byte
    boundary (row stride W + 2) must come out of a 3-cycle solve with the same bits, and with
    the same relative residual, as a contiguous one."""
    H, W = 1024, 1280
    _, _, _, div = _problem(H, W, False, 7)
    d = dev(div.astype(np.float32 if precision == "fp32" else np.float64))
    out = []
    for off in (False, True):
        if off:
            base = torch.zeros((H, W + 2), dtype=pdtype, device="cuda")
            p = base[:, 1:W + 1]
            assert (p.data_ptr() % 16) != 0
        else:
            p = torch.zeros((H, W), dtype=pdtype, device="cuda")
        solver = sg.GeometricMultigridSolver()
        solver(p, d, sg.OPEN_BOX, sg.OPEN_BOX, 0.7, 1.0, 1.0, precision=precision, fixed_cycles=3, coarsest=32,
               omega=OMEGA)
        assert solver.current_plan().fine_fused()
        out.append((p.clone(), solver.last_relres))
    assert torch.equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1]


@pytest.mark.parametrize("precision,remove_mean", [("mixed", False), ("mixed", True), ("fp64", False)])
def test_gmg_first_cycle_from_divergence_equals_prologue_residual(precision, remove_mean):
    """A graph solve from a zero guess on the fused fine level lets its first post kernel take
    p = 0 and, in mixed precision, form the carried float64 residual alpha div (- the fluid
    mean) from the divergence itself; a divergence whose rows are off 16-byte boundaries falls
    back to the prologue writing that residual and the kernel reading it. Both must give the
    same bits: pressure, cycle count and relative residual."""
    H, W = 1024, 1280
    _, _, _, div = _problem(H, W, False, 9)
    d = dev(div.astype(np.float32))
    base = torch.zeros((H, W + 4), dtype=torch.float32, device="cuda")
    base[:, 1:W + 1] = d
    d_off = base[:, 1:W + 1]
    assert d_off.data_ptr() % 16 != 0
    out = []
    for dd in (d, d_off):
        p = torch.zeros((H, W), dtype=torch.float64, device="cuda")
        solver = sg.GeometricMultigridSolver()
        solver(p, dd, sg.OPEN_BOX, sg.OPEN_BOX, 0.7, 1.0, 1.0, tol=1e-8, max_cycles=30, precision=precision,
               coarsest=32, omega=OMEGA, zero_initial_guess=True, remove_mean=remove_mean)
        assert solver.current_plan().fine_fused()
        out.append((p.clone(), solver.last_cycles, solver.last_relres))
    assert out[0][1] == out[1][1] and out[0][1] >= 3
    assert out[0][2] == out[1][2] and out[0][2] <= 1e-8
    assert torch.equal(out[0][0], out[1][0])
