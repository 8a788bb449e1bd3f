"""Red-black SOR on the checkerboard-split layout against the natural-layout kernel and the
CPU oracle (red_black_sor_gauss_seidel.py:8-42).

* The split planes give the same iterates as sg_rbsor_solve bit for bit, for both kernel
  variants (one launch per half sweep; shared-memory tiles of up to four sweeps), on odd and
  even extents, every mask kind and sweep counts that exercise the tile launches' splitting.
* The tolerance loop (sg_rbsor_tol_solve) stops after the same number of sweeps as the
  oracle's loop and returns the same pressure bit for bit, and its residual norm equals the
  natural-layout residual's.
"""
import ctypes

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
L = sg._lib


def _case(H, W, dtype, seed, obstacles):
    rng = np.random.default_rng(seed)
    solid = np.zeros((H, W), bool)
    if obstacles:
        solid = O.box_solid(H, W)
        solid[H // 3:H // 3 + max(H // 6, 1), W // 4:W // 2] = True
    fmu, fmv = O.face_masks_from_solid(solid)
    npdt = np.float32 if dtype == torch.float32 else np.float64
    div = rng.uniform(-1, 1, (H, W)).astype(npdt)
    p0 = rng.uniform(-1, 1, (H, W)).astype(npdt)
    return p0, div, fmu, fmv


def _masks(kind, fmu, fmv):
    if kind == "planes":
        mu = torch.from_numpy(fmu.astype(np.uint8)).cuda()
        mv = torch.from_numpy(fmv.astype(np.uint8)).cuda()
        return L.SG_MASK_PLANES, mu, mv
    return (L.SG_MASK_OPEN if kind == "open" else L.SG_MASK_RING), None, None


def _ws(dtype, H, W):
    code = L.dtype_code(torch.empty((), dtype=dtype))
    n = int(L.load().sg_rbsor_split_workspace_bytes(code, H, W))
    t = torch.empty(n, dtype=torch.uint8, device="cuda")
    assert t.data_ptr() % 256 == 0
    return t, code, n


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("shape,kind", [((16, 16), "open"), ((17, 13), "ring"), ((33, 70), "planes"),
                                        ((64, 129), "open"), ((100, 64), "ring"), ((97, 131), "planes"),
                                        ((1, 9), "open"), ((70, 2), "open")])
@pytest.mark.parametrize("variant", [0, 1])
def test_split_sweeps_equal_natural_layout(dtype, shape, kind, variant):
    H, W = shape
    lib = L.load()
    s = L.stream_ptr()
    p0, div, fmu, fmv = _case(H, W, dtype, 11 + H + W, kind == "planes")
    mode, mu, mv = _masks(kind, fmu, fmv)
    pu = ctypes.c_void_p(mu.data_ptr()) if mu is not None else None
    pv = ctypes.c_void_p(mv.data_ptr()) if mv is not None else None
    d = dev(div)
    ws, code, n = _ws(dtype, H, W)
    alpha, omega = -0.37, 1.9
    for iters in (1, 2, 3, 5, 8):
        ref = dev(p0)
        rc = lib.sg_rbsor_solve(code, H, W, ref.data_ptr(), W, d.data_ptr(), W, mode, pu, W + 1, pv, W, alpha, 0.25,
                                omega, iters, s)
        assert rc == L.SG_OK, lib.sg_last_error()
        start = dev(p0)
        assert lib.sg_rbsor_split_pack(code, H, W, start.data_ptr(), W, 0, ws.data_ptr(), n, s) == L.SG_OK
        assert lib.sg_rbsor_split_pack(code, H, W, d.data_ptr(), W, 1, ws.data_ptr(), n, s) == L.SG_OK
        rc = lib.sg_rbsor_split_sweeps(code, H, W, ws.data_ptr(), n, mode, pu, W + 1, pv, W, alpha, 0.25, omega, iters,
                                       variant, s)
        assert rc == L.SG_OK, lib.sg_last_error()
        got = torch.empty_like(start)
        assert lib.sg_rbsor_split_unpack(code, H, W, ws.data_ptr(), n, got.data_ptr(), W, s) == L.SG_OK
        torch.cuda.synchronize()
        assert torch.equal(got, ref), f"iterations {iters}: max {float((got - ref).abs().max()):.3e}"


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_split_sumsq_equals_natural_residual(dtype):
    H, W = 75, 92
    lib = L.load()
    s = L.stream_ptr()
    p0, div, fmu, fmv = _case(H, W, dtype, 5, True)
    mode, mu, mv = _masks("planes", fmu, fmv)
    p, d = dev(p0), dev(div)
    ws, code, n = _ws(dtype, H, W)
    lib.sg_rbsor_split_pack(code, H, W, p.data_ptr(), W, 0, ws.data_ptr(), n, s)
    lib.sg_rbsor_split_pack(code, H, W, d.data_ptr(), W, 1, ws.data_ptr(), n, s)
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    for zero_p in (0, 1):
        rc = lib.sg_rbsor_split_sumsq(code, H, W, ws.data_ptr(), n, mode, ctypes.c_void_p(mu.data_ptr()), W + 1,
                                      ctypes.c_void_p(mv.data_ptr()), W, -0.37, 0.25, zero_p,
                                      ctypes.c_void_p(out.data_ptr() + 8 * zero_p), s)
        assert rc == L.SG_OK, lib.sg_last_error()
    torch.cuda.synchronize()
    fl = O.is_fluid_from_faces(fmu, fmv)
    r = O.compute_residual(p0.copy(), div, fl, fmu, fmv, -0.37, 0.25, np.empty_like(p0))
    r0 = O.compute_residual(np.zeros_like(p0), div, fl, fmu, fmv, -0.37, 0.25, np.empty_like(p0))
    got = out.cpu().numpy()
    assert got[0] == pytest.approx(float(np.sum(r.astype(np.float64) ** 2)), rel=1e-12)
    assert got[1] == pytest.approx(float(np.sum(r0.astype(np.float64) ** 2)), rel=1e-12)


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-6), (torch.float32, 1e-3)])
@pytest.mark.parametrize("variant", [0, 1])
def test_tolerance_solve_matches_oracle_loop(dtype, tol, variant):
    """A plume step's divergence (96 x 80, closed box): same sweep count as the oracle's loop,
    pressure bit for bit."""
    H, W = 96, 80
    npdt = np.float32 if dtype == torch.float32 else np.float64
    ora = O.OracleSim(H, W, 1.0 / W, O.jacobi_pressure_solver, dict(iterations=0), dtype=npdt)
    ora.dt, ora.gravity = 0.5 / W, -1.0
    ora.plumes = [O.PlumeSpec(40.0, 9.6, 8.0, 1.0, 1.0, 0.05, seed=3)]
    ora.substep(ora.dt)
    div = ora.divergence.copy()
    p_ref = np.zeros((H, W), npdt)
    it_ref, rel_ref = O.rb_sor_tolerance(p_ref, div, ora.fmu, ora.fmv, 1.0, 1.0 / W, ora.dt, omega=1.9, tol=tol,
                                         check_every=50)
    solver = sg.SORToleranceSolver()
    p = torch.zeros((H, W), dtype=dtype, device="cuda")
    solver(p, dev(div), sg.OPEN_BOX, sg.OPEN_BOX, 1.0, 1.0 / W, ora.dt, omega=1.9, tol=tol, check_every=50,
           strict=True, variant=variant)
    assert solver.converged and solver.last_iterations == it_ref
    assert solver.last_relres == pytest.approx(rel_ref, rel=1e-9)
    assert np.array_equal(p.cpu().numpy(), p_ref)


def test_mixed_solve_matches_oracle_refinement():
    """float32 fields to 1e-7 (below float32's floor): same sweeps and refinements as the
    oracle's refinement loop, pressure bit for bit, float64 residual at the target."""
    H, W = 96, 80
    ora = O.OracleSim(H, W, 1.0 / W, O.jacobi_pressure_solver, dict(iterations=0), dtype=np.float32)
    ora.dt, ora.gravity = 0.5 / W, -1.0
    ora.plumes = [O.PlumeSpec(40.0, 9.6, 8.0, 1.0, 1.0, 0.05, seed=3)]
    ora.substep(ora.dt)
    div = ora.divergence.copy()
    p_ref = np.zeros((H, W), np.float32)
    it_ref, rel_ref, outer_ref = O.rb_sor_mixed(p_ref, div, ora.fmu, ora.fmv, 1.0, 1.0 / W, ora.dt, omega=1.9,
                                                tol=1e-7, check_every=50)
    solver = sg.SORToleranceSolver()
    p = torch.zeros((H, W), dtype=torch.float32, device="cuda")
    solver(p, dev(div), sg.OPEN_BOX, sg.OPEN_BOX, 1.0, 1.0 / W, ora.dt, omega=1.9, tol=1e-7, check_every=50,
           strict=True, precision="mixed")
    assert solver.converged and rel_ref <= 1e-7 and outer_ref >= 2
    assert (solver.last_iterations, solver.last_refinements) == (it_ref, outer_ref)
    assert solver.last_relres == pytest.approx(rel_ref, rel=1e-9)
    assert np.array_equal(p.cpu().numpy(), p_ref)


def test_tolerance_solve_reports_unreached_tolerance():
    H = W = 40
    p0, div, fmu, fmv = _case(H, W, torch.float64, 2, False)
    div -= div.mean()
    solver = sg.SORToleranceSolver()
    p = torch.zeros((H, W), dtype=torch.float64, device="cuda")
    with pytest.raises(sg.NotConverged):
        solver(p, dev(div), sg.OPEN_BOX, sg.OPEN_BOX, 1.0, 1.0 / W, 0.5 / W, tol=1e-30, max_iterations=30,
               check_every=10, strict=True)
    assert solver.last_iterations == 30 and not solver.converged
