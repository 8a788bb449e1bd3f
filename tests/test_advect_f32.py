"""float32 fields in float32 arithmetic -- advection (sg_advect_velocity_f32 /
sg_advect_scalar_f32) against the oracle's restatement of the reference kernels
(advection.py:112-180), which evaluate positions and weights in float64; the forces
(sg_apply_forces_f32) and the projection tail (sg_project_metrics_f32) against the
reference-arithmetic CUDA kernels, which equal the reference's bit for bit
(test_cuda_parity.py).

Stated tolerance: 1e-5 of the field's largest magnitude per value (the float32 bar); the
measured differences are rounding (~1e-7). Cases: backtraces of up to 3 cells that leave the
grid at every edge, odd shapes, every mask kind, and 20 plume substeps with the float32
advection against the oracle's reference-arithmetic substeps.
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
ops = sg.operators
TOL = 1e-5


def _case(H, W, seed, kind):
    rng = np.random.default_rng(seed)
    h = 1.0 / max(H, W)
    dt = 0.5 * h
    # |vel| * dt / h up to 3 cells
    u = rng.uniform(-6, 6, (H, W + 1)).astype(np.float32)
    v = rng.uniform(-6, 6, (H + 1, W)).astype(np.float32)
    src = rng.uniform(0, 1, (H, W)).astype(np.float32)
    solid = np.zeros((H, W), bool)
    if kind == "ring":
        solid = O.box_solid(H, W)
    if kind == "planes":
        solid = O.box_solid(H, W)
        solid[H // 3:H // 2, W // 4:W // 2] = True
    fmu, fmv = O.face_masks_from_solid(solid)
    fl = O.is_fluid_from_faces(fmu, fmv)
    return u, v, src, fmu, fmv, fl, dt, h


def _mask_args(kind, fmu, fmv, fl):
    if kind == "open":
        return sg.OPEN_BOX, sg.OPEN_BOX, sg.OPEN_BOX
    if kind == "ring":
        return sg.RING_BOX, sg.RING_BOX, sg.RING_BOX
    return dev(fmu), dev(fmv), dev(fl)


@pytest.mark.parametrize("shape", [(64, 64), (61, 45), (130, 257)])
@pytest.mark.parametrize("kind", ["open", "ring", "planes"])
def test_float32_arithmetic_matches_reference_kernels(shape, kind):
    H, W = shape
    u, v, src, fmu, fmv, fl, dt, h = _case(H, W, H * 7 + W, kind)
    if kind == "open":
        fmu_o, fmv_o = O.face_masks_from_solid(np.zeros((H, W), bool))
        fl_o = O.is_fluid_from_faces(fmu_o, fmv_o)
    elif kind == "ring":
        # the analytic ring mask: the open masks with the ring's faces closed
        fmu_o, fmv_o = O.face_masks_from_solid(O.box_solid(H, W))
        fl_o = O.is_fluid_from_faces(fmu_o, fmv_o)
    else:
        fmu_o, fmv_o, fl_o = fmu, fmv, fl
    ue, ve, de = np.zeros_like(u), np.zeros_like(v), np.zeros_like(src)
    O.advect_velocity_u(u, ue, v, fmu_o, dt, h)
    O.advect_velocity_v(v, ve, u, fmv_o, dt, h)
    O.advect_scalar_field(src, de, ue, ve, fl_o, dt, h)
    mu, mv, mf = _mask_args(kind, fmu, fmv, fl)
    ud, vd, sd = dev(np.zeros_like(u)), dev(np.zeros_like(v)), dev(np.zeros_like(src))
    ops.advect_velocity(dev(u), ud, dev(v), vd, mu, mv, dt, h, arithmetic="float32")
    # the density step reads the advected velocity, as the substep does
    ops.advect_scalar_field(dev(src), sd, dev(ue), dev(ve), mf, dt, h, arithmetic="float32")
    for got, exp in ((ud, ue), (vd, ve), (sd, de)):
        g = got.cpu().numpy()
        assert np.all(np.isfinite(g))
        assert np.max(np.abs(g - exp)) <= TOL * max(np.max(np.abs(exp)), 1e-30)
    # the mask zeros are exact
    assert np.array_equal(ud.cpu().numpy() == 0, ue == 0) or kind == "open"


def test_float32_arithmetic_plume_20_steps_vs_oracle():
    sc = sg.scenes.plume_128(steps=20)
    cu = sg.scenes.make_sim(sc, "jacobi", sg.JacobiParams(iterations=100), dtype=torch.float32)
    cu.advection_arithmetic = "float32"
    cu.operator_arithmetic = "float32"
    ora = O.OracleSim(sc.H, sc.W, sc.cell_size, O.jacobi_pressure_solver, dict(iterations=100), dtype=np.float32)
    ora.dt, ora.gravity = sc.dt, sc.gravity
    ora.plumes = [O.PlumeSpec(*row, seed=sc.seed) for row in sc.plumes]
    for _ in range(sc.steps):
        cu.substep(sc.dt)
        ora.substep(sc.dt)
    for name in ("density", "velocity_u", "velocity_v", "pressure"):
        g = getattr(cu, name).double().cpu().numpy()
        e = getattr(ora, name).astype(np.float64)
        assert np.linalg.norm(g - e) <= TOL * np.linalg.norm(e), name
    assert float(cu.density.max()) > 0.5


@pytest.mark.parametrize("temperature", [False, True])
@pytest.mark.parametrize("shape", [(64, 64), (61, 45), (130, 257)])
def test_float32_forces_match_reference_arithmetic(temperature, shape):
    """forces.py:19-105: buoyancy from the face-averaged density (rows 0 and H - 1 take their
    own row, row H none) and temperature; 1e-5 of |v|."""
    H, W = shape
    g = torch.Generator().manual_seed(H + W)
    v = torch.randn((H + 1, W), generator=g).cuda()
    d = torch.rand((H, W), generator=g).cuda()
    t = (300.0 + 20.0 * torch.rand((H, W), generator=g)).cuda() if temperature else None
    args = (0.5 / W, -9.81, 0.7, 1.3, 300.0)
    v_ref, v_f32 = v.clone(), v.clone()
    ops.apply_forces(v_ref, d, t, *args)
    ops.apply_forces(v_f32, d, t, *args, arithmetic="float32")
    assert not torch.equal(v_ref, v)
    assert float((v_f32 - v_ref).abs().max()) <= TOL * float(v_ref.abs().max())


@pytest.mark.parametrize("planes", [False, True])
@pytest.mark.parametrize("shape", [(64, 64), (61, 45), (130, 257)])
def test_float32_projection_tail_matches_reference_arithmetic(planes, shape):
    """The fused projection tail (projection out of place, divergence and residual after it)
    in float32 arithmetic: each output within 1e-5 of its magnitude of the reference-
    arithmetic kernel's, and the same zeros on closed and solid faces."""
    H, W = shape
    g = torch.Generator().manual_seed(3 * H + W)
    u, v, p = torch.randn((H, W + 1), generator=g).cuda(), torch.randn((H + 1, W), generator=g).cuda(), \
        torch.randn((H, W), generator=g).cuda()
    if planes:
        solid = torch.zeros((H, W), dtype=torch.bool)
        solid[0, :] = solid[-1, :] = solid[:, 0] = solid[:, -1] = True
        solid[H // 3:H // 2 + 1, W // 3:W // 2 + 1] = True
        fmu, fmv, fl = ops.build_masks(solid.cuda())
        solid_arg = solid.cuda()
    else:
        fmu = fmv = fl = sg.OPEN_BOX
        solid_arg = sg.RING_BOX
    h, dt, rho = 1.0 / W, 0.5 / W, 1.0
    alpha = sg.calculate_alpha(h, rho, dt)
    outs = {}
    for arith in ("reference", "float32"):
        u2, v2 = torch.empty_like(u), torch.empty_like(v)
        d2, r2 = torch.empty_like(p), torch.empty_like(p)
        ops.project_metrics(u, v, u2, v2, p, fmu, fmv, fl, solid_arg, rho, h, dt, alpha, 0.25, d2, r2,
                            arithmetic=arith)
        outs[arith] = (u2, v2, d2, r2)
    for a, b in zip(outs["reference"], outs["float32"]):
        assert float((a - b).abs().max()) <= TOL * float(a.abs().max())
        assert torch.equal(a == 0, b == 0) or not planes
