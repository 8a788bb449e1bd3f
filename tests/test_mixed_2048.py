"""The 2048^2 four-source scene over 20 substeps: the mixed-precision path (float32 state,
FP32 V(2,2) cycles in FP64 iterative refinement to 1e-8, 128^2 exact coarsest) against the
all-FP64 GPU path and against the CPU oracle (the reference's kernels restated in C with the
same multigrid, mixed precision, to 1e-8).

Stated tolerances (relative L2; pressure with its mean removed, the pressure being defined up
to a constant):
* vs the CPU oracle, reference advection arithmetic: the operators are bit-exact and the
  solves differ by the rounding of their FP32 cycles: density 1e-6, velocity 1e-5,
  pressure 1e-5.
* vs the CPU oracle, float32 advection arithmetic: density 1e-5, velocity 1e-5, pressure 1e-5
  (the float32 bar).
* vs the all-FP64 GPU path: the float32 state's rounding: density 1e-5, velocity 1e-4,
  pressure 1e-4.
* every solve reaches 1e-8; post-projection divergence on cells >= 2 from the wall ring is at
  most 1e-8 * ||divergence before the solve|| plus the float32 rounding of the faces.
"""
import numpy as np
import pytest
import torch

from conftest import package

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("CUDA device required", allow_module_level=True)

import oracle as O  # noqa: E402
from sim_checks import check_divergence_bound, recording  # noqa: E402

sg = package()
STEPS = 20
TOL = 1e-8


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _prel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return _rel(a - a.mean(), b - b.mean())


@pytest.fixture(scope="module")
def oracle_fields():
    sc = sg.scenes.mixed_2048(steps=STEPS)
    fmu, fmv = O.face_masks_from_solid(np.zeros((sc.H, sc.W), bool))
    fl = O.is_fluid_from_faces(fmu, fmv)
    gmg = O.GMGOracle(fmu, fmv, fl, coarsest=128, omega=1.3)
    rec = []

    def solver(p, div, fmu_, fmv_, rho, h, dt, **_):
        b = O.alpha_coeff(h, rho, dt) * div.astype(np.float64) * fl
        p64 = np.zeros(p.shape)
        c, hist = gmg.solve(p64, b, tol=TOL, max_cycles=40, precision="mixed")
        rec.append(hist[-1])
        p[:] = p64.astype(p.dtype)

    sim = O.OracleSim(sc.H, sc.W, sc.cell_size, solver, {}, dtype=np.float32)
    sim.dt, sim.gravity = sc.dt, sc.gravity
    sim.plumes = [O.PlumeSpec(*row, seed=sc.seed) for row in sc.plumes]
    for _ in range(STEPS):
        sim.substep(sc.dt)
    assert max(rec) <= TOL
    return {n: getattr(sim, n).copy() for n in ("density", "velocity_u", "velocity_v", "pressure")}


def _run(dtype, precision, arithmetic="reference"):
    sc = sg.scenes.mixed_2048(steps=STEPS)
    params = sg.GeometricMultigridParams(tol=TOL, max_cycles=40, precision=precision, omega=1.3, coarsest=128)
    sim = sg.scenes.make_sim(sc, "geometric_multigrid", params, dtype=dtype)
    sim.advection_arithmetic = arithmetic
    sim.operator_arithmetic = arithmetic
    name, norms = recording("geometric_multigrid")
    sim.pressure_solver_method = name
    solver = sg.get_solver("geometric_multigrid", "cuda")
    for _ in range(STEPS):
        norms.clear()
        sim.substep(sc.dt)
        assert solver.converged and solver.last_relres <= TOL
        check_divergence_bound(sim, norms[-1], TOL)
    out = {n: getattr(sim, n).double().cpu().numpy() for n in ("density", "velocity_u", "velocity_v", "pressure")}
    del sim
    torch.cuda.empty_cache()
    return out


@pytest.fixture(scope="module")
def fp64_fields():
    return _run(torch.float64, "fp64")


def test_mixed_reference_arithmetic_vs_oracle_and_fp64(oracle_fields, fp64_fields):
    g = _run(torch.float32, "mixed")
    o = oracle_fields
    assert np.max(o["density"]) > 0.5
    assert _rel(g["density"], o["density"]) <= 1e-6
    assert _rel(g["velocity_u"], o["velocity_u"]) <= 1e-5
    assert _rel(g["velocity_v"], o["velocity_v"]) <= 1e-5
    assert _prel(g["pressure"], o["pressure"]) <= 1e-5
    f = fp64_fields
    assert _rel(g["density"], f["density"]) <= 1e-5
    assert _rel(g["velocity_u"], f["velocity_u"]) <= 1e-4
    assert _rel(g["velocity_v"], f["velocity_v"]) <= 1e-4
    assert _prel(g["pressure"], f["pressure"]) <= 1e-4


def test_mixed_float32_arithmetic_vs_oracle(oracle_fields):
    g = _run(torch.float32, "mixed", arithmetic="float32")
    o = oracle_fields
    for n in ("density", "velocity_u", "velocity_v"):
        assert _rel(g[n], o[n]) <= 1e-5, n
    assert _prel(g["pressure"], o["pressure"]) <= 1e-5
