"""Known-answer tests of the reference, restated once against a pluggable backend.

The reference's unit/integration tests (tests/cfd/unit/test_advection.py,
test_divergence.py, test_pressure_gradient.py, test_pressure_solver.py,
tests/cfd/integration/test_projection.py, test_pipeline_invariants.py) check the
operators on 16x16 float32 grids with atol 1e-6. Each ``kat_*`` function here
takes ``ops``, an object exposing the reference operator signatures on numpy
arrays (in place), so the same checks run on the CPU oracle and on the CUDA
library (through a host<->device adapter).
"""
import numpy as np

ATOL = 1e-6


def _is_fluid(fmu, fmv):
    return fmu[:, :-1] | fmu[:, 1:] | fmv[:-1, :] | fmv[1:, :]


# ------------------------------------------------------------ advection (test_advection.py)
def kat_zero_velocity_advection(ops, face_masks, dtype=np.float32):
    fmu, fmv = face_masks
    fl = _is_fluid(fmu, fmv)
    u = np.zeros((16, 16), dtype)
    v = np.zeros((16, 16), dtype)
    s = np.random.default_rng(3).random((16, 16)).astype(dtype)
    dst = np.zeros_like(s)
    ops.advect_scalar_field(s, dst, u, v, fl, 0.1, 1.0)
    assert np.allclose(dst[1:-1, 1:-1], s[1:-1, 1:-1], atol=ATOL)


def kat_constant_velocity_advection(ops, face_masks, dtype=np.float32):
    fmu, fmv = face_masks
    fl = _is_fluid(fmu, fmv)
    s = np.full((16, 16), 7.0, dtype)
    u = np.full((16, 16), 3.0, dtype)
    v = np.full((16, 16), -2.0, dtype)
    dst = np.zeros_like(s)
    ops.advect_scalar_field(s, dst, u, v, fl, 0.1, 1.0)
    assert np.allclose(dst[1:-1, 1:-1], s[1:-1, 1:-1], atol=ATOL)


def kat_rightward_shift(ops, face_masks, dtype=np.float32):
    fmu, fmv = face_masks
    fl = _is_fluid(fmu, fmv)
    u = np.ones((16, 16), dtype)
    v = np.zeros((16, 16), dtype)
    s = np.tile(np.arange(16, dtype=dtype), (16, 1))
    dst = np.zeros_like(s)
    ops.advect_scalar_field(s, dst, u, v, fl, 1.0, 1.0)
    assert np.allclose(dst[1:-1, 2:-1], s[1:-1, 1:-2], atol=ATOL)


def kat_upward_shift(ops, face_masks, dtype=np.float32):
    fmu, fmv = face_masks
    fl = _is_fluid(fmu, fmv)
    u = np.zeros((16, 16), dtype)
    v = np.ones((16, 16), dtype)
    s = np.tile(np.arange(16, dtype=dtype)[:, None], (1, 16))
    dst = np.zeros_like(s)
    ops.advect_scalar_field(s, dst, u, v, fl, 1.0, 1.0)
    assert np.allclose(dst[2:-1, 1:-1], s[1:-2, 1:-1], atol=ATOL)


def kat_linear_field_bilinear(ops, face_masks, dtype=np.float32):
    fmu, fmv = face_masks
    fl = _is_fluid(fmu, fmv)
    j, i = np.indices((16, 16))
    s = (3.0 * i + 2.0 * j).astype(dtype)
    u = np.full((16, 16), 0.25, dtype)
    v = np.full((16, 16), 0.5, dtype)
    dst = np.zeros_like(s)
    ops.advect_scalar_field(s, dst, u, v, fl, 1.0, 1.0)
    expected = 3.0 * (i - 0.25) + 2.0 * (j - 0.5)
    assert np.allclose(dst[1:-1, 1:-1], expected[1:-1, 1:-1], atol=ATOL)


# ------------------------------------------------------------ divergence (test_divergence.py)
def _div(ops, u, v, face_masks, dtype):
    d = np.zeros((16, 16), dtype)
    ops.compute_divergence(u.astype(dtype), v.astype(dtype), d, face_masks[0], face_masks[1], 1.0)
    return d


def kat_divergence_constant(ops, face_masks, dtype=np.float32):
    for (a, b) in ((0.0, 0.0), (1.0, 0.0), (0.0, 1.0), (3.5, -2.5)):
        d = _div(ops, np.full((16, 17), a), np.full((17, 16), b), face_masks, dtype)
        assert np.allclose(d[2:-2, 2:-2], 0.0, atol=ATOL)


def kat_divergence_linear(ops, face_masks, dtype=np.float32):
    ju, iu = np.indices((16, 17))
    jv, iv = np.indices((17, 16))
    assert np.allclose(_div(ops, iu * 1.0, jv * 1.0, face_masks, dtype)[2:-2, 2:-2], 2.0, atol=ATOL)
    assert np.allclose(_div(ops, 3.0 * iu, 0.0 * jv, face_masks, dtype)[2:-2, 2:-2], 3.0, atol=ATOL)
    assert np.allclose(_div(ops, 0.0 * iu, 2.0 * jv, face_masks, dtype)[2:-2, 2:-2], 2.0, atol=ATOL)
    assert np.allclose(_div(ops, -1.0 * ju, 1.0 * iv, face_masks, dtype)[2:-2, 2:-2], 0.0, atol=ATOL)


def kat_divergence_quadratic(ops, face_masks, dtype=np.float32):
    ju, iu = np.indices((16, 17))
    jv, iv = np.indices((17, 16))
    d = _div(ops, iu ** 2 * 1.0, jv ** 2 * 1.0, face_masks, dtype)
    j, i = np.indices((16, 16))
    assert np.allclose(d[2:-2, 2:-2], (2 * i + 2 * j + 2)[2:-2, 2:-2], atol=ATOL)


# ------------------------------------------------------------ gradient (test_pressure_gradient.py)
def kat_gradient_constant(ops, face_masks, dtype=np.float32):
    p = np.full((16, 16), 5.0, dtype)
    u = np.zeros((16, 17), dtype)
    v = np.zeros((17, 16), dtype)
    ops.apply_pressure_gradient(u, v, p, face_masks[0], face_masks[1], 1.0, 1.0, 1.0)
    assert np.allclose(u, 0.0, atol=ATOL) and np.allclose(v, 0.0, atol=ATOL)


def kat_gradient_linear(ops, face_masks, dtype=np.float32):
    j, i = np.indices((16, 16))
    p = (3.0 * i - 2.0 * j).astype(dtype)
    u = np.zeros((16, 17), dtype)
    v = np.zeros((17, 16), dtype)
    ops.apply_pressure_gradient(u, v, p, face_masks[0], face_masks[1], 1.0, 1.0, 1.0)
    assert np.allclose(u[1:-1, 2:-2], -3.0, atol=ATOL)
    assert np.allclose(v[2:-2, 1:-1], 2.0, atol=ATOL)


def kat_gradient_quadratic(ops, face_masks, dtype=np.float32):
    j, i = np.indices((16, 16))
    p = (i ** 2 + j ** 2).astype(dtype)
    u = np.zeros((16, 17), dtype)
    v = np.zeros((17, 16), dtype)
    ops.apply_pressure_gradient(u, v, p, face_masks[0], face_masks[1], 1.0, 1.0, 1.0)
    eu = np.zeros((16, 17))
    ev = np.zeros((17, 16))
    for ii in range(2, 15):
        eu[:, ii] = -(2 * ii - 1)
    for jj in range(2, 15):
        ev[jj, :] = -(2 * jj - 1)
    for col in (1, -2):
        assert np.allclose(u[:, col], 0.0, atol=ATOL)
    for row in (1, -2):
        assert np.allclose(v[row, :], 0.0, atol=ATOL)
    assert np.allclose(u[0, :], 0, atol=ATOL) and np.allclose(u[-1, :], 0, atol=ATOL)
    assert np.allclose(v[:, 0], 0, atol=ATOL) and np.allclose(v[:, -1], 0, atol=ATOL)
    assert np.allclose(u[1:-1, 2:-2], eu[1:-1, 2:-2], atol=ATOL)
    assert np.allclose(v[2:-2, 1:-1], ev[2:-2, 1:-1], atol=ATOL)


# ------------------------------------------------------------ solver (test_pressure_solver.py)
def kat_jacobi_reduces_residual(ops, face_masks, dtype=np.float32):
    fmu, fmv = face_masks
    fl = _is_fluid(fmu, fmv)
    div = np.zeros((16, 16), dtype)
    div[8, 8], div[8, 9] = 1.0, -1.0
    alpha = -1.0  # calculateAlpha(1, 1, 1)

    def res(p):
        r = np.zeros_like(p, dtype=np.float64)
        for j in range(1, 15):
            for i in range(1, 15):
                if not fl[j, i]:
                    continue
                c = p[j, i]
                lap = ((p[j, i - 1] if fmu[j, i] else c) + (p[j, i + 1] if fmu[j, i + 1] else c)
                       + (p[j - 1, i] if fmv[j, i] else c) + (p[j + 1, i] if fmv[j + 1, i] else c) - 4 * c)
                r[j, i] = lap + alpha * div[j, i]
        return np.linalg.norm(r)

    p = np.zeros((16, 16), dtype)
    r0 = res(p)
    ops.jacobi_pressure_solver(p, div, fmu, fmv, 1.0, 1.0, 1.0, iterations=50)
    assert r0 > 1e-6 and res(p) < 0.1 * r0


def kat_jacobi_zero_divergence(ops, face_masks, dtype=np.float32):
    p = np.zeros((16, 16), dtype)
    ops.jacobi_pressure_solver(p, np.zeros((16, 16), dtype), face_masks[0], face_masks[1], 1.0, 1.0, 1.0,
                               iterations=50)
    assert np.allclose(p, 0.0, atol=ATOL)


# ------------------------------------------------------------ projection (test_projection.py)
def kat_div_grad_quadratic(ops, face_masks, dtype=np.float32):
    j, i = np.indices((16, 16))
    p = (i ** 2 + j ** 2).astype(dtype)
    u = np.zeros((16, 17), dtype)
    v = np.zeros((17, 16), dtype)
    ops.apply_pressure_gradient(u, v, p, face_masks[0], face_masks[1], 1.0, 1.0, 1.0)
    d = np.zeros((16, 16), dtype)
    ops.compute_divergence(u, v, d, face_masks[0], face_masks[1], 1.0)
    assert np.allclose(d[2:-2, 2:-2], -4.0, atol=ATOL)


def kat_div_grad_random(ops, face_masks, small_random_grid, dtype=np.float32):
    p = small_random_grid.astype(dtype).copy()
    u = np.zeros((16, 17), dtype)
    v = np.zeros((17, 16), dtype)
    ops.apply_pressure_gradient(u, v, p, face_masks[0], face_masks[1], 1.0, 1.0, 1.0)
    d = np.zeros((16, 16), dtype)
    ops.compute_divergence(u, v, d, face_masks[0], face_masks[1], 1.0)
    lap = np.zeros((16, 16))
    lap[1:-1, 1:-1] = (p[1:-1, :-2] + p[1:-1, 2:] + p[:-2, 1:-1] + p[2:, 1:-1] - 4 * p[1:-1, 1:-1])
    assert np.allclose(d[2:-2, 2:-2], -lap[2:-2, 2:-2], atol=ATOL)


# ------------------------------------------------------------ pipeline (test_pipeline_invariants.py)
def kat_zero_pipeline_noop(ops, face_masks, solver, dtype=np.float32):
    fmu, fmv = face_masks
    u = np.zeros((16, 17), dtype)
    v = np.zeros((17, 16), dtype)
    p = np.zeros((16, 16), dtype)
    d = np.zeros((16, 16), dtype)
    ops.compute_divergence(u, v, d, fmu, fmv, 1.0)
    assert np.allclose(d, 0.0)
    solver(p, d, fmu, fmv, 1000.0, 1.0, 1.0)
    assert np.allclose(p, 0.0)
    ops.apply_pressure_gradient(u, v, p, fmu, fmv, 1000.0, 1.0, 1.0)
    assert np.allclose(u, 0.0) and np.allclose(v, 0.0)
    ops.compute_divergence(u, v, d, fmu, fmv, 1.0)
    assert np.allclose(d, 0.0)


ALL_OPERATOR_KATS = [
    kat_zero_velocity_advection, kat_constant_velocity_advection, kat_rightward_shift, kat_upward_shift,
    kat_linear_field_bilinear, kat_divergence_constant, kat_divergence_linear, kat_divergence_quadratic,
    kat_gradient_constant, kat_gradient_linear, kat_gradient_quadratic, kat_jacobi_reduces_residual,
    kat_jacobi_zero_divergence, kat_div_grad_quadratic,
]
