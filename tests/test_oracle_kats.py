"""The reference's analytic known-answer tests, run on the CPU oracle (float32 and float64)."""
import numpy as np
import pytest

import kats
import oracle as O


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("kat", kats.ALL_OPERATOR_KATS, ids=lambda f: f.__name__)
def test_oracle_kat(kat, dtype, face_masks):
    kat(O, face_masks, dtype=dtype)


def test_oracle_div_grad_random(face_masks, small_random_grid):
    kats.kat_div_grad_random(O, face_masks, small_random_grid)


@pytest.mark.parametrize("solver", [O.jacobi_pressure_solver, O.rb_sor_pressure_solver,
                                    O.gauss_seidel_pressure_solver])
def test_oracle_zero_pipeline(face_masks, solver):
    kats.kat_zero_pipeline_noop(O, face_masks, lambda *a: solver(*a, iterations=10))
