"""The reference's own SmokeSimulation2D driven through the reference-side binding
(tests/reference_adapter.py): PressureSolverConfig(backend=Backend.CUDA) routes the
reference simulator's solve (src/cfd/solvers/dispatch.py:5-12) to the CUDA kernels, and its
substeps must equal the same simulator run on the reference's Numba solver bit for bit
(Jacobi and the reference multigrid: the CUDA kernels restate the Numba kernels' arithmetic).

Needs the reference package: an installed copy under baseline/_ref (the offline install of
the reference next to this repository) or REFERENCE_SRC pointing at its src/ directory; the
test is skipped when neither exists.
"""
import os
import sys
import tempfile

import numpy as np
import pytest
import torch

from conftest import ROOT

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("CUDA device required", allow_module_level=True)

REF = os.environ.get("REFERENCE_SRC") or os.path.join(ROOT, "baseline", "_ref")
if not os.path.isdir(os.path.join(REF, "cfd")):
    pytest.skip("the reference package is not installed next to the repository", allow_module_level=True)
try:
    import numba  # noqa: F401
except ImportError:
    pytest.skip("numba (the reference's compute library) is not installed", allow_module_level=True)

os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(tempfile.gettempdir(), "sg_reference_numba_cache"))
if REF not in sys.path:
    sys.path.insert(0, REF)

import cfd.solvers  # noqa: E402,F401  (registries first: the reference's import order)
import cfd.operators  # noqa: E402,F401
from cfd.common.config import Backend, GridConfig, PressureSolverConfig, SimulationConfig  # noqa: E402
from cfd.common.emitters import Emitter2D  # noqa: E402
from cfd.common.simulation import SmokeSimulation2D  # noqa: E402
from cfd.profiling import ProfileSession  # noqa: E402
from cfd.solvers.params import JacobiParams, MultigridParams  # noqa: E402

import reference_adapter  # noqa: E402

_registered = []


def _register():
    if not _registered:
        reference_adapter.register_cuda_backend()
        _registered.append(True)


def _run(backend, method, params, steps=8):
    H = W = 32
    cfg = SimulationConfig(grid=GridConfig(size=(W, H), cell_size=1.0 / H),
                           pressure_solver=PressureSolverConfig(method=method, backend=backend, params=params))
    sim = SmokeSimulation2D(cfg, profiler=ProfileSession.disabled((H, W)))
    sim.add_emitter(Emitter2D(position=(16, 6), radius=4.0, density_value=3.0, temperature_value=2.0,
                              velocity_value=(0.3, 2.0), approach="linear", numba_optimized=True))
    for _ in range(steps):
        sim.substep(sim.dt)
    return {n: getattr(sim, n).copy() for n in ("density", "velocity_u", "velocity_v", "pressure", "temperature",
                                                "divergence", "pressure_residual")}


@pytest.mark.parametrize("method,params", [
    ("jacobi", JacobiParams(iterations=30)),
    ("multigrid", MultigridParams(smoother_type="jacobi", num_levels=3, v_cycles=2, smoother_iterations=2,
                                  coarsest_iterations=20)),
])
def test_reference_simulator_on_cuda_solver_equals_numba(method, params):
    _register()
    ref = _run(Backend.NUMBA, method, params)
    got = _run(Backend.CUDA, method, params)
    assert np.max(ref["density"]) > 0.1
    for name in ref:
        assert np.array_equal(got[name], ref[name]), name


def test_reference_registry_serves_the_cuda_operators():
    """An operator looked up in the reference's registry under "cuda" computes in place into
    the caller's numpy array what the Numba operator computes."""
    _register()
    from cfd.operators.registry import get_operator

    rng = np.random.default_rng(4)
    H, W = 24, 20
    u = rng.uniform(-1, 1, (H, W + 1)).astype(np.float32)
    v = rng.uniform(-1, 1, (H + 1, W)).astype(np.float32)
    fmu = np.zeros((H, W + 1), bool)
    fmv = np.zeros((H + 1, W), bool)
    fmu[:, 1:-1] = True
    fmv[1:-1, :] = True
    a, b = np.zeros((H, W), np.float32), np.zeros((H, W), np.float32)
    get_operator("compute_divergence", "numba")(u, v, a, fmu, fmv, 1.0 / W)
    get_operator("compute_divergence", "cuda")(u, v, b, fmu, fmv, 1.0 / W)
    assert np.array_equal(a, b) and np.any(a != 0)
