"""Generate the profiling / cfd-bench golden fixtures with the reference's own code.

Run in a container that holds the reference source (it is not needed anywhere else):
    python tests/golden/make_profiling_golden.py path/to/reference/src
(or with REFERENCE_SRC set to that path)

Outputs (consumed by tests/test_profiling.py):
  * profiling_metrics.npz: seeded float32 / float64 fields and, for each, the values the
    reference's MetricsRecorder (src/cfd/profiling/metrics.py) reports after capture +
    process with every reducer over every scope;
  * bench_ids.json: a suite document written here, the benchmark ids and config
    dictionaries the reference's SuiteConfig.expand_suite (src/cfd/benchmarking/config.py)
    produces for it.
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SRC = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE_SRC")
if not REF_SRC:
    sys.exit("usage: python tests/golden/make_profiling_golden.py path/to/reference/src (or set REFERENCE_SRC)")
os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(HERE, "_numba_cache"))
sys.path.insert(0, REF_SRC)

import numpy as np  # noqa: E402

import cfd.solvers  # noqa: E402,F401  (registries first)
import cfd.operators  # noqa: E402,F401
from cfd.benchmarking.config import SuiteConfig  # noqa: E402
from cfd.profiling.config import REDUCERS, SCOPES, FieldMetricConfig, MetricsConfig  # noqa: E402
from cfd.profiling.metrics import MetricsRecorder  # noqa: E402

CASES = [  # (name, shape, dtype, offset, scale)
    ("f32_3x3", (3, 3), np.float32, 0.0, 1.0),
    ("f64_5x3", (5, 3), np.float64, 0.0, 1.0),
    ("f32_17x33", (17, 33), np.float32, 0.5, 2.0),
    ("f64_64x80", (64, 80), np.float64, -3.0, 0.25),
    ("f64_offset_40x40", (40, 40), np.float64, 1.0e6, 1.0),
    ("f32_130x257", (130, 257), np.float32, 0.0, 1.0e-3),
]


def metrics_fixture():
    rng = np.random.default_rng(11)
    out = {}
    for name, shape, dtype, offset, scale in CASES:
        a = (offset + scale * rng.standard_normal(shape)).astype(dtype)
        cfg = MetricsConfig(fields=[FieldMetricConfig(source="pressure", stages=["final"],
                                                      reducers=list(REDUCERS), scopes=list(SCOPES), every=1)])
        rec = MetricsRecorder(cfg, grid_shape=shape)
        rec.tick(1)
        rec.capture("pressure", "final", a)
        rec.process()
        vals = np.array([[rec.field_results[("pressure", "final", s, r)][0] for r in REDUCERS] for s in SCOPES])
        out[f"{name}__field"] = a
        out[f"{name}__values"] = vals
    np.savez_compressed(os.path.join(HERE, "profiling_metrics.npz"), **out)


SUITE = {
    "name": "golden suite",
    "schema_version": "0.1",
    "type": "suite",
    "benchmark": {
        "simulation": {
            "grid": {"size": [[24, 24], [32, 20]], "cell_size": [1.0, 0.5]},
            "pressure_solver": {
                "method": {
                    "jacobi": {"params": [{"iterations": 10}, {"iterations": 40}]},
                    "multigrid": {"params": [{"num_levels": 3, "smoother_backend": "numba"}]},
                },
                "backend": ["numba"],
            },
            "operators": {"advection": ["numba"], "boundaries": ["numba"], "divergence": ["numba"],
                          "forces": ["numba"], "pressure_gradient": ["numba"], "residual": ["numba"]},
        },
        "emitters": [{"position": [10, 6], "radius": 3, "density_value": 1.0, "temperature_value": 0.5,
                      "velocity_value": [0, 1], "approach": "linear", "numba_optimized": True}],
        "run": {"frames": [4, 6], "warmup_frames": [1], "repetitions": [2]},
        "profiling": {"timings": ["simulation.substep"],
                      "metrics": {"fields": [{"source": "pressure", "stages": ["final"], "reducers": ["max"],
                                              "scopes": ["all"], "every": 2}], "scalars": []},
                      "snapshots": []},
    },
}


def ids_fixture():
    expanded = SuiteConfig.from_dict(SUITE).expand_suite()
    doc = {"suite": SUITE, "ids": [b.name for b in expanded], "configs": [b.to_dict() for b in expanded]}
    with open(os.path.join(HERE, "bench_ids.json"), "w") as f:
        json.dump(doc, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    metrics_fixture()
    ids_fixture()
    print("wrote profiling_metrics.npz, bench_ids.json")
