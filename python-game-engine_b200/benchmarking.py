"""cfd-bench on the CUDA backend: benchmark and suite configs, runners, results, writer, CLI.

Mirrors src/cfd/benchmarking (config.py, runner.py, suite_runner.py, result.py, writer.py,
cli.py): the same JSON schema ("benchmark" and "suite" documents, schema version 0.1), the
same validation messages, suite expansion order and benchmark ids, the same result
dictionaries and on-disk layout (<root>/<execution id>/{config.json, summary.json,
results/<id>.json, raw/<id>/run_<k>.json}). The differences:
  * the simulation is this package's SmokeSimulation2D with this package's ProfileSession
    (CUDA-event timings, device-side field reductions);
  * operator backends are checked against the operator registry: every registry operation
    that a config field selects (advection -> advection_scalar / _velocity_u / _velocity_v,
    forces -> apply_forces + cool_temperature, ...) must be registered for the named backend
    (the check the reference leaves as TODO(operator-dispatch), config.py:317-335), so a
    suite naming "cuda" validates and one naming "numba" reports what is missing;
    ``retarget(data, "cuda")`` rewrites a reference document's backends;
  * a run's duration includes a device synchronisation, so it covers the GPU work.

Command line (the reference's ``cfd-bench``):
    python python-game-engine_b200 run <config.json> [--backend cuda] [--root DIR]
    python python-game-engine_b200 validate <config.json> [--backend cuda]
    python python-game-engine_b200 list {solvers,operators,backends,timings,metrics}
"""
from __future__ import annotations

import argparse
import copy
import hashlib
import json
import os
import re
import traceback
from dataclasses import asdict, dataclass, field
from datetime import datetime
from itertools import product
from time import perf_counter_ns
from typing import Any

import torch

from .config import Backend, OperatorBackendConfig, SimulationConfig
from .params import SOLVER_PARAM_TYPES
from .profiling import (REDUCERS, SCALAR_METRICS, SCOPES, SOURCE_STAGES, TIMINGS, ProfileConfig, ProfileSession)
from .registry import OPERATOR_REGISTRY, SOLVER_REGISTRY, get_operator, get_solver
from .simulation import APPROACHES as EMITTER_APPROACHES
from .simulation import Emitter2D, SmokeSimulation2D

SCHEMA_VERSION = "0.1"

# registry operations behind each OperatorBackendConfig field
OPERATOR_FIELDS = {
    "advection": ["advection_scalar", "advection_velocity_u", "advection_velocity_v"],
    "boundaries": ["enforce_boundary_conditions"],
    "divergence": ["compute_divergence"],
    "forces": ["apply_forces", "cool_temperature"],
    "pressure_gradient": ["apply_pressure_gradient"],
    "residual": ["compute_residual"],
}


def validate_emitters(emitters: list[dict]) -> None:
    """benchmarking/config.py:20-47."""
    if not emitters or not isinstance(emitters, list):
        raise ValueError("Emitters must be provided and must be a list of dictionaries.")
    for emitter in emitters:
        if not isinstance(emitter, dict):
            raise ValueError("Each emitter must be a dictionary.")
        if "position" not in emitter or "radius" not in emitter:
            raise ValueError("Each emitter must have 'position' and 'radius' keys.")
        if not isinstance(emitter["position"], (list, tuple)) or len(emitter["position"]) != 2:
            raise ValueError("Emitter 'position' must be a list or tuple of length 2.")
        if not isinstance(emitter["radius"], (int, float)) or emitter["radius"] <= 0:
            raise ValueError("Emitter 'radius' must be a positive number.")
        if "density_value" not in emitter or not isinstance(emitter["density_value"], (int, float)):
            raise ValueError("Emitter 'density_value' must be a number.")
        if "temperature_value" not in emitter or not isinstance(emitter["temperature_value"], (int, float)):
            raise ValueError("Emitter 'temperature_value' must be a number.")
        if "velocity_value" not in emitter or not isinstance(emitter["velocity_value"], (list, tuple)):
            raise ValueError("Emitter 'velocity_value' must be a list or tuple.")
        if (any(not isinstance(v, (int, float)) for v in emitter["velocity_value"])
                or len(emitter["velocity_value"]) != 2):
            raise ValueError("Emitter 'velocity_value' must contain only numbers and be length 2.")
        if "approach" not in emitter or not isinstance(emitter["approach"], str):
            raise ValueError("Emitter 'approach' must be a string.")
        if emitter.get("approach") not in EMITTER_APPROACHES:
            raise ValueError(f"Emitter 'approach' must be one of {list(EMITTER_APPROACHES)}.")
        if "numba_optimized" not in emitter or not isinstance(emitter["numba_optimized"], bool):
            raise ValueError("Emitter 'numba_optimized' must be a boolean.")


def validate_operator_backend(operator_name: str, backend: str) -> None:
    """Every registry operation behind `operator_name` must exist for `backend`."""
    supported = {b.value for b in Backend}
    if backend not in supported:
        raise ValueError(f"Unsupported backend '{backend}' for operator '{operator_name}'. "
                         f"Supported backends are: {sorted(supported)}")
    for op in OPERATOR_FIELDS.get(operator_name, []):
        try:
            get_operator(op, backend)
        except ValueError as e:
            raise ValueError(f"Operator '{operator_name}' is not available for backend '{backend}': {e}") from e


def retarget(data: dict, backend: str = "cuda") -> dict:
    """A copy of a benchmark or suite document with every solver, smoother and operator
    backend set to `backend` (what to run a reference document on this package)."""
    d = copy.deepcopy(data)
    body = d.get("benchmark") if d.get("type") == "suite" else d
    sim = body.get("simulation", {})
    ps = sim.get("pressure_solver", {})
    if "backend" in ps:
        ps["backend"] = [backend] if isinstance(ps["backend"], list) else backend
    # multigrid smoothers name a backend too
    if isinstance(ps.get("method"), dict):
        param_lists = [mc.get("params", []) for mc in ps["method"].values() if isinstance(mc, dict)]
    else:
        param_lists = [[ps.get("params", {})]]
    for params in (p for lst in param_lists for p in lst):
        if isinstance(params, dict) and "smoother_backend" in params:
            params["smoother_backend"] = backend
    ops = sim.get("operators", {})
    for name, b in list(ops.items()):
        ops[name] = [backend] if isinstance(b, list) else backend
    return d


@dataclass
class RunConfig:
    frames: int
    warmup_frames: int
    repetitions: int = 1


@dataclass
class BenchmarkConfig:
    """benchmarking/config.py:57-171."""
    name: str
    simulation: SimulationConfig
    run: RunConfig
    profiling: ProfileConfig = field(default_factory=ProfileConfig)
    emitters: list[dict] = field(default_factory=list)

    @classmethod
    def from_dict(cls, data: dict) -> "BenchmarkConfig":
        return cls(name=data["name"], simulation=SimulationConfig.from_dict(data["simulation"]),
                   run=RunConfig(**data["run"]), profiling=ProfileConfig.from_dict(data.get("profiling") or {}),
                   emitters=data.get("emitters", []))

    @classmethod
    def from_json(cls, path: str) -> "BenchmarkConfig":
        with open(path, "r") as f:
            return cls.from_dict(json.load(f))

    def validate_config(self) -> None:
        if self.run.repetitions <= 0:
            raise ValueError("Repetitions must be a positive integer.")
        try:
            self.simulation.validate_config()
            get_solver(self.simulation.pressure_solver.method, Backend(self.simulation.pressure_solver.backend).value)
            for name, backend in vars(self.simulation.operators).items():
                validate_operator_backend(name, Backend(backend).value)
        except ValueError as e:
            raise ValueError(f"Simulation config validation failed: {e}")
        if self.run.frames <= 0 or self.run.warmup_frames < 0:
            raise ValueError("Run config validation failed: frames and warmup_frames must be positive.")
        try:
            self.profiling.validate_config()
        except ValueError as e:
            raise ValueError(f"Profiling config validation failed: {e}")
        try:
            validate_emitters(self.emitters)
        except ValueError as e:
            raise ValueError(f"Emitters config validation failed: {e}")

    def to_dict(self) -> dict:
        return {"name": self.name, "schema_version": SCHEMA_VERSION, "type": "benchmark",
                "simulation": self.simulation.to_dict(), "emitters": self.emitters,
                "run": {"frames": self.run.frames, "warmup_frames": self.run.warmup_frames,
                        "repetitions": self.run.repetitions},
                "profiling": self.profiling.to_dict()}


def _slugify(value: object) -> str:
    value = str(value).lower()
    value = re.sub(r"[^a-z0-9]+", "-", value)
    return value.strip("-")


def _config_hash(config: BenchmarkConfig) -> str:
    encoded = json.dumps(config.to_dict(), sort_keys=True, separators=(",", ":")).encode()
    return hashlib.sha256(encoded).hexdigest()[:8]


def make_benchmark_id(index: int, config: BenchmarkConfig) -> str:
    """<index>-<method>-<backend>-<W>x<H>-<sha256 of the config, 8 hex> (config.py:174-192)."""
    readable = [config.simulation.pressure_solver.method, Backend(config.simulation.pressure_solver.backend).value,
                f"{config.simulation.grid.size[0]}x{config.simulation.grid.size[1]}"]
    return "-".join([f"{index:03d}", *(_slugify(x) for x in readable), _config_hash(config)])


@dataclass
class SuiteConfig:
    """benchmarking/config.py:207-616: a cartesian product of benchmark settings."""
    name: str
    benchmark_definitions: dict[str, Any]

    def _validate_simulation(self, simulation: dict | None) -> None:
        if not simulation:
            raise ValueError("Simulation configuration must be provided.")
        grid = simulation["grid"]
        if not grid:
            raise ValueError("Grid configuration must be provided.")
        grid_size = grid["size"]
        if not grid_size or any(not isinstance(size, (list, tuple)) or len(size) != 2 for size in grid_size):
            raise ValueError("Grid size must be a list of 2D tuples.")
        for size in grid_size:
            if any(not isinstance(dim, int) or dim <= 0 for dim in size):
                raise ValueError("Grid dimensions must be positive integers.")
        cell_size = grid.get("cell_size")
        if not cell_size or not isinstance(cell_size, list):
            raise ValueError("Grid cell size must be a list of positive numbers.")
        if any(not isinstance(size, (int, float)) or size <= 0 for size in cell_size):
            raise ValueError("Cell sizes must be all positive number.")
        pressure_solver = simulation["pressure_solver"]
        if not pressure_solver:
            raise ValueError("Pressure solver configuration must be provided.")
        methods = pressure_solver["method"]
        backends = pressure_solver["backend"]
        if not methods or not isinstance(methods, dict) or any(not isinstance(m, str) for m in methods.keys()):
            raise ValueError("Pressure solver methods must be a dictionary with string keys.")
        if not backends or not isinstance(backends, list) or any(not isinstance(b, str) for b in backends):
            raise ValueError("Pressure solver backend must be a list of strings.")
        if len(backends) != len(set(backends)):
            raise ValueError("Pressure solver backends must be unique.")
        for method, method_config in methods.items():
            if method not in SOLVER_PARAM_TYPES.keys():
                raise ValueError(f"Unsupported pressure solver method: {method}. Supported methods are: "
                                 f"{list(SOLVER_PARAM_TYPES.keys())}")
            if not isinstance(method_config, dict):
                raise ValueError(f"Pressure solver method configuration for {method} must be a dictionary.")
            for backend in backends:
                if backend not in [b.value for b in Backend]:
                    raise ValueError(f"Unsupported pressure solver backend: {backend}. Supported backends are: "
                                     f"{[b.value for b in Backend]}")
                try:
                    get_solver(method, backend)
                except ValueError as e:
                    raise ValueError(f"Suite pressure solver validation failed: {e}")
            if "params" not in method_config:
                raise ValueError(f"Pressure solver params for method {method} must be provided.")
            param_configs = method_config["params"]
            if not param_configs or not isinstance(param_configs, list):
                raise ValueError(f"Pressure solver params for method {method} must be a list of dictionaries.")
            param_type = SOLVER_PARAM_TYPES[method]
            for params in param_configs:
                if not isinstance(params, dict):
                    raise ValueError(f"Pressure solver params for method {method} must be a dictionary.")
                try:
                    param_type(**params)
                except (TypeError, ValueError) as e:
                    raise ValueError(f"Invalid parameters for pressure solver method {method}: {e}") from e
        operators = simulation["operators"]
        if not operators or not isinstance(operators, dict):
            raise ValueError("Operators configuration must be provided and must be a dictionary.")
        required_operators = set(asdict(OperatorBackendConfig()).keys())
        missing_operators = required_operators - set(operators.keys())
        if missing_operators:
            raise ValueError(f"Missing required operators: {missing_operators}. Required operators are: "
                             f"{required_operators}")
        for operator_name, operator_backends in operators.items():
            if not isinstance(operator_name, str):
                raise ValueError("Operator names must be strings.")
            if not isinstance(operator_backends, list) or not operator_backends:
                raise ValueError(f"Backends for operator '{operator_name}' must be a non-empty list of strings.")
            if any(not isinstance(backend, str) for backend in operator_backends):
                raise ValueError(f"Backends for operator '{operator_name}' must be strings.")
            if len(operator_backends) != len(set(operator_backends)):
                raise ValueError(f"Backends for operator '{operator_name}' must be unique.")
            for backend in operator_backends:
                validate_operator_backend(operator_name, backend)

    def validate(self) -> None:
        if not self.name:
            raise ValueError("Suite name must be provided.")
        if not self.benchmark_definitions:
            raise ValueError("Benchmark definitions must be provided.")
        self._validate_simulation(self.benchmark_definitions.get("simulation"))
        validate_emitters(self.benchmark_definitions.get("emitters", []))
        run = self.benchmark_definitions.get("run")
        if not run or not isinstance(run, dict):
            raise ValueError("Run configuration must be provided and must be a dictionary.")
        frames, warmup_frames, repetitions = run.get("frames"), run.get("warmup_frames"), run.get("repetitions")
        if not isinstance(frames, list) or not frames:
            raise ValueError("Frames must be a non-empty list of positive integers.")
        if any(not isinstance(frame, int) or frame <= 0 for frame in frames):
            raise ValueError("Frames must be a list of positive integers.")
        if not isinstance(warmup_frames, list) or not warmup_frames:
            raise ValueError("Warmup frames must be a non-empty list of positive integers.")
        if any(not isinstance(w, int) or w < 0 for w in warmup_frames):
            raise ValueError("Warmup frames must be a list of positive integers.")
        if not isinstance(repetitions, list) or not repetitions:
            raise ValueError("Repetitions must be a non-empty list of positive integers.")
        if any(not isinstance(rep, int) or rep <= 0 for rep in repetitions):
            raise ValueError("Repetitions must be a list of positive integers.")
        try:
            ProfileConfig.from_dict(self.benchmark_definitions.get("profiling") or {}).validate_config()
        except ValueError as e:
            raise ValueError(f"Suite config validation failed for profiler: {e}")

    @staticmethod
    def _expand_pressure_solvers(pressure_solver: dict) -> list[dict]:
        return [{"method": method, "backend": backend, "params": params}
                for method, method_config in pressure_solver["method"].items()
                for backend in pressure_solver["backend"]
                for params in method_config["params"]]

    @staticmethod
    def _expand_operators(operators: dict) -> list[dict[str, str]]:
        names = list(operators.keys())
        return [dict(zip(names, backends)) for backends in product(*[operators[n] for n in names])]

    @staticmethod
    def _expand_simulation(simulation: dict, solver_configs: list[dict], operator_configs) -> list[dict]:
        grid = simulation["grid"]
        return [{"grid": {"size": size, "cell_size": cell_size}, "pressure_solver": ps, "operators": oc}
                for size, cell_size, ps, oc in product(grid["size"], grid["cell_size"], solver_configs,
                                                        operator_configs)]

    def expand_suite(self) -> list[BenchmarkConfig]:
        d = self.benchmark_definitions
        simulation = d.get("simulation", {})
        run = d.get("run", {})
        sims = self._expand_simulation(simulation, self._expand_pressure_solvers(simulation["pressure_solver"]),
                                       self._expand_operators(simulation["operators"]))
        benchmarks = []
        for sim, frames, warmup, reps in product(sims, run["frames"], run["warmup_frames"], run["repetitions"]):
            cfg = BenchmarkConfig.from_dict({
                "name": "test", "simulation": sim, "emitters": d.get("emitters", []),
                "run": {"frames": frames, "warmup_frames": warmup, "repetitions": reps},
                "profiling": d.get("profiling"),
            })
            cfg.name = make_benchmark_id(len(benchmarks), cfg)
            benchmarks.append(cfg)
        return benchmarks

    def to_dict(self) -> dict:
        return {"name": self.name, "schema_version": SCHEMA_VERSION, "type": "suite",
                "benchmark": self.benchmark_definitions}

    @classmethod
    def from_dict(cls, data: dict) -> "SuiteConfig":
        return cls(name=data["name"], benchmark_definitions=data["benchmark"])

    @classmethod
    def from_document(cls, data: dict) -> "SuiteConfig":
        if data["type"] == "suite":
            return cls.from_dict(data)
        if data["type"] == "benchmark":
            return cls.from_benchmark_config(BenchmarkConfig.from_dict(data))
        raise ValueError(f"Invalid config type: {data['type']}. Expected 'suite' or 'benchmark'.")

    @classmethod
    def from_json(cls, path: str) -> "SuiteConfig":
        with open(path, "r") as f:
            return cls.from_document(json.load(f))

    @classmethod
    def from_benchmark_config(cls, bc: BenchmarkConfig) -> "SuiteConfig":
        ps = bc.simulation.pressure_solver
        simulation = {
            "pressure_solver": {"method": {ps.method: {"params": [asdict(ps.params)]}},
                                "backend": [Backend(ps.backend).value]},
            "operators": {name: [Backend(b).value] for name, b in vars(bc.simulation.operators).items()},
            "grid": {"size": [list(bc.simulation.grid.size)], "cell_size": [bc.simulation.grid.cell_size]},
        }
        return cls(name=bc.name, benchmark_definitions={
            "simulation": simulation, "emitters": bc.emitters or [],
            "run": {"frames": [bc.run.frames], "warmup_frames": [bc.run.warmup_frames],
                    "repetitions": [bc.run.repetitions]},
            "profiling": bc.profiling.to_dict()})


# ---------------------------------------------------------------- results (benchmarking/result.py)
@dataclass
class RunResult:
    run_index: int
    summary_result: dict[str, Any]
    duration_s: float
    status: str = "success"
    error: str | None = None

    def to_dict(self) -> dict:
        return {"run_index": self.run_index, "duration_s": self.duration_s, "status": self.status,
                "error": self.error, "profiler_summary": self.summary_result}


@dataclass
class BenchmarkResult:
    benchmark_id: str
    config: BenchmarkConfig
    runs: list[RunResult]
    status: str = "success"
    error: str | None = None

    def to_summary(self) -> dict:
        durations = [run.duration_s for run in self.runs if run.duration_s is not None]
        n = len(self.runs)
        avg = (sum(durations) / n) if n else -1.0
        total = sum(durations) if n else -1.0
        sd = (sum((d - avg) ** 2 for d in durations) / n) ** 0.5 if n else -1.0
        ok = [run.status == "success" for run in self.runs]
        return {
            "benchmark_id": self.benchmark_id,
            "status": "success" if all(ok) else "partial_failure" if any(ok) else "failure",
            "error": self.error,
            "config": self.config.to_dict(),
            "summary": {"total_runs": n, "successful_runs": sum(ok), "failed_runs": n - sum(ok),
                        "duration_avg_s": avg, "duration_total_s": total, "duration_std_s": sd},
        }

    def to_dict(self) -> dict:
        return {"benchmark_id": self.benchmark_id, "config": self.config.to_dict(), "status": self.status,
                "error": self.error, "runs": [run.to_dict() for run in self.runs]}


@dataclass
class SuiteResult:
    execution_id: str
    name: str
    benchmark_results: list[BenchmarkResult] = field(default_factory=list)

    def to_dict(self) -> dict:
        return {"execution_id": self.execution_id, "name": self.name,
                "benchmark_results": [b.to_dict() for b in self.benchmark_results]}

    def to_summary(self) -> dict:
        benchmarks = []
        for b in self.benchmark_results:
            s = b.to_summary()
            benchmarks.append({"benchmark_id": b.benchmark_id, "status": s["status"],
                               "result": os.path.join("results", f"{b.benchmark_id}.json"),
                               "duration_avg_s": s["summary"]["duration_avg_s"],
                               "duration_total_s": s["summary"]["duration_total_s"],
                               "duration_std_s": s["summary"]["duration_std_s"]})
        return {"execution_id": self.execution_id, "name": self.name,
                "total_benchmarks": len(self.benchmark_results),
                "successful_benchmarks": sum(1 for b in self.benchmark_results if b.status == "success"),
                "failed_benchmarks": sum(1 for b in self.benchmark_results if b.status != "success"),
                "duration_s": sum(r.duration_s for b in self.benchmark_results for r in b.runs
                                  if r.duration_s is not None),
                "benchmarks": benchmarks}


# ---------------------------------------------------------------- writer (benchmarking/writer.py)
class ResultWriter:
    def __init__(self, root: str, write_raw: bool = True):
        self.root = root
        self.write_raw_flag = write_raw
        self.execution_id = None
        self.execution_dir = None

    def set_execution_id(self, execution_id: str) -> None:
        self.execution_id = execution_id

    def initialize_execution(self, suite_name: str) -> None:
        if self.execution_id is None:
            raise ValueError("Execution ID must be set before initializing execution.")
        self.execution_dir = os.path.join(self.root, f"{self.execution_id}")
        os.makedirs(self.root, exist_ok=True)
        os.mkdir(self.execution_dir)
        os.mkdir(os.path.join(self.execution_dir, "results"))
        os.mkdir(os.path.join(self.execution_dir, "raw"))

    def _require_dir(self, what: str) -> None:
        if self.execution_dir is None:
            raise ValueError(f"Execution directory must be set before writing {what}.")

    def write_config(self, config: SuiteConfig) -> None:
        self._require_dir("config")
        with open(os.path.join(self.execution_dir, "config.json"), "w") as f:
            json.dump(config.to_dict(), f, indent=4)

    def write_raw(self, benchmark_id: str, run_index: int, raw_data: dict) -> None:
        if not self.write_raw_flag:
            return
        self._require_dir("raw data")
        path = os.path.join(self.execution_dir, "raw", benchmark_id, f"run_{run_index}.json")
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(raw_data, f, indent=4)

    def write_benchmark(self, result: BenchmarkResult) -> None:
        self._require_dir("benchmark results")
        with open(os.path.join(self.execution_dir, "results", f"{result.benchmark_id}.json"), "w") as f:
            json.dump(result.to_summary(), f, indent=4)

    def write_suite_result(self, result: SuiteResult) -> None:
        self._require_dir("suite results")
        with open(os.path.join(self.execution_dir, "summary.json"), "w") as f:
            json.dump(result.to_summary(), f, indent=4)


# ---------------------------------------------------------------- runners (runner.py, suite_runner.py)
class BenchmarkRunner:
    """Runs each repetition on a fresh simulation: warm-up frames, profiler reset, timed
    frames of substep(0.016), as the reference's runner (runner.py:21-84)."""

    def __init__(self, writer: ResultWriter | None, device=None):
        self.writer = writer
        self.device = device

    def run(self, config: BenchmarkConfig) -> BenchmarkResult:
        runs = []
        for run_index in range(config.run.repetitions):
            result, raw = self._run_once(config, run_index)
            runs.append(result)
            if self.writer is not None:
                self.writer.write_raw(benchmark_id=config.name, run_index=run_index, raw_data=raw)
        result = BenchmarkResult(benchmark_id=config.name, config=config, runs=runs)
        if self.writer is not None:
            self.writer.write_benchmark(result=result)
        return result

    def _run_once(self, config: BenchmarkConfig, run_index: int) -> tuple[RunResult, dict]:
        error = None
        status = "success"
        w, h = config.simulation.grid.size
        profiler = ProfileSession(config=config.profiling, grid_shape=(h, w), device=self.device)
        sim = SmokeSimulation2D(config=config.simulation, profiler=profiler, device=self.device)
        for e in config.emitters:
            sim.add_emitter(Emitter2D.from_dict(e))
        start = perf_counter_ns()
        try:
            for _ in range(config.run.warmup_frames):
                sim.substep(0.016)
            sim.profiler.reset()
            for _ in range(config.run.frames):
                sim.substep(0.016)
            torch.cuda.synchronize(sim.device)
        except Exception:
            status = "error"
            error = str(traceback.format_exc())
        finally:
            duration_s = (perf_counter_ns() - start) / 1_000_000_000
        result = RunResult(run_index=run_index, summary_result=sim.profiler.to_result().to_dict(),
                           duration_s=duration_s, status=status, error=error)
        return result, sim.profiler.to_dict()


class SuiteRunner:
    def __init__(self, writer: ResultWriter, device=None):
        self.writer = writer
        self.device = device

    @staticmethod
    def _make_execution_id(suite: SuiteConfig) -> str:
        ts = datetime.now().strftime("%Y%m%d%H%M%S")
        return f"{suite.name.replace(' ', '_').replace('/', '_').lower()}_{ts}"

    def run(self, suite: SuiteConfig) -> SuiteResult:
        execution_id = self._make_execution_id(suite)
        self.writer.set_execution_id(execution_id)
        self.writer.initialize_execution(suite.name)
        benchmarks = suite.expand_suite()
        self.writer.write_config(suite)
        runner = BenchmarkRunner(self.writer, device=self.device)
        results = [runner.run(b) for b in benchmarks]
        suite_result = SuiteResult(execution_id=execution_id, name=suite.name, benchmark_results=results)
        self.writer.write_suite_result(suite_result)
        return suite_result


# ---------------------------------------------------------------- command line (benchmarking/cli.py)
def build_parser() -> argparse.ArgumentParser:
    parser = argparse.ArgumentParser(prog="cfd-bench", description="CFD Benchmarking CLI (CUDA backend)")
    sub = parser.add_subparsers(dest="command", required=True)
    run_p = sub.add_parser("run", help="Run a single benchmark config")
    run_p.add_argument("config", type=str, help="Path to the benchmark config file")
    run_p.add_argument("--backend", default=None, help="Rewrite every solver/operator backend (e.g. cuda)")
    run_p.add_argument("--root", default=None, help="Result root (default: ./benchmarks/results)")
    val_p = sub.add_parser("validate", help="Validate a benchmark config or suite config")
    val_p.add_argument("config", type=str, help="Path to the benchmark config or suite config file")
    val_p.add_argument("--backend", default=None, help="Rewrite every solver/operator backend (e.g. cuda)")
    list_p = sub.add_parser("list", help="List registered benchmark components")
    list_p.add_argument("resource", type=str, choices=["solvers", "operators", "backends", "timings", "metrics"])
    return parser


def _load_suite(path: str, backend: str | None) -> SuiteConfig:
    with open(path, "r") as f:
        data = json.load(f)
    if backend:
        data = retarget(data, backend)
    return SuiteConfig.from_document(data)


def _report(e: ValueError) -> None:
    tb = traceback.extract_tb(e.__traceback__)
    last = tb[-1] if tb else None
    print(f"{last.filename}:{last.lineno} - {last.name}: {e}" if last else f"Invalid suite config: {e}")


def run_command(args) -> int:
    try:
        config = _load_suite(args.config, args.backend)
        root = args.root or os.path.join(os.getcwd(), "benchmarks", "results")
        result = SuiteRunner(writer=ResultWriter(root=root, write_raw=True)).run(config)
        print(result.to_summary())
    except ValueError as e:
        _report(e)
        return 1
    return 0


def validate_command(args) -> int:
    try:
        config = _load_suite(args.config, args.backend)
        config.validate()
        print(f"Valid suite config: {config.name}")
    except ValueError as e:
        _report(e)
        return 1
    return 0


def list_command(args) -> int:
    resource = args.resource
    if resource == "solvers":
        print("Registered solvers:")
        for solver, backend in SOLVER_REGISTRY:
            print(f"  - {solver} (backend: {backend})")
    elif resource == "operators":
        print("Registered operators:")
        for operator, backend in OPERATOR_REGISTRY:
            print(f"  - {operator} (backend: {backend})")
    elif resource == "backends":
        print("Registered backends:")
        for backend in Backend:
            print(f"  - {backend.value}")
    elif resource == "timings":
        print("Registered timings:")
        for timing in TIMINGS:
            print(f"  - {timing}")
    else:
        print("Registered scalar metrics:")
        for metric in SCALAR_METRICS:
            print(f"  - {metric}")
        print("\nRegistered field sources:")
        for source, stages in SOURCE_STAGES.items():
            print(f"  - {source} (stages: {', '.join(stages)})")
        print("Registered reducers:")
        for reducer in REDUCERS:
            print(f"  - {reducer}")
        print("Registered scopes:")
        for scope in SCOPES:
            print(f"  - {scope}")
    return 0


def main(argv=None) -> int:
    args = build_parser().parse_args(argv)
    try:
        if args.command == "run":
            return run_command(args)
        if args.command == "validate":
            return validate_command(args)
        return list_command(args)
    except ValueError as e:
        print(f"Error: {e}")
        return 1
    except KeyboardInterrupt:
        print("Execution interrupted by user.")
        return 1
