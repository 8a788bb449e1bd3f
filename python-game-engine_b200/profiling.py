"""Profiling session for the CUDA smoke step, with the reference's interface.

Mirrors src/cfd/profiling (config.py, timing.py, metrics.py, snapshots.py, session.py,
result.py, summary.py, schema.py): the same configuration classes, validation messages,
vocabularies (TIMINGS, SOURCES, SOURCE_STAGES, SCALAR_METRICS, SCOPES, reducer names),
frame gating ("every"), result dictionaries, report lines and JSON export, so a profiling
block written for the reference configures this one unchanged.

What differs is where the work happens:
  * TimingProfiler times a scope with two CUDA events on the current stream, so it measures
    the device work the scope enqueued (the reference takes host perf_counter_ns around a
    synchronous Numba call). Events are read, with one synchronisation, when durations are
    first asked for; event objects are pooled.
  * MetricsRecorder reduces a captured field on the device, in float64, at capture time
    (sg_field_stats: one launch computing every reducer over every scope) into a row of a
    device results table; process() only closes the frame's rows. The table reaches the host
    when results are read. The reference copies the field into a float64 host buffer at
    capture and reduces it in process(); both reduce the field as it was at capture.
There is no host fallback: without the CUDA library the recorder raises.
"""
from __future__ import annotations

import ctypes
import json
import platform
import subprocess
from collections import defaultdict
from contextlib import contextmanager
from dataclasses import dataclass, field
from datetime import datetime, timezone
from typing import Callable, Union

import numpy as np
import torch

from . import _lib as L

SCHEMA_VERSION = 1

# ---------------------------------------------------------------- vocabularies (profiling/config.py:233-268)
SCALAR_METRICS = ["solver.iterations"]

TIMINGS = [
    "simulation.substep",
    "simulation.emitters",
    "simulation.forces",
    "simulation.advection.velocity",
    "simulation.advection.density",
    "simulation.advection.temperature",
    "simulation.cooling",
    "simulation.dissipation",
    "simulation.divergence",
    "simulation.pressure.solve",
    "simulation.pressure.apply",
    "profiling.capture",
    "profiling.metrics",
]

SOURCES = ["divergence", "pressure", "pressure_residual", "velocity_u", "velocity_v"]

SOURCE_STAGES = {
    "divergence": {"before_projection", "after_projection"},
    "pressure": {"final"},
    "pressure_residual": {"final"},
}

SCOPES = ["all", "interior", "boundary"]


# Host definitions of the reducers (profiling/config.py:270-299). The recorder computes the
# same quantities on the device; these are the names' meaning and the validation vocabulary.
def rms(arr: np.ndarray) -> float:
    return float(np.sqrt(np.mean(np.square(arr))))


def mean(arr: np.ndarray) -> float:
    return float(np.mean(arr))


def mean_abs(arr: np.ndarray) -> float:
    return float(np.mean(np.abs(arr)))


def _max(arr: np.ndarray) -> float:
    return float(np.max(arr))


def max_abs(arr: np.ndarray) -> float:
    return float(np.max(np.abs(arr)))


def std(arr: np.ndarray) -> float:
    return float(np.std(arr))


REDUCERS: dict[str, Callable[[np.ndarray], float]] = {
    "rms": rms,
    "mean": mean,
    "mean_abs": mean_abs,
    "max": _max,
    "max_abs": max_abs,
    "std": std,
}
# column of each reducer / scope in a row of sg_field_stats output (scope-major)
_REDUCER_COL = {name: k for k, name in enumerate(REDUCERS)}
_SCOPE_COL = {name: k for k, name in enumerate(SCOPES)}
_STATS = len(SCOPES) * len(REDUCERS)


# ---------------------------------------------------------------- configuration (profiling/config.py:7-231)
@dataclass
class FieldMetricConfig:
    source: str
    stages: list[str] = field(default_factory=list)
    reducers: list[str] = field(default_factory=list)
    scopes: list[str] = field(default_factory=list)
    every: int = 1

    def validate_config(self) -> None:
        if self.source not in SOURCES:
            raise ValueError(f"Unknown field metric source: {self.source!r}. Must be one of {SOURCES}.")
        allowed_stages = SOURCE_STAGES.get(self.source, set())
        invalid_stages = set(self.stages) - allowed_stages
        if invalid_stages:
            raise ValueError(f"Invalid stages {sorted(invalid_stages)} for source {self.source!r}. "
                             f"Must be a subset of {sorted(allowed_stages)}.")
        invalid_reducers = set(self.reducers) - REDUCERS.keys()
        if invalid_reducers:
            raise ValueError(f"Invalid reducers {sorted(invalid_reducers)}. Must be a subset of "
                             f"{sorted(REDUCERS.keys())}.")
        invalid_scopes = set(self.scopes) - set(SCOPES)
        if invalid_scopes:
            raise ValueError(f"Invalid scopes {sorted(invalid_scopes)}. Must be a subset of {SCOPES}.")
        if self.every <= 0:
            raise ValueError(f"'every' must be a positive integer, got {self.every}.")

    def to_dict(self) -> dict:
        return {"source": self.source, "stages": self.stages, "reducers": self.reducers, "scopes": self.scopes,
                "every": self.every}

    @classmethod
    def from_dict(cls, data: dict) -> "FieldMetricConfig":
        return cls(source=data["source"], stages=data.get("stages", []), reducers=data.get("reducers", []),
                   scopes=data.get("scopes", []), every=data.get("every", 1))


@dataclass
class ScalarMetricConfig:
    name: str
    every: int = 1

    def validate_config(self) -> None:
        if self.name not in SCALAR_METRICS:
            raise ValueError(f"Unknown scalar metric: {self.name!r}. Must be one of {SCALAR_METRICS}.")
        if self.every <= 0:
            raise ValueError(f"'every' must be a positive integer, got {self.every}.")

    def to_dict(self) -> dict:
        return {"name": self.name, "every": self.every}

    @classmethod
    def from_dict(cls, data: dict) -> "ScalarMetricConfig":
        return cls(name=data["name"], every=data.get("every", 1))


@dataclass
class MetricsConfig:
    fields: list[FieldMetricConfig] = field(default_factory=list)
    scalars: list[ScalarMetricConfig] = field(default_factory=list)

    def validate_config(self) -> None:
        for f in self.fields:
            f.validate_config()
        for s in self.scalars:
            s.validate_config()

    def to_dict(self) -> dict:
        return {"fields": [f.to_dict() for f in self.fields], "scalars": [s.to_dict() for s in self.scalars]}

    @classmethod
    def from_dict(cls, data: dict) -> "MetricsConfig":
        return cls(fields=[FieldMetricConfig(**f) for f in data.get("fields", [])],
                   scalars=[ScalarMetricConfig(**s) for s in data.get("scalars", [])])


@dataclass
class ProfileConfig:
    timings: list[str] = field(default_factory=list)
    metrics: MetricsConfig = field(default_factory=MetricsConfig)
    snapshots: list[str] = field(default_factory=list)

    def validate_config(self) -> None:
        invalid_timings = set(self.timings) - set(TIMINGS)
        if invalid_timings:
            raise ValueError(f"Invalid timings {sorted(invalid_timings)}. Must be a subset of {TIMINGS}.")
        if not isinstance(self.metrics, MetricsConfig):
            raise ValueError("metrics must be an instance of MetricsConfig.")
        self.metrics.validate_config()

    @classmethod
    def disabled(cls) -> "ProfileConfig":
        return cls(timings=[], metrics=MetricsConfig(fields=[], scalars=[]), snapshots=[])

    @classmethod
    def full(cls) -> "ProfileConfig":
        field_metrics = [
            FieldMetricConfig(source=source, stages=sorted(stages), reducers=sorted(REDUCERS.keys()),
                              scopes=list(SCOPES), every=1)
            for source, stages in SOURCE_STAGES.items() if source in SOURCES
        ]
        scalar_metrics = [ScalarMetricConfig(name=name, every=1) for name in SCALAR_METRICS]
        return cls(timings=list(TIMINGS), metrics=MetricsConfig(fields=field_metrics, scalars=scalar_metrics),
                   snapshots=[])

    def to_dict(self) -> dict:
        return {"timings": self.timings, "metrics": self.metrics.to_dict(), "snapshots": self.snapshots}

    @classmethod
    def from_dict(cls, data: dict) -> "ProfileConfig":
        return cls(timings=data.get("timings", []), metrics=MetricsConfig.from_dict(data.get("metrics", {})),
                   snapshots=data.get("snapshots", []))

    @classmethod
    def from_json(cls, path: str) -> "ProfileConfig":
        with open(path, "r") as f:
            return cls.from_dict(json.load(f))


# ---------------------------------------------------------------- timing (profiling/timing.py:4-101)
class TimingProfiler:
    """Per-call durations of named scopes, in nanoseconds, measured on the device.

    ``with profiler.scope("simulation.pressure.solve"): ...`` records a CUDA event on the
    current stream on entry and on exit; the duration is the device time between them. An
    enabled scope is also an NVTX range of the same name (the TIMINGS names of
    profiling/config.py:228-242), so a timeline profiler shows the phases under the names
    the reference reports them. Scopes whose name is not enabled cost nothing.
    """

    def __init__(self, enabled_timings: list[str] | None = None):
        self.enabled_timings = set(enabled_timings or [])
        self.enabled = bool(self.enabled_timings)
        self._durations: dict[str, list[float]] = defaultdict(list)
        self._pending: list[tuple[str, torch.cuda.Event, torch.cuda.Event]] = []
        self._pool: list[torch.cuda.Event] = []

    def _event(self) -> torch.cuda.Event:
        return self._pool.pop() if self._pool else torch.cuda.Event(enable_timing=True)

    @contextmanager
    def scope(self, name: str):
        if not self.enabled or name not in self.enabled_timings:
            yield
            return
        start, end = self._event(), self._event()
        torch.cuda.nvtx.range_push(name)
        start.record()
        try:
            yield
        finally:
            end.record()
            torch.cuda.nvtx.range_pop()
            self._pending.append((name, start, end))

    def _resolve(self) -> None:
        if not self._pending:
            return
        for name, start, end in self._pending:
            end.synchronize()
            self._durations[name].append(start.elapsed_time(end) * 1e6)
            self._pool += [start, end]
        self._pending.clear()

    @property
    def durations_ns(self) -> dict[str, list[float]]:
        self._resolve()
        return self._durations

    def get_total_ns(self, name: str) -> float:
        d = self.durations_ns
        return sum(d[name]) if name in d else 0.0

    def get_avg_ns(self, name: str) -> float:
        values = self.durations_ns.get(name, [])
        return sum(values) / len(values) if values else 0.0

    def report_lines(self) -> list[str]:
        lines = []
        for name, values in sorted(self.durations_ns.items(), key=lambda item: sum(item[1]), reverse=True):
            calls = len(values)
            total_ms = sum(values) / 1_000_000
            avg_ms = total_ms / calls if calls else 0.0
            lines.append(f"{name:30s} | {calls:5d} calls | {total_ms:.3f} ms total | {avg_ms:.3f} ms avg")
        return lines

    def to_dict(self) -> dict:
        result = {}
        for name, values in self.durations_ns.items():
            calls = len(values)
            total_ms = sum(values) / 1_000_000
            result[name] = {"total_ms": total_ms, "calls": calls, "avg_ms": (total_ms / calls) if calls else 0.0}
        return result

    def reset(self) -> None:
        # events of scopes still in flight are dropped with their durations
        for _, start, end in self._pending:
            end.synchronize()
            self._pool += [start, end]
        self._pending.clear()
        self._durations.clear()


# ---------------------------------------------------------------- metrics (profiling/metrics.py:32-182)
class MetricsRecorder:
    """Scalar metrics (store) and device-reduced field captures (capture / process).

    Results for a captured (source, stage) accumulate one row per processed frame in a
    device float64 table of shape (rows, keys, 18); ``field_results`` copies it to the host.
    """

    _MIN_ROWS = 64

    def __init__(self, config: MetricsConfig, grid_shape: tuple[int, ...], device=None):
        self.config = config
        self.grid_shape = tuple(grid_shape)
        self.enabled = bool(config.fields or config.scalars)
        self._frame = 0
        self._scalar_configs = {s.name: s for s in config.scalars}
        self._scalars: dict[str, list] = defaultdict(list)
        self._field_configs: dict[tuple[str, str], FieldMetricConfig] = {}
        for field_cfg in config.fields:
            for stage in field_cfg.stages:
                self._field_configs[(field_cfg.source, stage)] = field_cfg
        self._keys = list(self._field_configs)
        self._key_index = {k: n for n, k in enumerate(self._keys)}
        self._rows = [0] * len(self._keys)  # processed frames per key
        self._order: list[tuple[str, str]] = []  # keys in order of first processing
        self._captured_this_frame: set[tuple[str, str]] = set()
        self._device = device
        self._table = None
        self._ws = None

    # --- device state
    def _ensure(self, device, rows_needed: int) -> None:
        if self._ws is None:
            self._device = torch.device(device)
            nbytes = int(L.load().sg_field_stats_workspace_bytes())
            self._ws = torch.zeros(nbytes, dtype=torch.uint8, device=self._device)
            self._table = torch.full((self._MIN_ROWS, max(len(self._keys), 1), _STATS), float("nan"),
                                     dtype=torch.float64, device=self._device)
        if rows_needed > self._table.shape[0]:
            grown = torch.full((max(rows_needed, 2 * self._table.shape[0]),) + tuple(self._table.shape[1:]),
                               float("nan"), dtype=torch.float64, device=self._device)
            grown[:self._table.shape[0]].copy_(self._table)
            self._table = grown

    def tick(self, frame: int) -> None:
        self._frame = frame

    # --- scalar path
    def store(self, name: str, value) -> None:
        if not self.enabled:
            return
        cfg = self._scalar_configs.get(name)
        if cfg is None or self._frame % cfg.every != 0:
            return
        self._scalars[name].append(value.detach().reshape(()) if isinstance(value, torch.Tensor) else float(value))

    @property
    def scalar_results(self) -> dict[str, list[float]]:
        for name, values in self._scalars.items():
            for k, v in enumerate(values):
                if isinstance(v, torch.Tensor):
                    values[k] = float(v.item())
        return self._scalars

    # --- field capture path
    def capture(self, source: str, stage: str, array) -> None:
        if not self.enabled:
            return
        key = (source, stage)
        cfg = self._field_configs.get(key)
        if cfg is None or self._frame % cfg.every != 0:
            return
        if not isinstance(array, torch.Tensor):
            dev = self._device if self._device is not None else torch.device("cuda", torch.cuda.current_device())
            array = torch.as_tensor(np.ascontiguousarray(array), device=dev)
        k = self._key_index[key]
        self._ensure(array.device, self._rows[k] + 1)
        ptr, ld = L.field(array, f"{source}.{stage}")
        out = self._table[self._rows[k], k]
        L.call("sg_field_stats", L.dtype_code(array), array.shape[0], array.shape[1], ptr, ld,
               ctypes.c_void_p(self._ws.data_ptr()), ctypes.c_void_p(out.data_ptr()), L.stream_ptr())
        self._captured_this_frame.add(key)

    # --- deferred processing
    def process(self) -> None:
        """Close this frame's captures: each captured key's row becomes a result."""
        if not self.enabled:
            return
        for key in sorted(self._captured_this_frame):
            k = self._key_index[key]
            if self._rows[k] == 0:
                self._order.append(key)
            self._rows[k] += 1
        self._captured_this_frame.clear()

    @property
    def field_results(self) -> dict[tuple[str, str, str, str], list[float]]:
        out: dict[tuple[str, str, str, str], list[float]] = defaultdict(list)
        if self._table is None or not self._order:
            return out
        host = self._table.cpu().numpy()
        for key in self._order:
            k = self._key_index[key]
            cfg = self._field_configs[key]
            for scope in cfg.scopes:
                for reducer in cfg.reducers:
                    col = _SCOPE_COL[scope] * len(REDUCERS) + _REDUCER_COL[reducer]
                    out[(key[0], key[1], scope, reducer)] = [float(x) for x in host[:self._rows[k], k, col]]
        return out

    # --- reporting / export
    def report_lines(self) -> list[str]:
        lines = []
        for name, values in sorted(self.scalar_results.items()):
            calls = len(values)
            avg = sum(values) / calls if calls else 0.0
            lines.append(f"{name:20s} | {calls:5d} calls | {sum(values):.3f} total | {avg:.3f} avg")
        for (source, stage, scope, reducer), values in sorted(self.field_results.items()):
            avg = sum(values) / len(values) if values else 0.0
            lines.append(f"{source}.{stage}.{scope}.{reducer:10s} | {len(values):5d} samples | {avg:.6f} avg")
        return lines

    def to_dict(self) -> dict:
        result = {"scalars": {}, "fields": {}}
        for name, values in self.scalar_results.items():
            calls = len(values)
            result["scalars"][name] = {"total": sum(values), "calls": calls,
                                       "avg": (sum(values) / calls) if calls else 0.0}
        for (source, stage, scope, reducer), values in self.field_results.items():
            calls = len(values)
            result["fields"][f"{source}.{stage}.{scope}.{reducer}"] = {
                "calls": calls, "avg": (sum(values) / calls) if calls else 0.0,
                "last": values[-1] if values else None}
        return result

    def reset(self) -> None:
        """Clear recorded samples and captures; the device table is kept and overwritten."""
        self._scalars.clear()
        self._rows = [0] * len(self._keys)
        self._order.clear()
        self._captured_this_frame.clear()


# ---------------------------------------------------------------- snapshots (profiling/snapshots.py:4-59)
class SnapshotRecorder:
    """Values and fields captured by getter at given frames (host-side, as the reference)."""

    def __init__(self, enabled: bool = True):
        self.enabled = enabled
        self._snapshots = {}
        self._field_snapshots = {}
        self._values = {}
        self._fields = {}

    def register_snapshot(self, name: str, frame: int, getter):
        self._snapshots[name] = (frame, getter)

    def register_field_snapshot(self, name: str, frame: int, getter):
        self._field_snapshots[name] = (frame, getter)

    def get_value(self, name: str):
        return self._values.get(name, None)

    def get_field(self, name: str):
        return self._fields.get(name, None)

    def tick(self, frame: int):
        if not self.enabled:
            return
        for name, (target_frame, getter) in self._snapshots.items():
            if frame == target_frame:
                value = getter()
                self._values[name] = float(value) if np.isscalar(value) else value
        for name, (target_frame, getter) in self._field_snapshots.items():
            if frame == target_frame:
                value = getter()
                self._fields[name] = float(value) if np.isscalar(value) else value

    def to_dict(self) -> dict:
        return {name: value for name, value in self._values.items()}

    def reset(self):
        self._snapshots.clear()
        self._field_snapshots.clear()
        self._values.clear()
        self._fields.clear()


# ---------------------------------------------------------------- summaries (profiling/summary.py, result.py)
@dataclass
class VariableSummary:
    name: str
    count: int
    total: float
    mean: float
    min: float
    max: float
    std: float
    p95: float
    p99: float

    @classmethod
    def from_values(cls, name: str, values: Union[list[float], list[int]]) -> "VariableSummary":
        if not values:
            return cls(name=name, count=0, total=0.0, mean=0.0, min=0.0, max=0.0, std=0.0, p95=0.0, p99=0.0)
        arr = np.asarray(values, dtype=np.float64)
        return cls(name=name, count=arr.size, total=float(arr.sum()), mean=float(arr.mean()), min=float(arr.min()),
                   max=float(arr.max()), std=float(arr.std()), p95=float(np.percentile(arr, 95)),
                   p99=float(np.percentile(arr, 99)))

    def to_dict(self) -> dict:
        return {"count": self.count, "total": self.total, "mean": self.mean, "min": self.min, "max": self.max,
                "std": self.std, "p95": self.p95, "p99": self.p99}


@dataclass
class ProfilerResult:
    timings: list[VariableSummary] = field(default_factory=list)
    scalars: list[VariableSummary] = field(default_factory=list)
    fields: list[VariableSummary] = field(default_factory=list)
    snapshots: dict = field(default_factory=dict)

    @classmethod
    def from_recorders(cls, timing: TimingProfiler, metrics: MetricsRecorder,
                       snapshots: SnapshotRecorder) -> "ProfilerResult":
        return cls(
            timings=[VariableSummary.from_values(name, [ns / 1_000_000 for ns in durations])
                     for name, durations in timing.durations_ns.items()],
            scalars=[VariableSummary.from_values(name, values) for name, values in metrics.scalar_results.items()],
            fields=[VariableSummary.from_values(f"{source}.{stage}.{scope}.{reducer}", values)
                    for (source, stage, scope, reducer), values in metrics.field_results.items()],
            snapshots=snapshots.to_dict(),
        )

    def to_dict(self) -> dict:
        return {"timings": {s.name: s.to_dict() for s in self.timings},
                "scalars": {s.name: s.to_dict() for s in self.scalars},
                "fields": {s.name: s.to_dict() for s in self.fields},
                "snapshots": self.snapshots}


def get_git_commit():
    try:
        return subprocess.check_output(["git", "rev-parse", "HEAD"], stderr=subprocess.DEVNULL).decode().strip()
    except Exception:
        return None


def build_metadata(extra: dict | None = None) -> dict:
    """profiling/schema.py:20-41, plus the backend and the device name."""
    metadata = {
        "schema_version": SCHEMA_VERSION,
        "timestamp": datetime.now(timezone.utc).isoformat(),
        "python_version": platform.python_version(),
        "platform": platform.platform(),
        "git_commit": get_git_commit(),
        "backend": "cuda",
        "device": torch.cuda.get_device_name() if torch.cuda.is_available() else None,
    }
    if extra:
        metadata.update(extra)
    return metadata


# ---------------------------------------------------------------- session (profiling/session.py:12-134)
class ProfileSession:
    """Timing, metrics and snapshots behind one object, as the reference's ProfileSession."""

    def __init__(self, config: ProfileConfig, grid_shape: tuple[int, ...], device=None):
        self.config = config
        self.timing = TimingProfiler(enabled_timings=config.timings)
        self.metrics = MetricsRecorder(config=config.metrics, grid_shape=grid_shape, device=device)
        self.snapshots = SnapshotRecorder(enabled=bool(config.snapshots))
        self._frame = 0

    @property
    def enabled(self) -> bool:
        return self.timing.enabled or self.metrics.enabled or self.snapshots.enabled

    @classmethod
    def disabled(cls, grid_shape: tuple[int, ...] = (1, 1)) -> "ProfileSession":
        return cls(ProfileConfig.disabled(), grid_shape=grid_shape)

    @classmethod
    def full(cls, grid_shape: tuple[int, ...] = (1, 1)) -> "ProfileSession":
        return cls(ProfileConfig.full(), grid_shape=grid_shape)

    def tick(self):
        self._frame += 1
        self.metrics.tick(self._frame)
        self.snapshots.tick(self._frame)

    def report(self):
        if not self.enabled:
            print("Profiling is disabled; no data recorded.")
            return
        print(self.to_string())

    def to_string(self) -> str:
        lines = ["Timing report:"]
        lines.extend(self.timing.report_lines())
        lines.append("\nVariable report:")
        lines.extend(self.metrics.report_lines())
        return "\n".join(lines)

    def to_dict(self, extra_metadata: dict | None = None) -> dict:
        return {"metadata": build_metadata(extra_metadata), "checkpoints": self.timing.to_dict(),
                "variables": self.metrics.to_dict(), "snapshots": self.snapshots.to_dict()}

    def to_result(self) -> ProfilerResult:
        return ProfilerResult.from_recorders(timing=self.timing, metrics=self.metrics, snapshots=self.snapshots)

    def export_json(self, filepath: str, indent: int = 2, extra_metadata: dict | None = None):
        if not self.enabled:
            print("Profiling is disabled; skipping export.")
            return
        with open(filepath, "w") as f:
            json.dump(self.to_dict(extra_metadata), f, indent=indent)

    @staticmethod
    def load_json(filepath: str) -> dict:
        with open(filepath) as f:
            return json.load(f)

    def reset(self):
        self.timing.reset()
        self.metrics.reset()
        self.snapshots.reset()
