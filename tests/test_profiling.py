"""Profiling session and cfd-bench on the CUDA backend.

CPU: configuration vocabularies and validation, frame gating, result summaries, suite
expansion and benchmark ids against the reference's own ids (tests/golden/bench_ids.json,
made by tests/golden/make_profiling_golden.py), the command line's validate/list.
GPU: sg_field_stats against the reference recorder's values (tests/golden/
profiling_metrics.npz) and numpy, the recorder and the event timings inside a running
simulation, and a suite run end to end into a results directory.
"""
import importlib
import json
import math
import os

import numpy as np
import pytest
import torch

sg = importlib.import_module("python-game-engine_b200")
prof = importlib.import_module("python-game-engine_b200.profiling")
bm = importlib.import_module("python-game-engine_b200.benchmarking")

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


# ------------------------------------------------------------------ CPU
def test_vocabularies_match_reference_names():
    assert list(prof.REDUCERS) == ["rms", "mean", "mean_abs", "max", "max_abs", "std"]
    assert prof.SCOPES == ["all", "interior", "boundary"]
    assert "simulation.pressure.solve" in prof.TIMINGS and "profiling.metrics" in prof.TIMINGS
    assert set(prof.SOURCE_STAGES["divergence"]) == {"before_projection", "after_projection"}


@pytest.mark.parametrize("bad, msg", [
    ({"timings": ["simulation.nope"]}, "Invalid timings"),
    ({"metrics": {"fields": [{"source": "nope"}]}}, "Unknown field metric source"),
    ({"metrics": {"fields": [{"source": "pressure", "stages": ["initial"]}]}}, "Invalid stages"),
    ({"metrics": {"fields": [{"source": "pressure", "reducers": ["median"]}]}}, "Invalid reducers"),
    ({"metrics": {"fields": [{"source": "pressure", "scopes": ["edge"]}]}}, "Invalid scopes"),
    ({"metrics": {"fields": [{"source": "pressure", "every": 0}]}}, "'every' must be a positive integer"),
    ({"metrics": {"scalars": [{"name": "x"}]}}, "Unknown scalar metric"),
])
def test_profile_config_validation(bad, msg):
    with pytest.raises(ValueError, match=msg):
        prof.ProfileConfig.from_dict(bad).validate_config()


def test_profile_config_round_trip():
    full = prof.ProfileConfig.full()
    full.validate_config()
    again = prof.ProfileConfig.from_dict(json.loads(json.dumps(full.to_dict())))
    assert again.to_dict() == full.to_dict()
    assert not prof.ProfileSession.disabled().enabled


def test_disabled_scopes_and_ungated_captures_touch_no_device():
    t = prof.TimingProfiler(["simulation.substep"])
    with t.scope("simulation.forces"):  # not enabled: no event is created
        pass
    assert t.durations_ns == {}
    cfg = prof.MetricsConfig(fields=[prof.FieldMetricConfig("pressure", ["final"], ["max"], ["all"], every=3)])
    m = prof.MetricsRecorder(cfg, (4, 4))
    cpu = torch.zeros(4, 4)  # a capture that reached the device would reject this CPU tensor
    for frame in (1, 2):
        m.tick(frame)
        m.capture("pressure", "final", cpu)
        m.capture("divergence", "after_projection", cpu)  # not configured
        m.process()
    assert dict(m.field_results) == {}


def test_variable_summary_matches_numpy():
    v = [3.0, 1.0, 4.0, 1.0, 5.0, 9.0, 2.0, 6.0]
    s = prof.VariableSummary.from_values("x", v).to_dict()
    a = np.asarray(v)
    assert s["count"] == 8 and s["total"] == a.sum() and s["std"] == pytest.approx(a.std())
    assert s["p95"] == pytest.approx(np.percentile(a, 95))
    assert prof.VariableSummary.from_values("x", []).to_dict()["count"] == 0


def test_suite_expansion_matches_reference_ids():
    with open(os.path.join(GOLDEN, "bench_ids.json")) as f:
        gold = json.load(f)
    expanded = bm.SuiteConfig.from_dict(gold["suite"]).expand_suite()
    assert [b.name for b in expanded] == gold["ids"]
    assert [b.to_dict() for b in expanded] == gold["configs"]


def test_suite_validation_checks_operator_backends():
    with open(os.path.join(GOLDEN, "bench_ids.json")) as f:
        suite = json.load(f)["suite"]
    with pytest.raises(ValueError, match="backend='numba'"):
        bm.SuiteConfig.from_document(suite).validate()
    retargeted = bm.retarget(suite, "cuda")
    bm.SuiteConfig.from_document(retargeted).validate()
    assert suite["benchmark"]["simulation"]["pressure_solver"]["backend"] == ["numba"]  # retarget copies
    one = bm.SuiteConfig.from_document(retargeted).expand_suite()[0]
    one.validate_config()
    assert one.name.split("-")[2] == "cuda"
    # an operator field whose registry operations are missing for the backend is reported
    with pytest.raises(ValueError, match="not available for backend 'numba'"):
        bm.validate_operator_backend("advection", "numba")


def test_benchmark_document_round_trips_to_suite():
    with open(os.path.join(GOLDEN, "bench_ids.json")) as f:
        cfg = json.load(f)["configs"][0]
    bc = bm.BenchmarkConfig.from_dict(bm.retarget(cfg, "cuda"))
    suite = bm.SuiteConfig.from_benchmark_config(bc)
    again = suite.expand_suite()
    assert len(again) == 1 and again[0].to_dict()["simulation"] == bc.to_dict()["simulation"]


def test_cli_validate_and_list(tmp_path, capsys):
    with open(os.path.join(GOLDEN, "bench_ids.json")) as f:
        suite = json.load(f)["suite"]
    p = tmp_path / "suite.json"
    p.write_text(json.dumps(suite))
    assert bm.main(["validate", str(p)]) == 1
    assert bm.main(["validate", str(p), "--backend", "cuda"]) == 0
    assert bm.main(["list", "timings"]) == 0
    out = capsys.readouterr().out
    assert "Valid suite config: golden suite" in out and "simulation.pressure.solve" in out


# ------------------------------------------------------------------ GPU
def _reducers_numpy(a):
    a = np.asarray(a, dtype=np.float64)
    masks = {"all": np.ones(a.shape, bool)}
    inner = np.zeros(a.shape, bool)
    inner[1:-1, 1:-1] = True
    masks["interior"], masks["boundary"] = inner, ~inner
    out = np.full((3, 6), np.nan)
    for s, name in enumerate(prof.SCOPES):
        x = a[masks[name]]
        if x.size:
            out[s] = [f(x) for f in prof.REDUCERS.values()]
    return out


def assert_stats_close(got, ref, what=""):
    """rtol 1e-12, plus what the conditioning allows: the mean of a field whose values
    cancel is only known to ~1e-13 mean_abs (absolute), and std to 1e-14 |mean| / std
    (relative), since both sides subtract a rounded mean."""
    got, ref = np.asarray(got), np.asarray(ref)
    assert got.shape == ref.shape == (3, 6)
    assert np.array_equal(np.isnan(got), np.isnan(ref)), what
    for s in range(3):
        for r in range(6):
            if np.isnan(ref[s, r]):
                continue
            rtol, atol = 1e-12, 1e-300
            if r == 1:
                atol += 1e-13 * ref[s, 2]
            if r == 5 and ref[s, 5] > 0:
                rtol += 1e-14 * abs(ref[s, 1]) / ref[s, 5]
            assert abs(got[s, r] - ref[s, r]) <= rtol * abs(ref[s, r]) + atol, (what, s, r, got[s, r], ref[s, r])


def _device_stats(t):
    ws = torch.zeros(int(sg._lib.load().sg_field_stats_workspace_bytes()), dtype=torch.uint8, device=t.device)
    out = torch.empty(18, dtype=torch.float64, device=t.device)
    import ctypes
    ptr, ld = sg._lib.field(t)
    sg._lib.call("sg_field_stats", sg._lib.dtype_code(t), t.shape[0], t.shape[1], ptr, ld,
                 ctypes.c_void_p(ws.data_ptr()), ctypes.c_void_p(out.data_ptr()), sg._lib.stream_ptr())
    return out.cpu().numpy().reshape(3, 6)


@pytest.mark.gpu
def test_field_stats_match_reference_recorder():
    g = np.load(os.path.join(GOLDEN, "profiling_metrics.npz"))
    names = sorted({k.split("__")[0] for k in g.files})
    assert len(names) >= 6
    for name in names:
        field = g[f"{name}__field"]
        got = _device_stats(torch.from_numpy(field).cuda())
        assert_stats_close(got, g[f"{name}__values"], name)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("shape", [(1, 1), (2, 7), (3, 3), (300, 1), (1, 500), (613, 1031)])
def test_field_stats_shapes_strides_and_nan(dtype, shape):
    g = torch.Generator().manual_seed(shape[0] * 7919 + shape[1])
    base = torch.randn(shape[0], shape[1] + 5, generator=g, dtype=torch.float64).to(dtype).cuda()
    view = base[:, 2:2 + shape[1]]  # row stride > row length
    got = _device_stats(view)
    ref = _reducers_numpy(view.cpu().numpy())
    assert_stats_close(got, ref, (dtype, shape))  # empty scopes: NaN on both sides
    view[0, 0] = float("nan")
    got = _device_stats(view)
    assert math.isnan(got[0, 3]) and math.isnan(got[0, 4]) and math.isnan(got[2, 1])


def _profiled_sim(config, frames=7):
    simcfg = sg.SimulationConfig(grid=sg.GridConfig(size=(40, 24), cell_size=1.0))
    session = prof.ProfileSession(config, grid_shape=(24, 40))
    sim = sg.SmokeSimulation2D(simcfg, profiler=session)
    sim.add_emitter(sg.Emitter2D((20, 6), 4, density_value=1.0, velocity_value=(0.0, 2.0), approach="gaussian"))
    for _ in range(frames):
        sim.substep(0.016)
    return sim, session


@pytest.mark.gpu
def test_recorder_in_simulation_matches_final_fields():
    sim, session = _profiled_sim(prof.ProfileConfig.full(), frames=7)
    res = session.metrics.field_results
    assert len(res[("pressure", "final", "all", "max")]) == 7
    for source, stage, field in (("pressure", "final", sim.pressure),
                                 ("pressure_residual", "final", sim.pressure_residual),
                                 ("divergence", "after_projection", sim.divergence)):
        ref = _reducers_numpy(field.cpu().numpy())
        got = [[res[(source, stage, scope, red)][-1] for red in prof.REDUCERS] for scope in prof.SCOPES]
        assert_stats_close(got, ref, source)
    d = session.to_dict()
    assert set(d) == {"metadata", "checkpoints", "variables", "snapshots"}
    assert d["metadata"]["backend"] == "cuda"
    assert d["checkpoints"]["simulation.substep"]["calls"] == 7
    t = session.timing.durations_ns
    assert all(x > 0 for x in t["simulation.substep"])
    assert sum(t["simulation.substep"]) >= sum(t["simulation.pressure.solve"])
    r = session.to_result().to_dict()
    assert r["fields"]["pressure.final.all.max"]["count"] == 7
    session.reset()
    assert session.timing.durations_ns == {} and dict(session.metrics.field_results) == {}


@pytest.mark.gpu
def test_recorder_every_gating_in_simulation():
    cfg = prof.ProfileConfig.from_dict({"timings": ["simulation.pressure.solve"], "metrics": {"fields": [
        {"source": "divergence", "stages": ["before_projection"], "reducers": ["rms"], "scopes": ["all"],
         "every": 3}]}})
    _, session = _profiled_sim(cfg, frames=7)
    assert len(session.metrics.field_results[("divergence", "before_projection", "all", "rms")]) == 2  # frames 3, 6
    assert len(session.timing.durations_ns["simulation.pressure.solve"]) == 7


@pytest.mark.gpu
def test_suite_runs_end_to_end(tmp_path):
    with open(os.path.join(GOLDEN, "bench_ids.json")) as f:
        suite = bm.retarget(json.load(f)["suite"], "cuda")
    suite["benchmark"]["simulation"]["grid"]["size"] = [[24, 24]]
    suite["benchmark"]["simulation"]["grid"]["cell_size"] = [1.0]
    suite["benchmark"]["run"]["frames"] = [4]
    cfg = bm.SuiteConfig.from_document(suite)
    cfg.validate()
    result = bm.SuiteRunner(bm.ResultWriter(str(tmp_path))).run(cfg)
    summary = result.to_summary()
    assert summary["total_benchmarks"] == 3 and summary["successful_benchmarks"] == 3, summary
    ex = tmp_path / result.execution_id
    assert (ex / "summary.json").exists() and (ex / "config.json").exists()
    for b in summary["benchmarks"]:
        doc = json.loads((ex / b["result"]).read_text())
        assert doc["status"] == "success" and doc["summary"]["total_runs"] == 2
        raw = json.loads((ex / "raw" / b["benchmark_id"] / "run_0.json").read_text())
        assert raw["checkpoints"]["simulation.substep"]["calls"] == 4
        assert len(raw["variables"]["fields"]) == 1
