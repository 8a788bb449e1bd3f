"""Host-side checks that need no GPU: the C ABI library, argument validation,
multigrid planning, registries, params and config (reference: src/cfd/solvers/
registry.py, operators/registry.py, solvers/params.py, common/config.py)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, package

sg = package()
L = sg._lib


def _declared():
    with open(os.path.join(ROOT, "include", "smoke_b200.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(sg_\w+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = L.load()
    names = _declared()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(L.SIGNATURES), set(names) ^ set(L.SIGNATURES)
    assert lib.sg_version().startswith(b"smoke_b200")
    assert isinstance(lib.sg_launch_count(), int)


def test_abi_rejects_bad_arguments_without_a_gpu():
    lib = L.load()
    null = None
    # empty grid
    rc = lib.sg_compute_divergence(L.SG_F32, 0, 4, null, 5, null, 4, null, 4, L.SG_MASK_OPEN, null, 0, null, 0, 1.0,
                                   null)
    assert rc == L.SG_ERR_ARG and b"grid" in lib.sg_last_error()
    # null field pointers
    rc = lib.sg_advect_scalar(L.SG_F32, 4, 4, null, 4, null, 4, null, 4, 5, 5, null, 5, 4, 4, L.SG_MASK_OPEN, null, 0,
                              0.1, 1.0, 1.0, null)
    assert rc == L.SG_ERR_ARG
    # mask planes required in planes mode
    fake = ctypes.c_void_p(16)
    rc = lib.sg_compute_divergence(L.SG_F32, 4, 4, fake, 5, fake, 4, fake, 4, L.SG_MASK_PLANES, null, 0, null, 0, 1.0,
                                   null)
    assert rc == L.SG_ERR_ARG
    # row stride below the row length
    rc = lib.sg_cool_temperature(L.SG_F32, 4, 4, fake, 3, 0.0, 0.5, 0.1, null)
    assert rc == L.SG_ERR_ARG
    # unsupported dtype code
    rc = lib.sg_cool_temperature(7, 4, 4, fake, 4, 0.0, 0.5, 0.1, null)
    assert rc == L.SG_ERR_DTYPE
    # bad cell size
    rc = lib.sg_compute_divergence(L.SG_F64, 4, 4, fake, 5, fake, 4, fake, 4, L.SG_MASK_OPEN, null, 0, null, 0, 0.0,
                                   null)
    assert rc == L.SG_ERR_ARG
    # split-layout SOR: workspace must be aligned and large enough, dtype known
    n = lib.sg_rbsor_split_workspace_bytes(L.SG_F32, 64, 64)
    assert n > 6 * 64 * 32 * 4 and lib.sg_rbsor_split_workspace_bytes(9, 64, 64) == -1
    rc = lib.sg_rbsor_split_pack(L.SG_F32, 64, 64, fake, 64, 0, ctypes.c_void_p(256 + 16), n, null)
    assert rc == L.SG_ERR_ARG and b"aligned" in lib.sg_last_error()
    rc = lib.sg_rbsor_split_sweeps(L.SG_F32, 64, 64, ctypes.c_void_p(256), n - 1, L.SG_MASK_OPEN, null, 0, null, 0,
                                   1.0, 0.25, 1.9, 3, 1, null)
    assert rc == L.SG_ERR_ARG and b"workspace" in lib.sg_last_error()
    rc = lib.sg_rbsor_split_sweeps(L.SG_F64, 64, 64, ctypes.c_void_p(256), 1 << 30, L.SG_MASK_OPEN, null, 0, null, 0,
                                   1.0, 0.25, 1.9, 3, 2, null)
    assert rc == L.SG_ERR_ARG and b"variant" in lib.sg_last_error()
    rc = lib.sg_rbsor_tol_solve(7, 64, 64, fake, 64, fake, 64, L.SG_MASK_OPEN, null, 0, null, 0, 1.0, 0.25, 1.9,
                                1e-6, 10, 5, 1, ctypes.c_void_p(256), 1 << 30, null, null, null)
    assert rc == L.SG_ERR_DTYPE
    rc = lib.sg_rbsor_mixed_solve(64, 64, fake, 64, fake, 64, L.SG_MASK_OPEN, null, 0, null, 0, 1.0, 0.25, 1.9, 1e-6,
                                  10, 5, -1, ctypes.c_void_p(256), 16, null, null, null, null)
    assert rc == L.SG_ERR_ARG and b"workspace" in lib.sg_last_error()
    # the Python layer turns codes into exceptions
    with pytest.raises(ValueError):
        L.check(L.SG_ERR_ARG, "x")
    with pytest.raises(L.NotConverged):
        L.check(L.SG_ERR_NOT_CONVERGED, "x")
    with pytest.raises(L.SmokeCudaError):
        L.check(L.SG_ERR_NONFINITE, "x")


def _plan(H, W, mode=L.SG_MASK_OPEN, masks=None, **kw):
    lib = L.load()
    h = ctypes.c_void_p()
    args = dict(coarsest=8, omega=1.4, pre=2, post=2, cycle=0, precision=L.SG_GMG_MIXED)
    args.update(kw)
    ptrs = [None, None, None] if masks is None else [m.ctypes.data_as(ctypes.c_void_p) for m in masks]
    rc = lib.sg_gmg_plan_create(ctypes.byref(h), H, W, mode, *ptrs, args["coarsest"], args["omega"], args["pre"],
                                args["post"], args["cycle"], args["precision"])
    return rc, h


@pytest.mark.parametrize("H,W,levels", [(2048, 2048, 9), (512, 512, 7), (128, 128, 5), (96, 96, 5), (37, 50, 4),
                                        (8, 8, 1), (2048, 1024, 9)])
def test_gmg_plan_hierarchy(H, W, levels):
    lib = L.load()
    rc, h = _plan(H, W)
    assert rc == L.SG_OK
    try:
        assert lib.sg_gmg_num_levels(h) == levels
        hh, ww = ctypes.c_int(), ctypes.c_int()
        assert lib.sg_gmg_level_shape(h, levels - 1, ctypes.byref(hh), ctypes.byref(ww)) == L.SG_OK
        assert max(hh.value, ww.value) <= 8
        assert lib.sg_gmg_workspace_bytes(h) > 0
    finally:
        lib.sg_gmg_plan_destroy(h)


def test_gmg_plan_with_obstacle_planes():
    import oracle as O

    H, W = 64, 48
    solid = O.box_solid(H, W)
    solid[20:30, 10:20] = True
    fmu, fmv = O.face_masks_from_solid(solid)
    fl = O.is_fluid_from_faces(fmu, fmv)
    masks = [np.ascontiguousarray(x.astype(np.uint8)) for x in (fl, fmu, fmv)]
    rc, h = _plan(H, W, L.SG_MASK_PLANES, masks)
    assert rc == L.SG_OK
    L.load().sg_gmg_plan_destroy(h)


@pytest.mark.parametrize("H,W,levels,last,coarsest", [(2048, 2048, 7, (32, 32), 32), (1100, 1300, 7, (18, 21), 32),
                                                      (20, 30, 1, (20, 30), 32), (64, 64, 2, (32, 32), 32),
                                                      (2048, 2048, 4, (256, 256), 256),
                                                      (1024, 768, 3, (256, 192), 256), (300, 260, 3, (75, 65), 80)])
def test_gmg_plan_cosine_coarsest(H, W, levels, last, coarsest):
    """coarsest 17..256 on an open box: the hierarchy stops at the first level <= coarsest a
    side (solved by the cosine transform: one block up to 64 a side, tiled products above)."""
    lib = L.load()
    rc, h = _plan(H, W, coarsest=coarsest)
    assert rc == L.SG_OK
    try:
        assert lib.sg_gmg_num_levels(h) == levels
        hh, ww = ctypes.c_int(), ctypes.c_int()
        assert lib.sg_gmg_level_shape(h, levels - 1, ctypes.byref(hh), ctypes.byref(ww)) == L.SG_OK
        assert (hh.value, ww.value) == last
    finally:
        lib.sg_gmg_plan_destroy(h)


def test_gmg_cosine_coarsest_needs_open_box():
    """A coarsest level above 16 a side that is not an open box is refused at plan creation."""
    import oracle as O

    H, W = 96, 80
    solid = O.box_solid(H, W)
    solid[:, W // 2 - 8:W // 2 + 8] = True  # a wall that survives coarsening
    fmu, fmv = O.face_masks_from_solid(solid)
    fl = O.is_fluid_from_faces(fmu, fmv)
    masks = [np.ascontiguousarray(x.astype(np.uint8)) for x in (fl, fmu, fmv)]
    rc, h = _plan(H, W, L.SG_MASK_PLANES, masks, coarsest=32)
    assert rc == L.SG_ERR_ARG and not h.value
    assert "open box" in L.load().sg_last_error().decode()


@pytest.mark.parametrize("kw", [dict(omega=2.5), dict(coarsest=0), dict(coarsest=257), dict(pre=0, post=0),
                                dict(cycle=3), dict(precision=9)])
def test_gmg_plan_rejects_bad_parameters(kw):
    rc, h = _plan(64, 64, **kw)
    assert rc == L.SG_ERR_ARG and not h.value


def test_registry_semantics():
    key = ("__test_op__", "cuda")
    sg.register_operator(*key, lambda: 1)
    with pytest.raises(ValueError, match="already registered"):
        sg.register_operator(*key, lambda: 2)
    assert sg.get_operator(*key)() == 1
    del sg.OPERATOR_REGISTRY[key]
    with pytest.raises(ValueError, match="Available"):
        sg.get_operator("__missing__", "cuda")
    with pytest.raises(ValueError, match="Unknown pressure solver"):
        sg.get_solver("jacobi", "numba")
    names = {k[0] for k in sg.OPERATOR_REGISTRY}
    assert names >= {"advection_scalar", "advection_velocity_u", "advection_velocity_v", "enforce_boundary_conditions",
                     "compute_divergence", "apply_forces", "cool_temperature", "apply_pressure_gradient",
                     "compute_residual"}
    assert {k[0] for k in sg.SOLVER_REGISTRY} >= {"jacobi", "gauss_seidel", "rb_sor_gauss_seidel", "multigrid"}


def test_params_match_reference_defaults():
    assert sg.JacobiParams().iterations == 40
    assert sg.GaussSeidelParams().iterations == 40
    assert sg.SORParams().iterations == 40 and sg.SORParams().omega == 0.0
    m = sg.MultigridParams()
    assert (m.smoother_type, m.num_levels, m.v_cycles, m.smoother_iterations, m.coarsest_iterations,
            m.rebuild_masks) == ("jacobi", 4, 2, 2, 30, False)
    assert sg.JacobiParams(7).string() == "JacobiParams_iters_7"


def test_config_round_trip_and_validation(tmp_path):
    cfg = sg.SimulationConfig(grid=sg.GridConfig(size=(64, 32), cell_size=0.5),
                              pressure_solver=sg.PressureSolverConfig(method="geometric_multigrid",
                                                                      params=sg.GeometricMultigridParams(tol=1e-8)))
    cfg.validate_config()
    path = tmp_path / "c.json"
    cfg.to_json(str(path))
    back = sg.SimulationConfig.from_json(str(path))
    assert back.grid.size == (64, 32) and back.pressure_solver.params.tol == 1e-8
    back.validate_config()
    bad = sg.SimulationConfig(grid=sg.GridConfig(size=(64, 0), cell_size=0.5))
    with pytest.raises(ValueError):
        bad.validate_config()
    # a reference-shaped JSON (backend "numba") still loads
    ref_json = {"grid": {"size": [16, 16], "cell_size": 1.0},
                "pressure_solver": {"method": "jacobi", "backend": "numba", "params": {"iterations": 5}}}
    c = sg.SimulationConfig.from_dict(ref_json)
    assert c.pressure_solver.params.iterations == 5


def test_scenes_are_seeded_and_sized():
    a = sg.scenes.mixed_2048()
    b = sg.scenes.mixed_2048()
    assert a.plumes == b.plumes and len(a.plumes) == 4
    assert all(16.0 <= p[2] <= 64.0 and 0.5 <= p[4] <= 1.5 for p in a.plumes)
    batch = sg.scenes.batch_256(256)
    assert {s.H for s in batch} <= set(sg.scenes.BATCH_SIZES)
    assert all(0.5 <= -s.gravity <= 2.0 for s in batch)
    assert sg.scenes.plume_128().dt == pytest.approx(0.5 / 128)


def test_product_path_does_not_import_the_oracle():
    pkg = os.path.join(ROOT, "python-game-engine_b200")
    for fn in os.listdir(pkg):
        if fn.endswith(".py"):
            with open(os.path.join(pkg, fn)) as f:
                src = f.read()
            assert not re.search(r"^\s*(import|from)\s+oracle\b", src, re.M), fn


def _batch_create(scenes, tol=1e-6):
    from importlib import import_module

    B = import_module("python-game-engine_b200.batch")
    n = len(scenes)
    H = (ctypes.c_int * n)(*[s.H for s in scenes])
    W = (ctypes.c_int * n)(*[s.W for s in scenes])
    params = np.ascontiguousarray(np.asarray([B.scene_params(s) for s in scenes], dtype=np.float64))
    h = ctypes.c_void_p()
    rc = L.load().sg_batch_create(ctypes.byref(h), n, H, W, params.ctypes.data_as(ctypes.c_void_p), tol, 50, 0)
    return rc, h


def test_batch_plan_layout_on_the_host():
    """A batch's pools, offsets and workspace are laid out on the host (no GPU): fields scene
    by scene, the velocity state in one fixed buffer, and every tile shape known."""
    lib = L.load()
    scenes = sg.scenes.batch_256(16)
    rc, h = _batch_create(scenes)
    assert rc == L.SG_OK
    try:
        cells = sum(s.H * s.W for s in scenes)
        nbytes = lib.sg_batch_workspace_bytes(h)
        # at least: two density buffers, two u and v buffers, p, p64, rhs (x2), r64, div, res
        assert nbytes >= 4 * cells * 14 and nbytes < 64 * cells * 20
        offs = [[ctypes.c_int64() for _ in range(4)] for _ in scenes]
        for k, o in enumerate(offs):
            assert lib.sg_batch_layout(h, k, *[ctypes.byref(x) for x in o]) == L.SG_OK
        for k in range(1, len(scenes)):
            a, b = scenes[k - 1], scenes[k]
            assert offs[k][0].value - offs[k - 1][0].value == 4 * a.H * a.W  # density
            assert offs[k][1].value - offs[k - 1][1].value == 4 * a.H * (a.W + 1)  # u faces
            assert offs[k][2].value - offs[k - 1][2].value == 4 * (a.H + 1) * a.W  # v faces
            assert offs[k][3].value - offs[k - 1][3].value == 4 * a.H * a.W  # pressure
        assert all(x.value % 4 == 0 and 0 <= x.value < nbytes for o in offs for x in o)
        assert lib.sg_batch_layout(h, len(scenes), None, None, None, None) == L.SG_ERR_ARG
    finally:
        lib.sg_batch_destroy(h)
    tx, ty = ctypes.c_int(), ctypes.c_int()
    shapes = []
    for t in range(4):
        assert lib.sg_batch_tile_shape(t, ctypes.byref(tx), ctypes.byref(ty)) == L.SG_OK
        shapes.append(f"{tx.value}x{ty.value}")
    assert shapes == sg.batch.TILE_NAMES
    assert lib.sg_batch_tile_shape(4, ctypes.byref(tx), ctypes.byref(ty)) == L.SG_ERR_ARG


def test_batch_create_rejects_bad_scenes():
    sc = sg.scenes.batch_scene(0)
    tiny = sg.scenes.Scene("tiny", 1, 64, 10, -1.0, [[32.0, 0.5, 0.4, 1.0, 1.0, 0.0]])
    rc, h = _batch_create([sc, tiny])
    assert rc == L.SG_ERR_ARG and not h.value and b"grid" in L.load().sg_last_error()
    rc, h = _batch_create([sc], tol=0.0)
    assert rc == L.SG_ERR_ARG and not h.value


@pytest.mark.parametrize("H,W,coarsest,precision,kind", [
    (64, 64, 8, L.SG_GMG_MIXED, 0), (2048, 2048, 32, L.SG_GMG_MIXED, 1), (2048, 2048, 128, L.SG_GMG_MIXED, 4),
    (2048, 2048, 128, L.SG_GMG_FP64, 4), (2048, 2048, 128, L.SG_GMG_FP32, 4), (2048, 2048, 256, L.SG_GMG_MIXED, 3),
    (300, 260, 80, L.SG_GMG_FP64, 2), (300, 260, 80, L.SG_GMG_MIXED, 2)])
def test_gmg_coarse_solve_kind_is_decided_on_the_host(H, W, coarsest, precision, kind):
    """Which exact coarsest solve a plan runs is fixed at plan creation: the dense pseudo-inverse
    (<= 16 a side), the one-block cosine transform (<= 64), the streaming transform on 4-CTA
    clusters when each CTA's share of its operands fits shared memory (128^2 in every precision),
    the single-CTA streaming transform when the level's rows are whole 16-byte units (256^2),
    and the four tiled products otherwise (a 75 x 65 level: rows of 65 values)."""
    lib = L.load()
    rc, h = _plan(H, W, coarsest=coarsest, precision=precision)
    assert rc == L.SG_OK
    try:
        assert lib.sg_gmg_coarse_solve_kind(h) == kind
    finally:
        lib.sg_gmg_plan_destroy(h)
    assert lib.sg_gmg_coarse_solve_kind(None) == -1


def test_new_entry_points_reject_bad_arguments_without_a_gpu():
    """The read-back staging copy, the float32-arithmetic forces / projection tail and the
    multigrid timing hook validate their arguments before any launch."""
    lib = L.load()
    null = None
    fake = ctypes.c_void_p(256)
    # staging copy: 16-byte units only, strides at least the row length
    rc = lib.sg_stage_copy(4, 40, fake, 48, fake, 48, null)
    assert rc == L.SG_ERR_ARG and b"16 bytes" in lib.sg_last_error()
    rc = lib.sg_stage_copy(4, 64, fake, 48, fake, 64, null)
    assert rc == L.SG_ERR_ARG
    assert lib.sg_stage_copy(0, 64, fake, 64, fake, 64, null) == L.SG_OK  # nothing to copy
    # float32-arithmetic forces: grid, pointers, strides
    rc = lib.sg_apply_forces_f32(0, 4, fake, 4, fake, 4, null, 0, 0.1, -9.8, 0.0, 1.0, 0.0, null)
    assert rc == L.SG_ERR_ARG and b"grid" in lib.sg_last_error()
    rc = lib.sg_apply_forces_f32(4, 4, fake, 3, fake, 4, null, 0, 0.1, -9.8, 0.0, 1.0, 0.0, null)
    assert rc == L.SG_ERR_ARG
    # float32-arithmetic projection tail: out of place only, known masks
    a = [fake, 5, fake, 4, ctypes.c_void_p(512), 5, ctypes.c_void_p(768), 4, fake, 4]
    rc = lib.sg_project_metrics_f32(4, 4, fake, 5, fake, 4, fake, 5, fake, 4, fake, 4, L.SG_MASK_OPEN, null, 0, null,
                                    0, null, 0, 0, null, 0, 1.0, 0.25, 0.1, -1.0, 0.25, fake, 4, fake, 4, null)
    assert rc == L.SG_ERR_ARG and b"out of place" in lib.sg_last_error()
    rc = lib.sg_project_metrics_f32(4, 4, *a, 9, null, 0, null, 0, null, 0, 0, null, 0, 1.0, 0.25, 0.1, -1.0, 0.25,
                                    fake, 4, fake, 4, null)
    assert rc == L.SG_ERR_ARG
    # timing hook: needs a plan, and events for every pair
    assert lib.sg_gmg_set_post_events(None, None, 0) == L.SG_ERR_ARG
    rc, h = _plan(256, 256)
    assert rc == L.SG_OK
    try:
        assert lib.sg_gmg_set_post_events(h, None, 2) == L.SG_ERR_ARG
        two = (ctypes.c_void_p * 2)(None, None)
        assert lib.sg_gmg_set_post_events(h, two, 1) == L.SG_ERR_ARG
        assert lib.sg_gmg_set_post_events(h, None, 0) == L.SG_OK
    finally:
        lib.sg_gmg_plan_destroy(h)
