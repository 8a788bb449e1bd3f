"""Batched scenes: every scene of a batch must step like a single-scene simulation of it,
every solve must reach the tolerance, the autotuner must leave the state alone, and the
scene sharding across ranks must cover each scene once (gloo ranks on the CPU)."""
import importlib
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

sg = importlib.import_module("python-game-engine_b200")
B = sg.batch
S = sg.scenes


def _scenes(ks):
    return [S.batch_scene(k) for k in ks]


def _single(sc, tol):
    params = sg.GeometricMultigridParams(tol=tol, max_cycles=50, precision="mixed")
    return S.make_sim(sc, "geometric_multigrid", params, dtype=torch.float32)


@pytest.mark.gpu
def test_each_scene_steps_like_a_single_scene_simulation():
    scs = _scenes(range(6))
    assert len({s.H for s in scs}) >= 3  # uneven sizes
    tol = 1e-6
    b = B.BatchedSmoke(scs, tol=tol)
    sims = [_single(sc, tol) for sc in scs]
    for _ in range(8):
        b.step()
        for sim, sc in zip(sims, scs):
            sim.substep(sc.dt)
    torch.cuda.synchronize()
    cyc, rel, _ = b.stats()
    assert np.all(rel <= tol) and np.all(cyc < 50)
    for k, (sim, sc) in enumerate(zip(sims, scs)):
        d, u, v, p = b.fields(k)
        # the operators are the same code; the solves agree to their tolerance
        assert float((d - sim.density).abs().max()) <= 1e-4, k
        su = max(float(sim.velocity_u.abs().max()), 1e-3)
        assert float((u - sim.velocity_u).abs().max()) <= 1e-4 * su, k
        assert float((v - sim.velocity_v).abs().max()) <= 1e-4 * max(float(sim.velocity_v.abs().max()), 1e-3), k


@pytest.mark.gpu
@pytest.mark.parametrize("shapes", [[(96, 70), (64, 64)], [(63, 77), (96, 96)]])
def test_irregular_sizes_step_like_single_scenes(shapes):
    """Odd level widths take depths off the register tiles (a fine width of 70 leaves depth 1
    at 35 columns; an odd fine width leaves every depth to the tile-list kernels): the
    batch must still step each scene like its single-scene simulation."""
    scs = [S.Scene(f"irregular_{H}x{W}", H, W, 10, -1.0, [[0.5 * W, 0.15 * H, 0.1 * min(H, W), 1.0, 1.0, 0.0]],
                   seed=7 + H) for H, W in shapes]
    tol = 1e-6
    b = B.BatchedSmoke(scs, tol=tol)
    sims = [_single(sc, tol) for sc in scs]
    for _ in range(5):
        b.step()
        for sim, sc in zip(sims, scs):
            sim.substep(sc.dt)
    torch.cuda.synchronize()
    assert np.all(b.stats()[1] <= tol)
    for k, sim in enumerate(sims):
        d, u, v, _ = b.fields(k)
        assert float((d - sim.density).abs().max()) <= 1e-4, k
        assert float((u - sim.velocity_u).abs().max()) <= 1e-4 * max(float(sim.velocity_u.abs().max()), 1e-3), k
        assert float((v - sim.velocity_v).abs().max()) <= 1e-4 * max(float(sim.velocity_v.abs().max()), 1e-3), k


@pytest.mark.gpu
@pytest.mark.parametrize("tile,sweeps,cycle", [(1, 1, "V"), (2, 2, "W"), (3, 2, "V"), (0, 4, "W")])
def test_configurations_agree(tile, sweeps, cycle):
    scs = _scenes(range(10, 18))
    ref = B.BatchedSmoke(scs, tol=1e-7)
    alt = B.BatchedSmoke(scs, tol=1e-7)
    alt.configure(tile, sweeps, cycle)
    ref.step(5)
    alt.step(5)
    torch.cuda.synchronize()
    for k in range(len(scs)):
        for a, r in zip(alt.fields(k)[:3], ref.fields(k)[:3]):
            assert float((a - r).abs().max()) <= 1e-4 * max(float(r.abs().max()), 1e-3)
    assert np.all(alt.stats()[1] <= 1e-7)


@pytest.mark.gpu
def test_autotune_keeps_the_state_and_picks_a_converging_choice():
    scs = _scenes(range(20, 36))
    b = B.BatchedSmoke(scs, tol=1e-6)
    b.step(3)
    torch.cuda.synchronize()
    before = [x.clone() for k in range(len(scs)) for x in b.fields(k)]
    choice = b.autotune(steps=1)
    after = [x.clone() for k in range(len(scs)) for x in b.fields(k)]
    assert all(torch.equal(x, y) for x, y in zip(before, after))
    assert choice["tile"] in B.TILE_NAMES and choice["cycle"] in ("V", "W") and choice["ms_per_step"] > 0
    b.step(2)
    assert np.all(b.stats()[1] <= 1e-6)


def test_sharding_covers_every_scene_once_and_balances_cells():
    scs = S.batch_256(256)
    for world in (1, 2, 3, 8):
        parts = [B.shard_scenes(scs, world, r) for r in range(world)]
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(scs)))
        loads = [sum(scs[k].H * scs[k].W for k in p) for p in parts]
        assert max(loads) - min(loads) <= max(s.H * s.W for s in scs)


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    scs = S.batch_256(64)
    mine = B.shard_scenes(scs, world, rank)
    cells = torch.tensor([sum(scs[k].H * scs[k].W for k in mine)], dtype=torch.int64)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    dist.all_reduce(cells)
    if rank == 0:
        out.put((gathered, int(cells.item())))
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_shards():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, cells = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    scs = S.batch_256(64)
    assert sorted(gathered[0] + gathered[1]) == list(range(64))
    assert cells == sum(s.H * s.W for s in scs)


# ---------------------------------------------------------------- against the CPU oracle
_ORACLE_RUNS = {}
ORACLE_STEPS = 5


def _oracle_batch(sweeps, cycle, scs):
    """The CPU oracle (the reference kernels restated in C, and the same multigrid: red-black
    over-relaxation 1.3, full weighting, bilinear prolongation, exact coarsest <= 8 a side,
    FP32 cycles in FP64 refinement to 1e-6) stepping every scene of `scs`; cached per
    (sweeps, cycle), which is all the autotuner's choices change in the arithmetic."""
    import oracle as O

    key = (sweeps, cycle)
    if key not in _ORACLE_RUNS:
        out = []
        for sc in scs:
            fmu, fmv = O.face_masks_from_solid(np.zeros((sc.H, sc.W), bool))
            fl = O.is_fluid_from_faces(fmu, fmv)
            gmg = O.GMGOracle(fmu, fmv, fl, coarsest=8, omega=1.3, pre=sweeps, post=sweeps, cycle=cycle)
            rels = []

            def solver(p, div, fmu_, fmv_, rho, h, dt, gmg=gmg, fl=fl, rels=rels, **_):
                b = O.alpha_coeff(h, rho, dt) * div.astype(np.float64) * fl
                p64 = np.zeros(p.shape)
                _, hist = gmg.solve(p64, b, tol=1e-6, max_cycles=50, precision="mixed")
                rels.append(hist[-1])
                p[:] = p64.astype(p.dtype)

            sim = O.OracleSim(sc.H, sc.W, sc.cell_size, solver, {}, dtype=np.float32)
            sim.dt, sim.gravity = sc.dt, sc.gravity
            sim.plumes = [O.PlumeSpec(*row, seed=sc.seed) for row in sc.plumes]
            for _ in range(ORACLE_STEPS):
                sim.substep(sc.dt)
            assert max(rels) <= 1e-6
            out.append((sim.density.copy(), sim.velocity_u.copy(), sim.velocity_v.copy(), sim.pressure.copy()))
        _ORACLE_RUNS[key] = out
    return _ORACLE_RUNS[key]


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.gpu
@pytest.mark.parametrize("cycle", ["V", "W"])
@pytest.mark.parametrize("sweeps", [1, 2, 3])
@pytest.mark.parametrize("tile", [0, 1, 2, 3])
def test_batch_matches_the_cpu_oracle_for_every_autotuner_choice(tile, sweeps, cycle):
    """Seven scenes of four sizes (64 .. 256), every (tile, sweeps, V/W) candidate of the
    autotuner, 5 steps, against the oracle stepping each scene on its own.
    Stated tolerance: 1e-5 relative L2 on density, u, v and the pressure (mean removed). The
    operators are bit-exact; the solves run the same cycles and stop at the same 1e-6, and
    differ only by the rounding of their float32 cycles (the GPU contracts multiply-adds,
    the oracle does not), ~1e-7 of the pressure per solve."""
    scs = _scenes(range(7))
    assert len({s.H for s in scs}) >= 4
    b = B.BatchedSmoke(scs, tol=1e-6)
    b.configure(tile, sweeps, cycle)
    b.step(ORACLE_STEPS)
    torch.cuda.synchronize()
    cyc, rel, _ = b.stats()
    assert np.all(rel <= 1e-6) and np.all(cyc < 50)
    ref = _oracle_batch(sweeps, cycle, scs)
    for k, (d0, u0, v0, p0) in enumerate(ref):
        d, u, v, p = (t.double().cpu().numpy() for t in b.fields(k))
        assert np.max(d0) > 0.5, k
        assert _rel(d, d0) <= 1e-5, (k, "density", _rel(d, d0))
        assert _rel(u, u0) <= 1e-5, (k, "u", _rel(u, u0))
        assert _rel(v, v0) <= 1e-5, (k, "v", _rel(v, v0))
        pc, p0c = p - p.mean(), p0 - p0.mean()
        assert _rel(pc, p0c) <= 1e-5, (k, "pressure", _rel(pc, p0c))
