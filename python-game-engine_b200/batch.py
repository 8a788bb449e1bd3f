"""Many independent smoke scenes of uneven sizes stepped together on one GPU.

``BatchedSmoke`` wraps the sg_batch_* entries of libsmoke_b200: every scene is the default
scene of SmokeSimulation2D (open box, solid ring, one overwriting plume, float32 fields) with
its own size, cell size, time step and buoyancy coefficient; each operator of the step is
one persistent launch over a work list of tiles of all scenes, the multigrid pressure solve
runs to a per-scene relative residual, and the step is one CUDA graph launch. The workspace
is a torch allocation owned here; scene fields are views into it.

``shard_scenes`` splits a scene list across ranks by cell count (scenes are independent, so
a multi-GPU run needs no exchange beyond gathering per-rank metrics).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib as L
from .scenes import Scene

TILE_NAMES = ["32x8", "64x4", "16x16", "128x2"]


def scene_params(sc: Scene, fluid_density: float = 1.0) -> list:
    """The 10 per-scene parameters of sg_batch_create for a single-plume scene (the
    buoyancy coefficient rides in the gravity, density coefficient 1, as in the
    single-scene simulation)."""
    if len(sc.plumes) != 1:
        raise ValueError("batched scenes carry exactly one plume source")
    cx, cy, r, dens, vin, noise = sc.plumes[0]
    if noise != 0.0:
        raise ValueError("batched plume sources carry no noise")
    return [sc.cell_size, sc.dt, fluid_density, sc.gravity, 1.0, cx, cy, r, dens, vin]


class BatchedSmoke:
    def __init__(self, scenes, tol: float = 1e-6, max_cycles: int = 50, seed: int = 0, device=None):
        self.scenes = list(scenes)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        n = len(self.scenes)
        H = (ctypes.c_int * n)(*[s.H for s in self.scenes])
        W = (ctypes.c_int * n)(*[s.W for s in self.scenes])
        params = np.ascontiguousarray(np.asarray([scene_params(s) for s in self.scenes], dtype=np.float64))
        self._params = params
        handle = ctypes.c_void_p()
        L.call("sg_batch_create", ctypes.byref(handle), n, H, W, params.ctypes.data_as(ctypes.c_void_p), float(tol),
               int(max_cycles), int(seed) & (2**64 - 1))
        self.handle = handle
        lib = L.load()
        self.bytes = int(lib.sg_batch_workspace_bytes(handle))
        with torch.cuda.device(self.device):
            self.workspace = torch.empty(self.bytes, dtype=torch.uint8, device=self.device)
            L.call("sg_batch_bind", handle, ctypes.c_void_p(self.workspace.data_ptr()), self.bytes, L.stream_ptr())
        self.config = (0, 2, 0)
        self.cells = int(sum(s.H * s.W for s in self.scenes))

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                L.load().sg_batch_destroy(h)
            except Exception:  # interpreter shutdown: the library may already be gone
                pass
            self.handle = None

    # ------------------------------------------------------------------ configuration
    def configure(self, tile: int = 0, sweeps: int = 2, cycle: str = "V"):
        L.call("sg_batch_configure", self.handle, int(tile), int(sweeps), 1 if cycle == "W" else 0)
        self.config = (int(tile), int(sweeps), 1 if cycle == "W" else 0)

    def autotune(self, steps: int = 2):
        """Time every (tile, sweeps, V/W) candidate for `steps` steps from the current state
        and keep the fastest; the state is left unchanged. Returns the choice."""
        nbytes = int(L.load().sg_batch_snapshot_bytes(self.handle))
        scratch = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        t, s, w = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        ms = ctypes.c_double(0.0)
        L.call("sg_batch_autotune", self.handle, int(steps), ctypes.c_void_p(scratch.data_ptr()), nbytes,
               L.stream_ptr(), ctypes.byref(t), ctypes.byref(s), ctypes.byref(w), ctypes.byref(ms))
        self.config = (t.value, s.value, w.value)
        return {"tile": TILE_NAMES[t.value], "sweeps": s.value, "cycle": "W" if w.value else "V",
                "ms_per_step": ms.value}

    # ------------------------------------------------------------------ stepping
    def step(self, n: int = 1):
        L.call("sg_batch_step", self.handle, int(n), L.stream_ptr())

    def stats(self):
        """Per-scene (cycles of the last solve, its relative residual, cycles since bind)."""
        n = len(self.scenes)
        c = np.zeros(n, dtype=np.int32)
        r = np.zeros(n, dtype=np.float64)
        t = np.zeros(n, dtype=np.int64)
        L.call("sg_batch_stats", self.handle, c.ctypes.data_as(ctypes.c_void_p), r.ctypes.data_as(ctypes.c_void_p),
               t.ctypes.data_as(ctypes.c_void_p), L.stream_ptr())
        return c, r, t

    def loops(self):
        """Cycle-loop iterations (all scenes together) run since bind."""
        n = ctypes.c_longlong(0)
        L.call("sg_batch_loops", self.handle, ctypes.byref(n), L.stream_ptr())
        return n.value

    def graph_nodes(self):
        a, b = ctypes.c_int(0), ctypes.c_int(0)
        L.call("sg_batch_graph_nodes", self.handle, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    # ------------------------------------------------------------------ fields
    def _view(self, off, rows, cols):
        return self.workspace[off:off + 4 * rows * cols].view(torch.float32).view(rows, cols)

    def fields(self, s: int):
        """(density, u, v, pressure) of scene s: views of the current state (valid until the
        next step, which moves the state to the other buffer)."""
        sc = self.scenes[s]
        o = [ctypes.c_int64(0) for _ in range(4)]
        L.call("sg_batch_layout", self.handle, int(s), *[ctypes.byref(x) for x in o])
        H, W = sc.H, sc.W
        return (self._view(o[0].value, H, W), self._view(o[1].value, H, W + 1), self._view(o[2].value, H + 1, W),
                self._view(o[3].value, H, W))


def shard_scenes(scenes, world: int, rank: int):
    """Indices of the scenes rank `rank` of `world` steps: greedy by cell count (largest
    first onto the least loaded rank), deterministic on every rank."""
    order = sorted(range(len(scenes)), key=lambda k: (-scenes[k].H * scenes[k].W, k))
    load = [0] * world
    mine = []
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += scenes[k].H * scenes[k].W
        if r == rank:
            mine.append(k)
    return sorted(mine)
