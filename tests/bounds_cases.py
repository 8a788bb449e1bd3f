"""Small and odd-shaped runs of the tiled kernels, for the bounds-check build.

    python tests/bounds_cases.py OUT.npz     (SG_LIBRARY_VARIANT=bounds selects that build)

Runs: one multigrid cycle in FP64, FP32 and mixed precision on 3 x 65, 9 x 33, 63 x 77,
130 x 67 and 1100 x 1300 open boxes and on a 40 x 40 box whose obstacle leaves one fluid
cell open; the split-layout SOR (both kernel variants) and the multi-sweep Jacobi tiles on
the small shapes; a batch of odd-sized scenes for two steps. Writes every result and the
bounds-check record (first failed source line and unit, or 0 / -1) to OUT.npz."""
import importlib
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sg = importlib.import_module("python-game-engine_b200")
L = sg._lib

SHAPES = [(3, 65), (9, 33), (63, 77), (130, 67)]


def cases():
    out = {}
    rng = np.random.default_rng(0)
    for H, W in SHAPES + [(1100, 1300)]:
        div = rng.standard_normal((H, W))
        div -= div.mean()
        for prec in ("fp64", "fp32", "mixed"):
            p = torch.zeros((H, W), dtype=torch.float32 if prec == "fp32" else torch.float64, device="cuda")
            d = torch.from_numpy(div.astype(np.float32 if prec == "fp32" else np.float64)).cuda()
            s = sg.GeometricMultigridSolver()
            s(p, d, sg.OPEN_BOX, sg.OPEN_BOX, 1.0, 1.0 / W, 0.5 / W, precision=prec, fixed_cycles=1)
            out[f"gmg_{prec}_{H}x{W}"] = p.double().cpu().numpy()
    # one fluid cell: the obstacle covers every cell but (20, 20)
    H = W = 40
    solid = np.ones((H, W), bool)
    solid[20, 20] = False
    fmu, fmv, fl = sg.operators.build_masks(torch.from_numpy(solid).cuda())
    p = torch.zeros((H, W), dtype=torch.float64, device="cuda")
    s = sg.GeometricMultigridSolver()
    s(p, torch.from_numpy(rng.standard_normal((H, W))).cuda(), fmu, fmv, 1.0, 1.0 / W, 0.5 / W, precision="fp64",
      fixed_cycles=1)
    out["gmg_one_fluid_cell"] = p.cpu().numpy()
    for H, W in SHAPES:
        div = rng.uniform(-1, 1, (H, W))
        for variant in (0, 1):
            p = torch.zeros((H, W), dtype=torch.float64, device="cuda")
            sg.SORToleranceSolver()(p, torch.from_numpy(div).cuda(), sg.OPEN_BOX, sg.OPEN_BOX, 1.0, 1.0 / W, 0.5 / W,
                                    tol=1e-30, max_iterations=13, check_every=13, variant=variant)
            out[f"sor_v{variant}_{H}x{W}"] = p.cpu().numpy()
        p = torch.from_numpy(rng.uniform(-1, 1, (H, W))).cuda()
        sg.solvers.jacobi_pressure_solver(p, torch.from_numpy(div).cuda(), sg.OPEN_BOX, sg.OPEN_BOX, 1.0, 1.0 / W,
                                          0.5 / W, iterations=11)
        out[f"jacobi_{H}x{W}"] = p.cpu().numpy()
    scs = [sg.scenes.Scene(f"odd_{H}x{W}", H, W, 2, -1.0, [[0.5 * W, 0.2 * H, 0.15 * min(H, W), 1.0, 1.0, 0.0]],
                           seed=H) for H, W in ((63, 77), (96, 70), (65, 33))]
    b = sg.batch.BatchedSmoke(scs, tol=1e-6)
    b.step(2)
    torch.cuda.synchronize()
    for k in range(len(scs)):
        d, u, v, p = b.fields(k)
        out[f"batch_{k}_density"] = d.cpu().numpy()
        out[f"batch_{k}_pressure"] = p.cpu().numpy()
    torch.cuda.synchronize()
    line, unit = L.bounds_check()
    out["bounds_line"] = np.array(line)
    out["bounds_unit"] = np.array(unit)
    out["bounds_enabled"] = np.array(int(L.load().sg_bounds_check_enabled()))
    return out


if __name__ == "__main__":
    np.savez(sys.argv[1], **cases())
