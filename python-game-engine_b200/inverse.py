"""Differentiable inverse problem on the GPU: steer a smoke plume onto a target blob.

    python python-game-engine_b200/inverse.py [--n 256] [--steps 64] [--iters 100] [--fd 32]

The control is a per-step FP32 force field (steps x 2 x n x n, N(0, 0.01^2) at start) on the
left / lower faces of every cell; the loss is the squared L2 distance between the final
density and a Gaussian blob (sigma 20 cells at 256^2) centred at a seeded point in the upper
half. Gradients come from the adjoint kernels through checkpointed rollouts (one state kept
every 8 steps). The run
  1. checks the FP64 adjoint gradient against FP64 central differences (eps = 1e-6) on
     `--fd` random control entries of the full problem,
  2. runs `--iters` steps of gradient descent in FP32,
and prints one JSON line with the gradient errors, the loss history and the timings.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import sys
import time

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sg = importlib.import_module("python-game-engine_b200")
A = sg.adjoint


def _final_density(model, force):
    with torch.no_grad():
        d, _, _ = A.rollout(model, *model.zeros_state(), force)
    return d


def fd_check(n, steps, n_entries, eps=(1e-6, 1e-4), seed=11):
    """Central differences of the loss on `n_entries` control entries drawn uniformly and on
    as many drawn from the entries whose adjoint gradient is at least 1 % of the largest,
    for each step size in `eps`. The difference L(f + e) - L(f - e) is summed cell by cell
    as (d+ - d-) (d+ + d- - 2 target), the same number without the cancellation of two
    losses of ~1e3. What remains at e = 1e-6 is the rounding of the FP64 rollouts, which
    the pressure solves amplify by their condition number (~3e4 at 256^2)."""
    model, force, target = A.inverse_problem(n=n, steps=steps, dtype=torch.float64, precision="fp64",
                                             fixed_cycles=30, exact_forces=True, adjoint_advection="gather")
    loss0, g = A.loss_and_grad(model, force, target)
    rng = np.random.default_rng(seed)
    gmax = float(g.abs().max())
    strong = torch.nonzero(g.abs() >= 0.01 * gmax).cpu().numpy()
    picks = {"uniform": [tuple(int(rng.integers(0, s)) for s in force.shape) for _ in range(n_entries)],
             "strong": [tuple(int(x) for x in strong[rng.integers(0, len(strong))]) for _ in range(n_entries)]}
    out = {"entries_per_set": n_entries, "loss": loss0, "grad_max": gmax}
    for e in eps:
        for name, idx in picks.items():
            rel, resolved, worst = [], [], None
            for k in idx:
                fp, fm = force.clone(), force.clone()
                fp[k] += e
                fm[k] -= e
                dp, dm = _final_density(model, fp), _final_density(model, fm)
                fd = float(((dp - dm) * (dp + dm - 2 * target)).sum()) / (2 * e)
                an = float(g[k])
                r = abs(fd - an) / max(abs(fd), abs(an), 1e-30)
                rel.append(r)
                if max(abs(fd), abs(an)) >= 1e-3 * gmax:
                    resolved.append(r)
                if worst is None or r > worst[0]:
                    worst = (r, fd, an)
            out[f"eps={e:g} {name}"] = {
                "max_rel_err": max(rel), "median_rel_err": float(np.median(rel)),
                "worst": {"fd": worst[1], "adjoint": worst[2]}, "entries_above_1e-3_of_max": len(resolved),
                "max_rel_err_above_1e-3_of_max": max(resolved) if resolved else None}
    return out


def fd_floor_check(n=256, steps=64, n_entries=8, eps=1e-6, spread=(0.8, 0.9, 1.0, 1.1, 1.2), eps_wide=1e-4,
                   seed=11, tol=1e-12):
    """Where the central differences' error at eps comes from, on `n_entries` control entries
    drawn from those with |grad| >= 1 % of the largest. Forward in FP64 with every pressure
    solve to `tol` relative residual.

    For each entry the differences are taken at eps times each factor in `spread`. Their
    truncation error changes by < 1e-3 of itself across that range (it goes as eps^2), so
    their scatter is the non-smooth part of the FP64 forward, i.e. its rounding. Reported: the
    error at eps against the adjoint, that scatter (both relative to |grad|), the error of the
    mean over the spread, the error at eps_wide, and the floor set by the final density's own
    FP64 representation alone: sqrt(sum_c (ulp(d_c)^2 / 6) (2 (d_c - t_c))^2) / (2 eps |grad|),
    the standard deviation of the differences if every cell of the two rollouts' densities
    were rounded independently to nearest once and nothing else rounded."""
    model, force, target = A.inverse_problem(n=n, steps=steps, dtype=torch.float64, precision="fp64", tol=tol,
                                             max_cycles=60, exact_forces=True, adjoint_advection="gather")
    loss0, g = A.loss_and_grad(model, force, target)
    d0 = _final_density(model, force)
    spacing = torch.nextafter(d0.abs(), torch.full_like(d0, float("inf"))) - d0.abs()
    ulp_norm = float(torch.sqrt(((spacing * spacing / 6.0) * (2.0 * (d0 - target)) ** 2).sum()))
    rng = np.random.default_rng(seed)
    gmax = float(g.abs().max())
    strong = torch.nonzero(g.abs() >= 0.01 * gmax).cpu().numpy()
    idx = [tuple(int(x) for x in strong[rng.integers(0, len(strong))]) for _ in range(n_entries)]

    def fd(k, e):
        fp, fm = force.clone(), force.clone()
        fp[k] += e
        fm[k] -= e
        dp, dm = _final_density(model, fp), _final_density(model, fm)
        return float(((dp - dm) * (dp + dm - 2 * target)).sum()) / (2 * e)

    rows = []
    for k in idx:
        an = float(g[k])
        fs = [fd(k, eps * m) for m in spread]
        fw = fd(k, eps_wide)
        rel = lambda a: abs(a - an) / max(abs(a), abs(an), 1e-300)  # noqa: E731
        rows.append({"adjoint": an, "err": rel(fs[list(spread).index(1.0)]), "scatter": float(np.std(fs)) / abs(an),
                     "err_of_mean": rel(float(np.mean(fs))), "err_wide": rel(fw),
                     "ulp_floor": ulp_norm / (2 * eps * abs(an))})
    col = lambda key: [r[key] for r in rows]  # noqa: E731
    return {"grid": [n, n], "steps": steps, "forward": f"FP64, every solve to {tol:g} relative residual",
            "entries": n_entries, "selection": "|grad| >= 1 % of the largest", "loss": loss0, "grad_max": gmax,
            "eps": eps, "spread": list(spread),
            "max_rel_err": max(col("err")), "median_rel_err": float(np.median(col("err"))),
            "median_scatter": float(np.median(col("scatter"))), "max_scatter": max(col("scatter")),
            "median_err_over_scatter": float(np.median([r["err"] / r["scatter"] for r in rows])),
            "median_rel_err_of_mean": float(np.median(col("err_of_mean"))),
            "median_density_ulp_floor": float(np.median(col("ulp_floor"))),
            f"eps={eps_wide:g}": {"max_rel_err": max(col("err_wide")),
                                  "median_rel_err": float(np.median(col("err_wide")))},
            "rows": rows}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--steps", type=int, default=64)
    ap.add_argument("--iters", type=int, default=100)
    ap.add_argument("--fd", type=int, default=32)
    ap.add_argument("--step", type=float, default=5.0, help="gradient-descent step in the max norm")
    args = ap.parse_args()
    out = {"problem": f"inverse {args.n}^2 x {args.steps} steps", "checkpoint_every": 8}
    if args.fd:
        t0 = time.perf_counter()
        # the step sizes bracket the rounding floor: below ~1e-5 the error of the differences
        # grows like 1 / eps (rounding of the rollouts), above it like eps^2 (truncation)
        out["fd_check_fp64"] = fd_check(args.n, args.steps, args.fd, eps=(1e-7, 1e-6, 1e-5, 1e-4))
        out["fd_check_fp64"]["seconds"] = time.perf_counter() - t0
    model, force, target = A.inverse_problem(n=args.n, steps=args.steps, dtype=torch.float32, precision="fp32",
                                             tol=1e-6)
    torch.cuda.synchronize()
    times = []

    def log(it, loss):
        torch.cuda.synchronize()
        times.append(time.perf_counter())

    t0 = time.perf_counter()
    f, hist = A.optimize(model, force, target, iters=args.iters, step=args.step, log=log)
    torch.cuda.synchronize()
    total = time.perf_counter() - t0
    out["gradient_descent_fp32"] = {"iters": args.iters, "loss_first": hist[0], "loss_last": hist[-1],
                                    "loss_ratio": hist[-1] / hist[0], "seconds": total,
                                    "ms_per_iteration": 1e3 * total / max(args.iters, 1),
                                    "history": [round(x, 6) for x in hist[:: max(1, len(hist) // 20)]]}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
