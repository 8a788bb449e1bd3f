"""Adjoint kernels of the controlled smoke step: gradients against an FP64 PyTorch-autodiff
restatement of the step, against central finite differences, between the scatter and the
deterministic gather form of the advection transpose, across checkpoint spacings, and one
short gradient-descent run."""
import importlib

import numpy as np
import pytest
import torch

from autodiff_ref import RefStep

sg = importlib.import_module("python-game-engine_b200")
A = sg.adjoint

pytestmark = pytest.mark.gpu


def _model(H, W, mode="scatter", dtype=torch.float64, **kw):
    h = 1.0 / W
    plumes = np.array([[0.45 * W, 0.2 * H, 0.15 * W, 1.0, 1.0, 0.0]])
    base = dict(gravity=-1.0, plumes=plumes, seed=3, dtype=dtype, precision="fp64" if dtype == torch.float64 else
                "fp32", fixed_cycles=40 if dtype == torch.float64 else 0, tol=1e-6, exact_forces=True,
                adjoint_advection=mode)
    base.update(kw)
    return A.ControlledSmoke(H, W, h, 0.5 * h, **base)


def _inputs(model, T, seed):
    g = torch.Generator().manual_seed(seed)
    H, W = model.H, model.W
    dev, dt = model.device, model.dtype
    d0 = (0.5 * torch.rand((H, W), generator=g, dtype=torch.float64)).to(dt).to(dev)
    u0 = (0.3 * torch.randn((H, W + 1), generator=g, dtype=torch.float64)).to(dt).to(dev)
    v0 = (0.3 * torch.randn((H + 1, W), generator=g, dtype=torch.float64)).to(dt).to(dev)
    f = (0.5 * torch.randn((T, 2, H, W), generator=g, dtype=torch.float64)).to(dt).to(dev)
    target = torch.rand((H, W), generator=g, dtype=torch.float64).to(dt).to(dev)
    return d0, u0, v0, f, target


def _loss(d, u, v, target):
    return ((d - target) ** 2).sum() + 0.1 * (u ** 2).sum() + 0.1 * (v ** 2).sum()


def _grads(model, d0, u0, v0, f, target, every):
    leaves = [x.detach().clone().requires_grad_(True) for x in (d0, u0, v0, f)]
    d, u, v = A.rollout(model, *leaves[:3], leaves[3], checkpoint_every=every)
    loss = _loss(d, u, v, target)
    gs = torch.autograd.grad(loss, leaves)
    return float(loss.detach()), [x.detach() for x in gs]


@pytest.mark.parametrize("mode", ["scatter", "gather"])
def test_gradient_matches_fp64_autodiff(mode):
    H, W, T = 20, 24, 5
    model = _model(H, W, mode)
    d0, u0, v0, f, target = _inputs(model, T, 1)
    loss, grads = _grads(model, d0, u0, v0, f, target, 2)
    ref = RefStep(H, W, model.cell_size, model.dt, model.gravity, model.plumes)
    leaves = [x.detach().cpu().clone().requires_grad_(True) for x in (d0, u0, v0, f)]
    d, u, v = leaves[0], leaves[1], leaves[2]
    for t in range(T):
        d, u, v = ref(d, u, v, leaves[3][t, 0], leaves[3][t, 1])
    rloss = _loss(d, u, v, target.cpu())
    rgrads = torch.autograd.grad(rloss, leaves)
    assert loss == pytest.approx(float(rloss), rel=1e-10)
    for name, g, r in zip(("d0", "u0", "v0", "force"), grads, rgrads):
        err = float((g.cpu() - r).abs().max())
        assert err <= 1e-8 * float(r.abs().max()), f"{name}: max abs error {err:.3e} vs max {float(r.abs().max()):.3e}"


def test_gradient_matches_central_differences():
    """32 random control entries, eps = 1e-6, FP64 forward; relative agreement 1e-4 above
    the differences' own rounding floor (a few ulps of the loss over 2 eps)."""
    H = W = 48
    T = 12
    model = _model(H, W, "gather")
    d0, u0, v0, f, target = _inputs(model, T, 2)
    d0.zero_(), u0.zero_(), v0.zero_()
    f *= 0.2

    def loss_of(ff):
        with torch.no_grad():
            d, u, v = A.rollout(model, d0, u0, v0, ff)
            return float(_loss(d, u, v, target))

    loss0, grads = _grads(model, d0, u0, v0, f, target, 4)
    g = grads[3]
    floor = 8 * np.finfo(np.float64).eps * abs(loss0) / (2 * 1e-6)
    rng = np.random.default_rng(5)
    idx = [tuple(int(rng.integers(0, n)) for n in f.shape) for _ in range(32)]
    eps = 1e-6
    gmax = float(g.abs().max())
    for k in idx:
        fp, fm = f.clone(), f.clone()
        fp[k] += eps
        fm[k] -= eps
        fd = (loss_of(fp) - loss_of(fm)) / (2 * eps)
        an = float(g[k])
        assert abs(fd - an) <= 1e-4 * max(abs(fd), abs(an)) + floor, f"{k}: fd {fd:.9e} adjoint {an:.9e}"
    assert floor <= 1e-3 * gmax  # the check resolves gradients down to 0.1 % of the largest


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-11), (torch.float32, 2e-4)])
def test_scatter_and_gather_agree(dtype, tol):
    H, W, T = 40, 36, 6
    out = {}
    for mode in ("scatter", "gather"):
        model = _model(H, W, mode, dtype)
        d0, u0, v0, f, target = _inputs(model, T, 3)
        out[mode] = _grads(model, d0, u0, v0, f, target, 3)[1]
    for a, b in zip(out["scatter"], out["gather"]):
        assert float((a - b).abs().max()) <= tol * float(b.abs().max())


def test_checkpoint_spacing_does_not_change_the_gradient():
    H, W, T = 32, 32, 8
    model = _model(H, W, "gather")
    d0, u0, v0, f, target = _inputs(model, T, 4)
    ref = _grads(model, d0, u0, v0, f, target, T)[1]
    for every in (1, 3):
        got = _grads(model, d0, u0, v0, f, target, every)[1]
        for a, b in zip(got, ref):
            # equal up to the summation order of the velocity-advection scatter's atomics
            assert float((a - b).abs().max()) <= 1e-12 * float(b.abs().max())


def test_gradient_descent_reduces_the_loss():
    """A reachable target (the uncontrolled final density moved two cells sideways): a few
    steps of gradient descent on the control must cut the loss."""
    model, force, _ = A.inverse_problem(n=64, steps=16)
    with torch.no_grad():
        d, _, _ = A.rollout(model, *model.zeros_state(), force)
    target = torch.roll(d, shifts=2, dims=1)
    f, hist = A.optimize(model, force, target, iters=8, step=2.0, checkpoint_every=4)
    assert all(np.isfinite(hist))
    assert hist[-1] < 0.7 * hist[0]


def test_inverse_problem_mid_size_central_differences():
    """The inverse problem's own scene at 96^2 x 16 steps (one source, control ~ N(0, 0.01^2),
    Gaussian target, checkpoints every 8 steps), FP64 forward with every solve exact to
    rounding (30 cycles), 16 entries drawn from those carrying >= 1 % of the largest gradient.
    Central differences at eps = 1e-4 agree with the adjoint to 1e-5 relative. At eps = 1e-6
    the median agreement is 1e-4 and the worst entry's 1e-3: there the differences' own error
    is the rounding of the FP64 rollouts, which grows as 1 / eps (asserted: at least twice the
    error at eps = 1e-5), not an error of the adjoint (which matches FP64 autodiff to 1e-8)."""
    inv = importlib.import_module("python-game-engine_b200.inverse")
    out = inv.fd_check(96, 16, 16, eps=(1e-6, 1e-5, 1e-4), seed=11)
    e6, e5, e4 = (out[f"eps={e:g} strong"] for e in (1e-6, 1e-5, 1e-4))
    assert e4["max_rel_err"] <= 1e-5, e4
    assert e6["median_rel_err"] <= 1e-4 and e6["max_rel_err"] <= 1e-3, e6
    assert e6["max_rel_err"] >= 2 * e5["max_rel_err"], (e6, e5)


def test_inverse_problem_fd_error_is_the_forward_rounding():
    """The error of eps = 1e-6 central differences is the FP64 forward's rounding, not the
    adjoint's: at 128^2 x 32 steps (every solve to 1e-12), the differences taken at eps x
    {0.8, 0.9, 1.0, 1.1, 1.2} scatter by about as much as they miss the adjoint gradient (a
    smooth function's differences change by < 1e-3 of their truncation error across that
    range, so the scatter is rounding), and at eps = 1e-4, where the rounding weighs 100 times
    less, they agree to 1e-4 relative."""
    inv = importlib.import_module("python-game-engine_b200.inverse")
    out = inv.fd_floor_check(128, 32, n_entries=6)
    assert out["eps=0.0001"]["max_rel_err"] <= 1e-4, out
    assert out["median_err_over_scatter"] <= 4.0, out
    assert out["median_scatter"] >= 2 * out["eps=0.0001"]["median_rel_err"], out
