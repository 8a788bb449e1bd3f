"""sg_jacobi_solve_noalloc: the Jacobi solve for callers that cannot allocate device memory.

A game loop or other real-time host must not call cudaMalloc in the middle of a frame
(an allocation can synchronise the device and stall the frame), and some hosts run
under a fixed device-memory budget set at start-up. For them the library offers a
Jacobi entry point whose ping-pong buffer is a fixed array inside the library. These
tests call it through the C ABI and check it against sg_jacobi_solve (which takes a
caller-provided buffer) on two calls in a row; the operators are bit-exact, so the
results must be identical (well inside the 1e-5 / 1e-6 relative bar of the suite).
The inputs are made with torch beforehand; the entry point itself allocates nothing.
This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

from conftest import package

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("CUDA device required", allow_module_level=True)

L = package()._lib


def _problem(H, W, dtype, seed):
    rng = np.random.default_rng(seed)
    solid = np.zeros((H, W), bool)
    solid[0, :] = solid[-1, :] = True
    solid[:, 0] = solid[:, -1] = True
    solid[H // 3:H // 3 + 3, W // 4:W // 4 + 5] = True
    fmu = np.zeros((H, W + 1), np.uint8)
    fmv = np.zeros((H + 1, W), np.uint8)
    fmu[:, 1:-1] = ~(solid[:, :-1] | solid[:, 1:])
    fmv[1:-1, :] = ~(solid[:-1, :] | solid[1:, :])
    div = torch.from_numpy(rng.uniform(-1, 1, (H, W))).to(dtype).cuda()
    p0 = torch.from_numpy(rng.uniform(-1, 1, (H, W))).to(dtype).cuda()
    return p0, div, torch.from_numpy(fmu).cuda(), torch.from_numpy(fmv).cuda()


def _code(dtype):
    return L.SG_F32 if dtype == torch.float32 else L.SG_F64


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_noalloc_matches_allocating_entry_on_two_calls(dtype):
    lib = L.load()
    stream = L.stream_ptr()
    for call, (H, W, iters) in enumerate(((96, 80, 23), (131, 67, 40))):
        p0, div, fmu, fmv = _problem(H, W, dtype, 100 + call)
        expected = p0.clone()
        got = p0.clone()
        scratch = torch.empty((H, W), dtype=dtype, device="cuda")
        for mode, mu, mv in ((L.SG_MASK_PLANES, fmu.data_ptr(), fmv.data_ptr()), (L.SG_MASK_OPEN, None, None)):
            expected.copy_(p0)
            got.copy_(p0)
            rc = lib.sg_jacobi_solve(_code(dtype), H, W, expected.data_ptr(), W, div.data_ptr(), W, mode, mu, W + 1, mv,
                                     W, -0.37, 0.25, iters, scratch.data_ptr(), stream)
            assert rc == L.SG_OK, lib.sg_last_error()
            rc = lib.sg_jacobi_solve_noalloc(_code(dtype), H, W, got.data_ptr(), W, div.data_ptr(), W, mode, mu, W + 1,
                                             mv, W, -0.37, 0.25, iters, stream)
            assert rc == L.SG_OK, lib.sg_last_error()
            torch.cuda.synchronize()
            e, g = expected.double().cpu().numpy(), got.double().cpu().numpy()
            tol = 1e-5 if dtype == torch.float32 else 1e-6
            assert np.max(np.abs(g - e)) <= tol * max(np.max(np.abs(e)), 1e-30)
            assert np.array_equal(g, e), f"call {call}, mode {mode}"


def test_noalloc_rejects_grids_above_its_capacity():
    lib = L.load()
    n = 1024
    p = torch.zeros((n, n), dtype=torch.float64, device="cuda")  # 8 MiB > 4 MiB of float64 scratch
    div = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    rc = lib.sg_jacobi_solve_noalloc(L.SG_F64, n, n, p.data_ptr(), n, div.data_ptr(), n, L.SG_MASK_OPEN, None, 0, None,
                                     0, -1.0, 0.25, 3, L.stream_ptr())
    assert rc == L.SG_ERR_CAPACITY
    assert b"static" in lib.sg_last_error()
    # the largest float32 grid that fits is accepted, and its result equals the allocating entry's
    rng = np.random.default_rng(7)
    q0 = torch.from_numpy(rng.uniform(-1, 1, (n, n)).astype(np.float32)).cuda()
    qdiv = torch.from_numpy(rng.uniform(-1, 1, (n, n)).astype(np.float32)).cuda()
    got, expected = q0.clone(), q0.clone()
    scratch = torch.empty((n, n), dtype=torch.float32, device="cuda")
    rc = lib.sg_jacobi_solve_noalloc(L.SG_F32, n, n, got.data_ptr(), n, qdiv.data_ptr(), n, L.SG_MASK_OPEN, None, 0,
                                     None, 0, -1.0, 0.25, 3, L.stream_ptr())
    assert rc == L.SG_OK, lib.sg_last_error()
    rc = lib.sg_jacobi_solve(L.SG_F32, n, n, expected.data_ptr(), n, qdiv.data_ptr(), n, L.SG_MASK_OPEN, None, 0, None,
                             0, -1.0, 0.25, 3, scratch.data_ptr(), L.stream_ptr())
    assert rc == L.SG_OK, lib.sg_last_error()
    torch.cuda.synchronize()
    assert torch.equal(got, expected)
