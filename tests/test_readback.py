"""Host read-back of the density every step while the simulation keeps stepping
(FieldReadback over sg_stage_copy)."""
import numpy as np
import pytest
import torch

from conftest import package

pytestmark = pytest.mark.gpu

sg = package()


@pytest.fixture(autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_readback_slots_hold_each_steps_density(dtype):
    """Every step's density lands in its slot unchanged although the next substeps rewrite
    the field in place; with two slots, the slot of step k holds step k's field until step
    k + 2 is submitted."""
    sc = sg.scenes.Scene("rb_96", 96, 80, 6, -1.0, [[40.0, 10.0, 6.0, 1.0, 1.0, 0.05]], seed=5)
    sim = sg.scenes.make_sim(sc, "jacobi", sg.JacobiParams(iterations=20), dtype=dtype, device="cuda")
    rb = sg.FieldReadback(sim, "density", slots=2)
    expect = []
    for k in range(5):
        sim.substep(sc.dt)
        expect.append(sim.density.cpu().clone())
        slot = rb.submit()
        assert slot == k % 2
        if k >= 1:  # the previous step's slot is not reused before the next submit
            assert torch.equal(rb.result((k - 1) % 2), expect[k - 1])
    rb.wait()
    torch.cuda.synchronize()
    assert torch.equal(rb.result(4 % 2), expect[4])
    assert torch.equal(rb.result(3 % 2), expect[3])
    assert float(expect[4].abs().sum()) > 0.0


def test_stage_copy_rejects_unaligned_rows_and_copies_strided():
    """sg_stage_copy copies rows with byte strides (16-byte units only)."""
    lib = sg._lib.load()
    src = torch.arange(64 * 40, dtype=torch.float32, device="cuda").reshape(64, 40)
    dst = torch.zeros((64, 48), dtype=torch.float32, device="cuda")
    sg._lib.call("sg_stage_copy", 64, 40 * 4, src.data_ptr(), 40 * 4, dst.data_ptr(), 48 * 4, sg._lib.stream_ptr())
    torch.cuda.synchronize()
    assert torch.equal(dst[:, :40], src) and float(dst[:, 40:].abs().sum()) == 0.0
    rc = lib.sg_stage_copy(64, 39 * 4, src.data_ptr(), 40 * 4, dst.data_ptr(), 48 * 4, None)
    assert rc == sg._lib.SG_ERR_ARG
    np.testing.assert_array_equal(dst[:, :40].cpu().numpy(), src.cpu().numpy())
