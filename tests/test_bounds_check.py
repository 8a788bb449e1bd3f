"""The bounds-check build (lib/libsmoke_b200_bc.so: -DSG_BOUNDS_CHECK=1, the tiled kernels
check every index before use, skip a failed access and record its source line) runs small and
odd-shaped cases of the register-tile and shared-memory-tile multigrid kernels, the split-layout
SOR, the multi-sweep Jacobi tiles and the batch work lists (tests/bounds_cases.py) in a child
process: no check may fail, and every result must equal the normal build's bit for bit (the
checks change nothing when the indices are right)."""
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

from conftest import ROOT, TESTS

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("CUDA device required", allow_module_level=True)

BC_LIB = os.path.join(ROOT, "python-game-engine_b200", "lib", "libsmoke_b200_bc.so")


def _run(tmp_path, variant):
    out = str(tmp_path / f"{variant}.npz")
    env = dict(os.environ)
    if variant == "bounds":
        env["SG_LIBRARY_VARIANT"] = "bounds"
    else:
        env.pop("SG_LIBRARY_VARIANT", None)
    r = subprocess.run([sys.executable, os.path.join(TESTS, "bounds_cases.py"), out], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return dict(np.load(out))


def test_index_checks_pass_and_change_nothing(tmp_path):
    if not os.path.exists(BC_LIB):
        pytest.fail("the bounds-check library is not built (python-game-engine_b200/build.py builds it)")
    bc = _run(tmp_path, "bounds")
    assert int(bc["bounds_enabled"]) == 1
    assert int(bc["bounds_line"]) == 0, f"index check failed at line {int(bc['bounds_line'])} of unit " \
                                        f"{int(bc['bounds_unit'])}"
    ref = _run(tmp_path, "normal")
    assert int(ref["bounds_enabled"]) == 0
    for k in ref:
        if k.startswith("bounds_"):
            continue
        assert np.array_equal(bc[k], ref[k]), k
