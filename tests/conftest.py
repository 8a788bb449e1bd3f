"""Shared fixtures. Mirrors the reference's tests/conftest.py fixtures (16x16 grids,
closed-box face masks, unit cell size and density) and registers the ``gpu`` marker."""
import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)
GOLDEN = os.path.join(TESTS, "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


def package():
    """The product package (its directory name is not a Python identifier)."""
    return importlib.import_module("python-game-engine_b200")


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def make_face_masks(height, width, solid_mask):
    face_mask_u = np.zeros((height, width + 1), dtype=bool)
    face_mask_v = np.zeros((height + 1, width), dtype=bool)
    face_mask_u[:, 1:-1] = ~(solid_mask[:, :-1] | solid_mask[:, 1:])
    face_mask_v[1:-1, :] = ~(solid_mask[:-1, :] | solid_mask[1:, :])
    return face_mask_u, face_mask_v


@pytest.fixture
def small_grid_size():
    return (16, 16)


@pytest.fixture
def small_random_grid():
    rng = np.random.default_rng(seed=42)
    return rng.random((16, 16), dtype=np.float32)


@pytest.fixture
def face_masks():
    solid = np.zeros((16, 16), dtype=bool)
    solid[0, :] = solid[-1, :] = True
    solid[:, 0] = solid[:, -1] = True
    return make_face_masks(16, 16, solid)


@pytest.fixture
def cell_size():
    return 1.0


@pytest.fixture
def fluid_density():
    return 1.0
