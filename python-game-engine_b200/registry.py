"""Operator and pressure-solver registries keyed by (name, backend).

Same interface and error behaviour as the reference's plugin points
(src/cfd/operators/registry.py:8-34, src/cfd/solvers/registry.py:6-33): a duplicate
key or an unknown key raises ValueError, the latter listing what is available.
This package registers its CUDA implementations under backend "cuda"
(Backend.CUDA, src/cfd/common/config.py:11).
"""
from __future__ import annotations

from collections.abc import Callable
from typing import Any

OperatorFn = Callable[..., Any]

OPERATOR_REGISTRY: dict[tuple[str, str], OperatorFn] = {}
SOLVER_REGISTRY: dict[tuple[str, str], Any] = {}


def register_operator(operation: str, backend: str, fn: OperatorFn) -> None:
    key = (operation, backend)
    if key in OPERATOR_REGISTRY:
        raise ValueError(f"Operator already registered: operation={operation!r}, backend={backend!r}")
    OPERATOR_REGISTRY[key] = fn


def get_operator(operation: str, backend: str) -> OperatorFn:
    try:
        return OPERATOR_REGISTRY[(operation, backend)]
    except KeyError:
        available = [f"{op}/{b}" for op, b in OPERATOR_REGISTRY]
        raise ValueError(
            f"Unknown operator operation={operation!r}, backend={backend!r}. Available: {available}"
        ) from None


def register_solver(method: str, backend: str, fn) -> None:
    key = (method, backend)
    if key in SOLVER_REGISTRY:
        raise ValueError(f"Pressure solver already registered: method={method!r}, backend={backend!r}")
    SOLVER_REGISTRY[key] = fn


def get_solver(method: str, backend: str):
    try:
        return SOLVER_REGISTRY[(method, backend)]
    except KeyError:
        available = [f"{m}/{b}" for m, b in SOLVER_REGISTRY]
        raise ValueError(
            f"Unknown pressure solver method={method!r}, backend={backend!r}. Available: {available}"
        ) from None
