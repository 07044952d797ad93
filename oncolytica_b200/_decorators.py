"""Rule decorators (reference framework/src/oncolytica/cpu/_decorators.py:23-59).

They only tag the method; ``Engine.load_model`` finds rules by the tag and the
translator compiles them to CUDA.
"""
from __future__ import annotations

from typing import Callable, Optional


def tissue_rule(_func: Optional[Callable] = None) -> Callable:
    def deco(func: Callable) -> Callable:
        func._rule_type = "tissue"
        return func

    return deco(_func) if _func is not None else deco


def chemistry_rule(iterations: int = 1) -> Callable:
    if callable(iterations):  # used bare: @ol.chemistry_rule
        func = iterations
        func._rule_type = "chemistry"
        func._iterations = 1
        return func

    def deco(func: Callable) -> Callable:
        func._rule_type = "chemistry"
        func._iterations = int(iterations)
        return func

    return deco


def cell_rule(_func: Optional[Callable] = None) -> Callable:
    def deco(func: Callable) -> Callable:
        func._rule_type = "cell"
        return func

    return deco(_func) if _func is not None else deco


def metric_rule(_func: Optional[Callable] = None) -> Callable:
    def deco(func: Callable) -> Callable:
        func._rule_type = "metric"
        return func

    return deco(_func) if _func is not None else deco
