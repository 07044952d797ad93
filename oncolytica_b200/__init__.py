"""oncolytica_b200 — the Oncolytica per-step simulation path on NVIDIA B200.

Import it the way the reference is imported::

    import oncolytica_b200 as ol

    class MyCell(ol.Cell):
        pos: ol.vec3
        volume: ol.f32 = 1.0

    class Sim(ol.Simulation[MyTissue, MyChem, MyCell, MyMetrics, MyParams]):
        @ol.cell_rule
        def grow(self, cell: MyCell):
            cell.volume += 0.1

    engine = ol.Engine(backend="cuda")

The public names mirror the reference package's ``oncolytica/__init__.py``.
"""
from __future__ import annotations

from oncolytica_b200._types import (  # noqa: F401
    BaseData,
    Cell,
    Chemistry,
    Metrics,
    Params,
    Simulation,
    Tissue,
    bool,
    f32,
    i32,
    ivec3,
    random,
    random_dir,
    u32,
    vec3,
)
from oncolytica_b200 import _math as math  # noqa: F401
from oncolytica_b200._containers import AgentList, Grid  # noqa: F401
from oncolytica_b200._decorators import cell_rule, chemistry_rule, metric_rule, tissue_rule  # noqa: F401
from oncolytica_b200._errors import CompilationError  # noqa: F401
from oncolytica_b200.engine import Engine  # noqa: F401

__all__ = [
    "f32", "i32", "u32", "bool", "vec3", "ivec3",
    "BaseData", "Tissue", "Chemistry", "Cell", "Metrics", "Params",
    "random", "random_dir", "math",
    "Grid", "AgentList",
    "tissue_rule", "chemistry_rule", "cell_rule", "metric_rule",
    "Simulation", "Engine", "CompilationError",
]

__version__ = "0.1.0"
