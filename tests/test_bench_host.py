"""Host logic of bench.py that needs no GPU: the workloads --workload precision
measures, and the summary that keeps the line's headline figures short."""
from __future__ import annotations

import sys

import pytest

from conftest import REPO

sys.path.insert(0, REPO)
import bench  # noqa: E402
from oncolytica_b200 import workloads as W  # noqa: E402


def test_precision_specs_of_a_named_workload():
    (sp,) = bench.precision_specs("scale", 1000)
    assert sp.name == W.SCALE.name and sp.capacity == 32 * W.SCALE.n_agents
    (sp,) = bench.precision_specs("scale", 1000, encoding="value", rank=1)
    assert sp.encoding == "value" and sp.seed == W.SCALE.seed + 1


def test_precision_specs_of_sweep_members():
    members = W.batched_specs(512, steps=500)
    specs = bench.precision_specs("batch:110,21,1,180", 500, encoding="value")
    assert [sp.name for sp in specs] == ["sweep_110", "sweep_21", "sweep_1", "sweep_180"]
    for sp, k in zip(specs, (110, 21, 1, 180)):
        # the member as the batched run builds it, encoding aside
        assert sp.field_dims == members[k].field_dims and sp.capacity == members[k].capacity
        assert sp.n_agents == members[k].n_agents and sp.encoding == "value"
    with pytest.raises(ValueError):
        bench.precision_specs("batch:", 500)


def test_summary_carries_the_recorded_member_errors():
    line = {"value": 1.0, "e2e": {"value": 0.9, "value_waiting": 0.8}, "roofline": {"frac": 1.0},
            "recorded": bench.recorded_runs()}
    out = bench.summarise(line)
    assert out["e2e_waiting"] == 0.8
    worst = out["recorded_sweep_members_worst_rel_l2_500_steps_values"]
    assert worst["f16_sr"] < 1e-3 < worst["bf16_sr"]
