"""Cell-rule decisions pinned against the reference's own CPU backend.

tests/golden/cpu_rules.json holds every live agent after each of 12 steps of
tests/pinned_model.py run on the reference's CPUBackend
(framework/src/oncolytica/cpu/_cpu_backend.py:36-70; generated by
tests/golden/make_cpu_rules_golden.py from the reference itself).  The same
rules run here on the GPU from the same initial state: the live set, every
integer column and the positions match exactly, the float energy to 2e-6
relative (FP32 here, Python doubles there; its decisions stay at least 0.016
from their threshold).  The reference CPU's metrics accumulate over steps and
count the agents that died in the step (its AgentList iteration does not skip
them); this package clears metrics per collection and counts live agents
(declared divergence), so each step's metrics are checked against the live
agents, and the fixture's accumulated counts against live + died.
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

import oncolytica_b200 as ol
import pinned_model as PM
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def test_rules_match_the_reference_cpu_backend(cuda):
    with open(os.path.join(GOLDEN, "cpu_rules.json")) as fh:
        gold = json.load(fh)
    st = gold["initial"]
    eng = ol.Engine(backend="cuda", max_agents=4096)
    eng.setup_geometry(tissue_shape=tuple(gold["tissue_shape"]), tissue_voxel_size=gold["tissue_voxel_size"],
                       cell_diameter=1.0)
    eng.setup_tissue(PM.PTissue)
    eng.tissue.column("stiff")[...] = np.array(st["stiff"], np.int32)
    eng.setup_chemistry(PM.PChem)
    eng.chemistry.column("nutrient")[...] = np.array(st["nutrient"], np.float32)
    n = len(st["uid"])
    eng.cells.add_arrays(PM.PCell, pos=np.array(st["pos"], np.float32), uid=np.array(st["uid"], np.int32),
                         age=np.zeros(n, np.int32), kind=np.array(st["kind"], np.int32),
                         energy=np.array(st["energy"], np.float32))
    eng.load_model(PM.PinnedSim())
    prev = {"n": 0, "n_b": 0, "age_sum": 0}
    for rec in gold["steps"]:
        eng.run_step(collect_metrics=True)
        eng.sync_to_host()
        cols = eng.cells.columns()
        order = np.argsort(cols["uid"], kind="stable")
        exp = np.array(rec["agents"], np.float64)  # uid, age, kind, energy, x, y, z (sorted by uid)
        assert len(order) == len(exp), rec["step"]
        np.testing.assert_array_equal(cols["uid"][order], exp[:, 0].astype(np.int32), err_msg=f"step {rec['step']}")
        np.testing.assert_array_equal(cols["age"][order], exp[:, 1].astype(np.int32))
        np.testing.assert_array_equal(cols["kind"][order], exp[:, 2].astype(np.int32))
        np.testing.assert_allclose(cols["energy"][order], exp[:, 3], rtol=2e-6, atol=0)
        for k, a in enumerate(("pos.x", "pos.y", "pos.z")):
            np.testing.assert_array_equal(cols[a][order], exp[:, 4 + k].astype(np.float32))
        m = eng.get_metrics()
        live_b = int((exp[:, 2] == 1).sum())
        assert (m.n, m.n_b, m.age_sum) == (len(exp), live_b, int(exp[:, 1].sum())), rec["step"]
        # the reference's accumulated count gained this step's live and dead agents
        assert rec["metrics"]["n"] - prev["n"] == len(exp) + len(rec["died"])
        prev = rec["metrics"]
    assert sum(len(r["died"]) for r in gold["steps"]) > 0
