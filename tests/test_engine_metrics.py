"""The engine's metrics set (engine/assets/shaders/tumor_sim.wgsl:248-361,
MetricIndex of engine/src/sim/readback.rs:25-50): the oracle's formulas on a
hand-checked case (CPU), and the device kernel (olc_engine_metrics) against
the oracle on the tumour workload (GPU)."""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle

EXACT = ("total_live", "n_prolif", "n_quiesc", "n_necr", "csc_count", "step")


def test_engine_metric_formulas_known_answer():
    # five agents on the diagonal; states: prolif, quiescent, necrotic,
    # prolif, deleted; one dead row that must not count
    x = np.array([10, 20, 30, 40, 50, 60], np.float32)
    life = np.array([0, 0, 0, 0, 0, 1], np.uint8)
    state = np.array([1, 2, 3, 1, 0, 1], np.int32)
    o2 = np.array([0.05, 0.5], np.float32)  # two voxels along x (cvs 30)
    csc = np.array([1, 0, 1, 0, 0, 1], np.int32)
    m = oracle.engine_metrics(x, x, x, life, state, (30.0, 30.0, 30.0), 7, o2=o2, cdims=(2, 1, 1), cvs=30.0,
                              csc=csc, energy=np.array([2, 4, 9, 6, 9, 9], np.float32))
    assert (m["total_live"], m["n_prolif"], m["n_quiesc"], m["n_necr"]) == (3, 2, 1, 1)
    assert m["frac_prolif"] == pytest.approx(2 / 3) and m["frac_necr"] == pytest.approx(1 / 4)
    # offsets -20, -10, +10 on each axis
    assert m["centroid_x"] == pytest.approx(30 - 20 / 3)
    assert m["r_gyration"] == pytest.approx(math.sqrt((1200 + 300 + 300) / 3))
    assert m["r_invasive"] == pytest.approx(math.sqrt(1200))
    assert m["r_necrotic"] == pytest.approx(0.5 * (1 / 0.65) ** 0.333333)
    assert m["rim_thickness"] == pytest.approx(math.sqrt(1200) - 0.5 * (1 / 0.65) ** 0.333333)
    # voxels: x 10, 20 -> 0 (O2 0.05, hypoxic); x 40 -> 1 (O2 0.5)
    assert m["mean_o2"] == pytest.approx((0.05 + 0.05 + 0.5) / 3, rel=1e-6)
    assert m["frac_hypoxic"] == pytest.approx(2 / 3)
    assert m["csc_count"] == 1 and m["mean_energy"] == pytest.approx(4.0)
    assert m["step"] == 7


@pytest.mark.gpu
@pytest.mark.parametrize("storage,crowd", [("f32", 12), ("f32", 3), ("f16_sr", 4)])
def test_engine_metrics_match_the_oracle(cuda, storage, crowd):
    from oncolytica_b200 import workloads as W
    from oncolytica_b200._geometry import voxel_table_size

    spec = W.scaled(W.SCALE, n_agents=3000, domain=120.0, ball_radius=35.0, field_dims=(32, 32, 32),
                    capacity=20_000, seed=5, uptake=2.0, death_k=0.3, init_drug=0.2, v_lo=1.9, v_hi=2.0,
                    storage=storage)
    eng = W.build_engine(spec)
    # an O2 ramp along x: no oxygen in the lower half of the domain, so the
    # first step holds necrotic, quiescent and proliferating agents (the
    # oracle's run of this case: 50 / 1874 / 993 after one step)
    x = (np.arange(spec.field_dims[0], dtype=np.float32) + 0.5) / spec.field_dims[0]
    eng.chemistry.column("o2")[...] = np.clip(2.0 * x - 1.0, 0.0, 1.0)[:, None, None]
    eng.sync_to_device()
    be = eng._backend_impl
    before = be.snapshot()
    eng.run_step(collect_metrics=True)
    after = be.snapshot()
    got = eng.get_engine_metrics(crowd_threshold=crowd)
    again = eng.get_engine_metrics(crowd_threshold=crowd)
    assert got == again, "repeated calls must give the same bits"

    b = before["cols"]
    counts = oracle.bin_counts_of(b["pos.x"], b["pos.y"], b["pos.z"], before["life"], spec.tissue_dims,
                                  spec.bin_size, voxel_table_size(spec.tissue_dims))
    code = {"f32": 0, "f16_sr": 4}[storage]

    def field(name):
        f = after["fields"][name]
        return f if code == 0 else oracle.from_bits16(f, code)

    c = after["cols"]
    exp = oracle.engine_metrics(c["pos.x"], c["pos.y"], c["pos.z"], after["life"], c["state"], be.caps.center,
                                be.counters()["steps"], o2=field("o2"), glu=field("drug"), cdims=spec.field_dims,
                                cvs=spec.dx, bin_counts=counts, tdims=spec.tissue_dims, tvs=spec.bin_size,
                                crowd=crowd)
    assert exp["n_necr"] > 0 and exp["n_quiesc"] > 0, "the case should hold every state"
    for k, v in exp.items():
        if k in EXACT:
            assert got[k] == v, (k, got[k], v)
        else:
            assert got[k] == pytest.approx(v, rel=1e-12, abs=1e-12), (k, got[k], v)
    if crowd < 12:
        assert got["crowd_frac"] > 0.0
    # the device counts agree with the per-step reductions and the metric rule
    red = eng.get_reductions()
    assert red["state_counts"][1] == got["n_prolif"] and red["state_counts"][3] == got["n_necr"]
