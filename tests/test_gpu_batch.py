"""Batched mode: every member of a batch reproduces its solo run bit for bit
(agent columns, life flags, fields), and per-member counts, metrics and
reductions agree with the solo engine's."""
from __future__ import annotations

import numpy as np
import pytest

from oncolytica_b200 import workloads as W
from oncolytica_b200._types import metric_fields

pytestmark = pytest.mark.gpu


def _members(storage="f32"):
    """Four uneven members: different grids, agent counts, diffusion, uptake,
    death rates and seeds (substep counts differ, odd and even)."""
    base = dict(r_lo=4.0, r_hi=6.0, has_drug=True, v_lo=1.85, v_hi=2.0, storage=storage)
    return [
        W.TumourSpec(name="m0", n_agents=1500, domain=128.0, ball_radius=45.0, field_dims=(32, 32, 32),
                     D_o2=1500.0, uptake=0.6, death_k=0.3, seed=11, init_drug=0.3, **base),
        W.TumourSpec(name="m1", n_agents=4000, domain=192.0, ball_radius=70.0, field_dims=(48, 48, 48),
                     D_o2=2600.0, uptake=0.9, death_k=0.1, seed=12, init_drug=0.2, **base),
        W.TumourSpec(name="m2", n_agents=600, domain=128.0, ball_radius=30.0, field_dims=(32, 32, 32),
                     D_o2=1000.0, uptake=2.0, death_k=0.0, seed=13, **base),
        W.TumourSpec(name="m3", n_agents=6000, domain=256.0, ball_radius=80.0, field_dims=(64, 64, 64),
                     D_o2=3000.0, uptake=1.2, death_k=0.5, seed=14, init_drug=0.4, decay_drug=0.2, **base),
    ]


def _metrics(eng):
    m = eng.get_metrics()
    return {k: getattr(m, k) for k in metric_fields(type(m))}


@pytest.mark.parametrize("graphs,storage", [(False, "f32"), (True, "f32"), (True, "bf16"), (False, "f16"),
                                            (True, "bf16_sr"), (True, "f16_sr")])
def test_batch_members_match_solo_runs(cuda, graphs, storage):
    specs = _members(storage)
    assert len({s.S_o2 % 2 for s in specs}) == 2  # odd and even substep counts
    states = [W.initial_state(s) for s in specs]
    solos = [W.build_engine(s, st) for s, st in zip(specs, states)]
    batch = W.build_batch(specs, states)
    batch.set_graphs(graphs)
    for step in range(7):
        collect = step % 3 == 2
        for e in solos:
            e.run_step(collect_metrics=collect)
        batch.run_step(collect_metrics=collect)
        for k, (spec, e) in enumerate(zip(specs, solos)):
            a = e._backend_impl.snapshot()
            b = batch.snapshot(k)
            assert a["rows"] == b["rows"], (step, k)
            np.testing.assert_array_equal(a["life"], b["life"], err_msg=f"life step {step} member {k}")
            for col in a["cols"]:
                np.testing.assert_array_equal(a["cols"][col], b["cols"][col], err_msg=f"{col} step {step} member {k}")
            for f in a["fields"]:
                np.testing.assert_array_equal(a["fields"][f], b["fields"][f], err_msg=f"{f} step {step} member {k}")
            for f in a.get("residuals", {}):
                np.testing.assert_array_equal(a["residuals"][f], b["residuals"][f], err_msg=f"{f} residual {step} {k}")
            assert ("residuals" in a) == (storage != "f32")
        if collect:
            reds = batch.get_reductions()
            for k, e in enumerate(solos):
                assert _metrics(e) == _metrics(batch.engines[k]), (step, k)
                ra, rb = e.get_reductions(), reds[k]
                for key in ("n_live", "state_counts", "radial_hist"):
                    assert ra[key] == rb[key], (step, k, key)
                assert ra["max_r"] == rb["max_r"]
                np.testing.assert_allclose(ra["sum_pos"], rb["sum_pos"], rtol=1e-12)
                np.testing.assert_allclose(ra["sum_r2"], rb["sum_r2"], rtol=1e-12)
                for f in ra["field_mass"]:
                    np.testing.assert_allclose(ra["field_mass"][f], rb["field_mass"][f], rtol=1e-12)
                    assert ra["field_min"][f] == rb["field_min"][f]
                    assert ra["field_max"][f] == rb["field_max"][f]
    # the members divided and died, so the check covered births and compaction
    c = batch.counters()
    assert c["status"] == 0
    assert sum(e._backend_impl.counters()["n_agents"] for e in solos) == \
        int(sum(len(np.nonzero(batch.member_rows()[0] == k)[0]) for k in range(len(specs))))


def test_batch_sync_to_host_splits_members(cuda):
    specs = _members()[:3]
    batch = W.build_batch(specs)
    batch.run_steps(3)
    batch.sync_to_host()
    solos = [W.build_engine(s) for s in specs]
    for e in solos:
        e.run_steps(3)
        e.sync_to_host()
    for k, e in enumerate(solos):
        a = e.cells.columns()
        b = batch.engines[k].cells.columns()
        for col in a:
            np.testing.assert_array_equal(a[col], b[col], err_msg=f"{col} member {k}")
        for f in ("o2", "drug"):
            np.testing.assert_array_equal(e.chemistry.column(f), batch.engines[k].chemistry.column(f))


def _chem_engine(shape, seed, n):
    import chem_model as CM
    import oncolytica_b200 as ol

    rng = np.random.default_rng(seed)
    eng = ol.Engine(backend="cuda", max_agents=8 * n)
    eng.setup_geometry(tissue_shape=shape, tissue_voxel_size=4.0)
    eng.setup_chemistry(CM.CChem)
    eng.chemistry.column("signal")[...] = rng.uniform(0.0, 0.5, size=eng.chemistry_shape).astype(np.float32)
    hi = np.array(shape, np.float32) * 4.0
    eng.cells.add_arrays(CM.CCell, pos=(rng.uniform(0.1, 0.9, size=(n, 3)) * hi).astype(np.float32),
                         kind=rng.integers(0, 2, n), energy=rng.uniform(0.0, 1.1, n).astype(np.float32))
    return eng, CM.ChemSim()


@pytest.mark.parametrize("graphs", [False, True])
def test_batched_chemistry_rules_match_solo_runs(cuda, graphs):
    """Chemistry rules in a batch: members of three grid sizes (chemistry
    8^3, 12^3 and 16x16x8) each give their solo run's agents and field bits."""
    from oncolytica_b200.batch import BatchEngine

    cases = [((16, 16, 16), 1, 300), ((24, 24, 24), 2, 700), ((32, 32, 16), 3, 500)]
    solos = []
    for shape, seed, n in cases:
        e, sim = _chem_engine(shape, seed, n)
        e.load_model(sim)
        e.set_graphs(graphs)
        e.run_steps(4)
        solos.append(e._backend_impl.snapshot())
    pairs = [_chem_engine(shape, seed, n) for shape, seed, n in cases]
    b = BatchEngine([e for e, _ in pairs], [s for _, s in pairs])
    b.set_graphs(graphs)
    b.run_steps(4)
    for k, ref in enumerate(solos):
        got = b.snapshot(k)
        assert got["rows"] == ref["rows"], k
        np.testing.assert_array_equal(got["life"], ref["life"])
        for c in ref["cols"]:
            np.testing.assert_array_equal(got["cols"][c], ref["cols"][c], err_msg=f"member {k} {c}")
        np.testing.assert_array_equal(got["fields"]["signal"], ref["fields"]["signal"], err_msg=f"member {k}")
    assert any(s["rows"] != n for s, (_, _, n) in zip(solos, cases)), "births or deaths should happen"
