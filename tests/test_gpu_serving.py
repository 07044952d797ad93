"""Serving pool on the GPU: requests that join and leave a running batch at
different steps (slots and arena ranges reused, out-of-order completion) each
return exactly what their solo run produces: live agents in device order,
fields (16-bit bits and residuals), metrics and reductions."""
from __future__ import annotations

import numpy as np
import pytest

from oncolytica_b200 import workloads as W
from oncolytica_b200._types import metric_fields
from oncolytica_b200.serving import CapacityError, PoolDevice, ServingPool, SimRequest

pytestmark = pytest.mark.gpu


def _specs(storage="f32"):
    base = dict(r_lo=4.0, r_hi=6.0, has_drug=True, v_lo=1.85, v_hi=2.0, storage=storage)
    return [
        W.TumourSpec(name="s0", n_agents=1500, domain=128.0, ball_radius=45.0, field_dims=(32, 32, 32),
                     D_o2=1500.0, uptake=0.6, death_k=0.3, seed=21, init_drug=0.3, **base),
        W.TumourSpec(name="s1", n_agents=4000, domain=192.0, ball_radius=70.0, field_dims=(48, 48, 48),
                     D_o2=2600.0, uptake=0.9, death_k=0.1, seed=22, init_drug=0.2, **base),
        W.TumourSpec(name="s2", n_agents=600, domain=128.0, ball_radius=30.0, field_dims=(32, 32, 32),
                     D_o2=1000.0, uptake=2.0, death_k=0.0, seed=23, **base),
        W.TumourSpec(name="s3", n_agents=6000, domain=256.0, ball_radius=80.0, field_dims=(64, 64, 64),
                     D_o2=3000.0, uptake=1.2, death_k=0.5, seed=24, init_drug=0.4, decay_drug=0.2, **base),
        W.TumourSpec(name="s4", n_agents=2500, domain=160.0, ball_radius=55.0, field_dims=(40, 40, 40),
                     D_o2=2000.0, uptake=0.8, death_k=0.2, seed=25, init_drug=0.1, **base),
    ]


def _device(specs, max_slots, voxels=None):
    proto = W.configure_engine(specs[0])
    tdims = tuple(max(s.tissue_dims[i] for s in specs) for i in range(3))
    from oncolytica_b200._geometry import voxel_table_size

    return PoolDevice(proto, max_slots=max_slots, max_rows=sum(s.capacity for s in specs),
                      table_entries=sum(voxel_table_size(s.tissue_dims) for s in specs),
                      field_voxels=voxels or sum(int(np.prod(s.field_dims)) + 64 for s in specs),
                      max_tissue_dims=tdims)


def _solo(spec, steps):
    e = W.build_engine(spec)
    if steps > 1:
        e.run_steps(steps - 1)
    e.run_step(collect_metrics=True)
    return e


def _check_same(spec, res, e):
    assert res.status == "done", res.error
    snap = e._backend_impl.snapshot()
    live = snap["life"] == 0
    for col, a in snap["cols"].items():
        np.testing.assert_array_equal(res.agents[col], a[live], err_msg=f"{spec.name} column {col}")
    for f, a in snap["fields"].items():
        if "residuals" in snap:
            np.testing.assert_array_equal(res.field_bits[f], a, err_msg=f"{spec.name} field {f} bits")
            np.testing.assert_array_equal(res.residuals[f], snap["residuals"][f], err_msg=f"{spec.name} {f} residual")
        else:
            np.testing.assert_array_equal(res.fields[f].ravel(order="F"), a, err_msg=f"{spec.name} field {f}")
    m = e.get_metrics()
    assert res.metrics == {k: getattr(m, k) for k in metric_fields(type(m))}, spec.name
    ra, rb = e.get_reductions(), res.reductions
    for key in ("n_live", "state_counts", "radial_hist", "max_r"):
        assert ra[key] == rb[key], (spec.name, key)
    np.testing.assert_allclose(ra["sum_pos"], rb["sum_pos"], rtol=1e-12)
    np.testing.assert_allclose(ra["sum_r2"], rb["sum_r2"], rtol=1e-12)
    for f in ra["field_mass"]:
        np.testing.assert_allclose(ra["field_mass"][f], rb["field_mass"][f], rtol=1e-12)
        assert ra["field_min"][f] == rb["field_min"][f] and ra["field_max"][f] == rb["field_max"][f]


@pytest.mark.parametrize("storage", ["f32", "bf16_sr", "f16_sr"])
def test_each_request_in_the_mix_matches_its_solo_run(cuda, storage):
    specs = _specs(storage)
    steps = [6, 3, 7, 4, 5]
    dev = _device(specs, max_slots=3)
    pool = ServingPool(dev)

    def req(k):
        eng, sim = W.configure_engine(specs[k])
        return SimRequest(eng, sim, steps[k], request_id=k)

    # 0, 1 and 2 start together; 3 and 4 arrive later and wait for free slots
    for k in (0, 1, 2):
        pool.submit(req(k))
    pool.step()
    pool.step()
    pool.submit(req(3))
    pool.submit(req(4))
    assert set(pool.residents) == {0, 1, 2}
    done = pool.drain()
    assert sorted(r.request_id for r in done) == [0, 1, 2, 3, 4]
    assert [r.request_id for r in done].index(1) < [r.request_id for r in done].index(0)  # out of order
    assert pool.device.counters()["status"] == 0
    for k, spec in enumerate(specs):
        _check_same(spec, pool.results[k], _solo(spec, steps[k]))
    u = dev.usage()
    assert u["slots_used"] == 0 and u["field_used"] == 0 and u["table_used"] == 0
    dev.close()


def test_admission_waits_for_field_memory(cuda):
    specs = _specs()[:4]
    big = int(np.prod(specs[3].field_dims))
    # room for the 64^3 member or the three small ones, not for all four
    dev = _device(specs, max_slots=8, voxels=big + 64)
    m = dev.admit(SimRequest(*W.configure_engine(specs[3]), 1, request_id=98))
    with pytest.raises(CapacityError):
        dev.admit(SimRequest(*W.configure_engine(specs[0]), 1, request_id=99))
    dev.retire(m)
    assert dev.usage()["field_used"] == 0
    dev.close()

    dev = _device(specs, max_slots=8, voxels=big + 64)
    pool = ServingPool(dev)
    steps = [2, 2, 2, 3]
    for k in (3, 0, 1, 2):
        e, s = W.configure_engine(specs[k])
        pool.submit(SimRequest(e, s, steps[k], request_id=k))
    pool.step()
    assert set(pool.residents) == {3}
    pool.drain()
    for k, spec in enumerate(specs):
        _check_same(spec, pool.results[k], _solo(spec, steps[k]))
    dev.close()


def test_mismatched_requests_are_rejected(cuda):
    specs = _specs()
    dev = _device(specs[:2], max_slots=4)
    pool = ServingPool(dev)
    e, s = W.configure_engine(W.scaled(specs[0], dt=0.05))
    pool.submit(SimRequest(e, s, 2, request_id=0))
    e, s = W.configure_engine(W.scaled(specs[1], storage="f16"))
    pool.submit(SimRequest(e, s, 2, request_id=1))
    e, s = W.configure_engine(specs[0])
    pool.submit(SimRequest(e, s, 2, request_id=2))
    pool.drain()
    assert pool.results[0].status == "rejected" and "dt" in pool.results[0].error
    assert pool.results[1].status == "rejected" and "storage" in pool.results[1].error
    _check_same(specs[0], pool.results[2], _solo(specs[0], 2))
    dev.close()


def test_served_chemistry_rules_match_solo_runs(cuda):
    """A model with a chemistry rule (chem_model: neighbour Laplacian, .cells
    secretion, three iterations) through the pool: three requests of two grid
    sizes, one joining two steps late, each return their solo run's agents
    and field."""
    import chem_model as CM

    import oncolytica_b200 as ol
    from oncolytica_b200._geometry import voxel_table_size

    def engine(shape, seed, n):
        rng = np.random.default_rng(seed)
        e = ol.Engine(backend="cuda", max_agents=8 * n)
        e.setup_geometry(tissue_shape=shape, tissue_voxel_size=4.0)
        e.setup_chemistry(CM.CChem)
        e.chemistry.column("signal")[...] = rng.uniform(0.0, 0.5, size=e.chemistry_shape).astype(np.float32)
        hi = np.array(shape, np.float32) * 4.0
        e.cells.add_arrays(CM.CCell, pos=(rng.uniform(0.1, 0.9, size=(n, 3)) * hi).astype(np.float32),
                           kind=rng.integers(0, 2, n), energy=rng.uniform(0.0, 1.1, n).astype(np.float32))
        return e

    cases = [((16, 16, 16), 5, 300, 5), ((24, 24, 24), 6, 600, 4), ((16, 16, 16), 7, 200, 3)]
    dev = PoolDevice((engine(*cases[0][:3]), CM.ChemSim()), max_slots=3, max_rows=sum(8 * c[2] for c in cases),
                     table_entries=sum(voxel_table_size(c[0]) for c in cases),
                     field_voxels=sum(int(np.prod([d // 2 for d in c[0]])) + 64 for c in cases),
                     max_tissue_dims=(24, 24, 24))
    pool = ServingPool(dev, depth=1)
    ids = [pool.submit(SimRequest(engine(*c[:3]), CM.ChemSim(), c[3], return_state=True)) for c in cases[:2]]
    pool.step()
    pool.step()
    ids.append(pool.submit(SimRequest(engine(*cases[2][:3]), CM.ChemSim(), cases[2][3], return_state=True)))
    pool.drain()
    for rid, (shape, seed, n, steps) in zip(ids, cases):
        res = pool.results[rid]
        assert res.status == "done", res.error
        e = engine(shape, seed, n)
        e.load_model(CM.ChemSim())
        e.run_steps(steps)
        snap = e._backend_impl.snapshot()
        live = snap["life"] == 0
        for col, a in snap["cols"].items():
            np.testing.assert_array_equal(res.agents[col], a[live], err_msg=f"request {rid} {col}")
        np.testing.assert_array_equal(res.fields["signal"].ravel(order="F"), snap["fields"]["signal"])
    dev.close()
