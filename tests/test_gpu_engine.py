"""Engine-level GPU tests: the reference's own GPU end-to-end tests
(framework/tests/test_gpu.py, framework/tests/test_oncolytica.py) run on the
CUDA backend, and the tumour workload step against the C oracle."""
from __future__ import annotations

import json
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN

import oncolytica_b200 as ol
from oncolytica_b200 import workloads as W
from oncolytica_b200._geometry import get_tissue_voxel_key, voxel_table_size
from oncolytica_b200._types import metric_fields

pytestmark = pytest.mark.gpu


# ---------------------------------------------------------------- fixtures of the reference tests

class MockCell(ol.Cell):
    pos: ol.vec3
    id: int


class MockTissue(ol.Tissue):
    pad: int = 0


class MockChemistry(ol.Chemistry):
    pad: ol.f32 = 0.0


class MockMetrics(ol.Metrics):
    pad: int = 0


class MockParams(ol.Params):
    pass


class FakeSim(ol.Simulation[MockTissue, MockChemistry, MockCell, MockMetrics, MockParams]):
    pass


class MyCell(ol.Cell):
    pos: ol.vec3 = ol.vec3(50.0, 50.0, 50.0)
    health: ol.f32
    mutated: ol.bool


class MyTissue(ol.Tissue):
    oxygen: ol.f32 = 1.0


class MyChem(ol.Chemistry):
    drug_conc: ol.f32 = 0.0


class MyMetrics(ol.Metrics):
    alive_cells: ol.u32 = 0


class MyParams(ol.Params):
    pass


class BasicSim(ol.Simulation[MyTissue, MyChem, MyCell, MyMetrics, MyParams]):
    @ol.cell_rule
    def cell_logic(self, cell: MyCell):
        cell.health -= 10.0
        if cell.health <= 0.0:
            cell.die()

    @ol.metric_rule
    def track_deaths(self, cell: MyCell, metrics: MyMetrics):
        metrics.alive_cells += 1


def test_sort_contract_through_engine(cuda):
    """framework/tests/test_gpu.py:17-61 on Engine(backend='cuda')."""
    d = np.load(os.path.join(GOLDEN, "sort_contract.npz"))
    pos = d["pos"]
    n = len(pos)
    gdim = tuple(int(v) for v in d["dims"])
    vs = float(d["vs"])
    eng = ol.Engine(backend="cuda", max_agents=n)
    eng.setup_geometry(gdim, vs)
    for i in range(n):
        c = MockCell()
        c.pos, c.id = ol.vec3(*pos[i]), i
        eng.cells.add(c)
    eng.load_model(FakeSim())
    eng.run_step()
    eng.sync_to_host()
    nv = voxel_table_size(gdim)
    buckets: dict[int, list[int]] = {}
    for c in eng.cells._data:
        vk = get_tissue_voxel_key(*(int(float(v) / vs) for v in (c.pos.x, c.pos.y, c.pos.z)))
        buckets.setdefault(vk, []).append(c.id)
    ref: dict[int, list[int]] = {}
    for i, k in enumerate(d["keys"].tolist()):
        ref.setdefault(k, []).append(i)
    for vk in range(nv):
        assert sorted(buckets.get(vk, [])) == sorted(ref.get(vk, [])), vk
    ids = [c.id for c in eng.cells._data]
    assert sorted(ids) == list(range(n))
    # deterministic refinement: stable, so ids ascend within each key
    for vk, lst in buckets.items():
        assert lst == sorted(lst)


def test_die_removes_agent_and_metrics_skip_it(cuda):
    """framework/tests/test_oncolytica.py:300-365 (die + metrics + count)."""

    class TestCell(ol.Cell):
        pos: ol.vec3
        type_id: ol.i32 = 0

    class TestMetrics(ol.Metrics):
        alive_count: ol.u32 = 0

    class TestParams(ol.Params):
        pass

    class DieSim(ol.Simulation[MyTissue, MyChem, TestCell, TestMetrics, TestParams]):
        @ol.cell_rule
        def rule(self, cell: TestCell):
            if cell.type_id == 1:
                cell.die()

        @ol.metric_rule
        def calc_metrics(self, cell: TestCell, m: TestMetrics):
            m.alive_count += 1

    eng = ol.Engine(backend="cuda", max_agents=4)
    eng.setup_geometry(tissue_shape=(10, 10, 10), tissue_voxel_size=2.0)
    eng.cells.add(TestCell(pos=ol.vec3(5.0, 5.0, 5.0), type_id=2))
    eng.cells.add(TestCell(pos=ol.vec3(1.0, 1.0, 1.0), type_id=1))
    eng.load_model(DieSim())
    eng.run_step(collect_metrics=True)
    assert eng.get_metrics().alive_count == 1
    eng.sync_to_host()
    types = [c.type_id for c in eng.cells._data]
    assert types == [2]
    assert math.isclose(eng.cells._data[0].pos.x, 5.0)
    eng.run_step(collect_metrics=True)
    assert eng.get_metrics().alive_count == 1
    assert eng._backend_impl.counters()["deaths"] == 1


def test_divide_appends_child(cuda):
    """framework/tests/test_oncolytica.py:367-405."""

    class DivCell(ol.Cell):
        pos: ol.vec3
        generation: ol.i32 = 0

    class DivideSim(ol.Simulation[MyTissue, MyChem, DivCell, MyMetrics, MyParams]):
        @ol.cell_rule
        def rule(self, cell: DivCell):
            if cell.generation == 0:
                new_cell = DivCell()
                new_cell.pos = cell.pos + ol.vec3(1.0, 0.0, 0.0)
                new_cell.generation = 1
                cell.divide(new_cell)
                cell.generation = 1

    eng = ol.Engine(backend="cuda", max_agents=10)
    eng.setup_geometry(tissue_shape=(10, 10, 10))
    eng.cells.add(DivCell(pos=ol.vec3(5.0, 5.0, 5.0)))
    eng.load_model(DivideSim())
    eng.run_step()
    eng.sync_to_host()
    assert len(eng.cells._data) == 2
    assert [c.generation for c in eng.cells._data] == [1, 1]
    assert eng.cells._data[1].pos.x == np.float32(6.0)


def test_cpu_lifecycle_golden(cuda):
    """framework/tests/test_oncolytica.py:58-93, per-step counts from the
    reference CPUBackend run (tests/golden/cpu_lifecycle.json)."""
    g = json.load(open(os.path.join(GOLDEN, "cpu_lifecycle.json")))
    for key, health in (("A_default_health", None), ("B_health_100", 100.0)):
        eng = ol.Engine(backend="cuda")
        for i in range(5):
            cell = MyCell()
            cell.pos = ol.vec3(50.0, 50.0, 50.0) + 5.0 * ol.vec3(float(i))
            if health is not None:
                cell.health = health
            eng.cells.add(cell)
        eng.load_model(BasicSim())
        for rec in g[key]:
            collect = "metric_alive_cells" in rec
            eng.run_step(collect_metrics=collect)
            eng.sync_to_host()
            assert len(eng.cells._data) == rec["alive_after"], (key, rec)
            if collect:
                assert eng.get_metrics().alive_cells == rec["metric_alive_cells"]


def test_noncubic_grid_runs(cuda):
    """framework/tests/test_oncolytica.py:267-298 (cell rule part)."""

    class FullSim(ol.Simulation[MyTissue, MyChem, MyCell, MyMetrics, MyParams]):
        @ol.cell_rule
        def cell_logic(self, cell: MyCell):
            if cell.health > 50.0:
                cell.pos.x += 0.5

    eng = ol.Engine(backend="cuda")
    eng.setup_geometry(tissue_shape=(120, 64, 32))
    for i in range(4):
        eng.cells.add(MyCell(pos=ol.vec3(float(i) * 5.0, 0.0, 0.0), health=60.0))
    eng.load_model(FullSim())
    eng.run_step()
    eng.run_step()
    eng.sync_to_host()
    xs = sorted(float(c.pos.x) for c in eng.cells._data)
    assert xs == [1.0, 6.0, 11.0, 16.0]


def test_randomness_runs_and_is_reproducible(cuda):
    """framework/tests/test_oncolytica.py:437-459, plus reproducibility."""

    class RandSim(ol.Simulation[MyTissue, MyChem, MyCell, MyMetrics, MyParams]):
        @ol.cell_rule
        def rule(self, cell: MyCell):
            dist = ol.random() * 2.0
            direction = ol.random_dir()
            cell.pos += direction * dist

    def run():
        eng = ol.Engine(backend="cuda")
        eng.setup_geometry(tissue_shape=(20, 20, 20), tissue_voxel_size=2.0)
        for i in range(100):
            eng.cells.add(MyCell(pos=ol.vec3(20.0 + 0.1 * i, 20.0, 20.0)))
        eng.load_model(RandSim())
        for _ in range(3):
            eng.run_step()
        eng.sync_to_host()
        return np.array([[c.pos.x, c.pos.y, c.pos.z] for c in eng.cells._data])

    a, b = run(), run()
    np.testing.assert_array_equal(a, b)
    assert np.abs(a - 20.0).max() > 0.1


def test_update_params_reaches_device(cuda):
    class PCell(ol.Cell):
        pos: ol.vec3
        v: ol.f32 = 0.0

    class PParams(ol.Params):
        inc: ol.f32 = 1.0

    class PSim(ol.Simulation[MyTissue, MyChem, PCell, MyMetrics, PParams]):
        @ol.cell_rule
        def rule(self, cell: PCell):
            cell.v += self.params.inc

    eng = ol.Engine(backend="cuda")
    eng.cells.add(PCell(pos=ol.vec3(1.0, 1.0, 1.0)))
    eng.load_model(PSim())
    eng.run_step()
    eng.update_params(inc=10.0)
    eng.run_step()
    eng.sync_to_host()
    assert eng.cells._data[0].v == np.float32(11.0)


# ---------------------------------------------------------------- tumour workload vs the C oracle

def _parity_spec():
    return W.scaled(W.SCALE, n_agents=20_000, domain=200.0, ball_radius=55.0, field_dims=(48, 48, 48),
                    capacity=100_000, seed=3, uptake=4.0, death_k=0.5, init_drug=0.2, v_lo=1.85, v_hi=2.0)


def test_tumour_step_parity_with_oracle(cuda):
    """Each step from an identical state: integer columns, life flags, volumes,
    radii and both fields bit-exact; positions to 1e-4 µm (children are placed
    with cos/sin of the random direction, which the two math libraries may
    round differently by an ulp)."""
    import oracle

    spec = _parity_spec()
    eng = W.build_engine(spec)
    # an O2 ramp along x puts agents in every branch of the rule
    x = (np.arange(spec.field_dims[0], dtype=np.float32) + 0.5) / spec.field_dims[0]
    eng.chemistry.column("o2")[...] = np.clip(2.2 * x - 0.6, 0.0, 1.0)[:, None, None]
    eng.sync_to_device()
    be = eng._backend_impl
    seen = {"div": 0, "dead": 0, "quiescent": 0, "necrotic": 0}
    for step in range(6):
        snap = be.snapshot()
        orc = oracle.TumourOracle.from_snapshot(spec, snap, spec.capacity)
        eng.run_step()
        orc.step(nthreads=4)
        got = be.snapshot()
        n = got["rows"]
        assert n == orc.rows, step
        np.testing.assert_array_equal(got["life"], orc.dead[:n])
        for col, key in (("state", "state"), ("_rng_state", "rng"), ("volume", "volume"), ("radius", "radius")):
            np.testing.assert_array_equal(got["cols"][col], orc.bufs[key][:n], err_msg=f"{col} step {step}")
        for a, key in (("pos.x", "x"), ("pos.y", "y"), ("pos.z", "z")):
            np.testing.assert_allclose(got["cols"][a], orc.bufs[key][:n], rtol=0, atol=1e-4)
        np.testing.assert_array_equal(got["fields"]["o2"], orc.o2.ravel())
        np.testing.assert_array_equal(got["fields"]["drug"], orc.drug.ravel())
        np.testing.assert_array_equal(got["sinks"]["o2"], orc.o2_sink.ravel())
        seen["div"] += int(orc.t.births)
        seen["dead"] += int(orc.dead[:n].sum())
        st = got["cols"]["state"]
        seen["quiescent"] += int((st == 2).sum())
        seen["necrotic"] += int((st == 3).sum())
    # the case exercises every branch of the rule
    assert all(v > 0 for v in seen.values()), seen


def test_empty_and_extinct_populations(cuda):
    """No agents at all, and a population that the drug kills within one step
    (death_k * drug far above 1): steps run eagerly and from CUDA graphs, rows,
    life flags and both fields follow the oracle's steps bit for bit, the dead
    leave at the next sort, and the step status stays clean with zero rows."""
    import oracle

    base = _parity_spec()
    for spec in (W.scaled(base, n_agents=0), W.scaled(base, n_agents=2000, death_k=1.0e6)):
        eng = W.build_engine(spec)
        be = eng._backend_impl
        for step in range(4):
            eng.set_graphs(step >= 2)
            snap = be.snapshot()
            orc = oracle.TumourOracle.from_snapshot(spec, snap, spec.capacity)
            eng.run_step(collect_metrics=True)
            orc.step(nthreads=4)
            got = be.snapshot()
            n = got["rows"]
            assert n == orc.rows, (spec.n_agents, step)
            np.testing.assert_array_equal(got["life"], orc.dead[:n])
            np.testing.assert_array_equal(got["fields"]["o2"], orc.o2.ravel())
            np.testing.assert_array_equal(got["fields"]["drug"], orc.drug.ravel())
            if spec.n_agents and step == 0:
                assert n == spec.n_agents and got["life"].all()  # every agent died in the first step
        c = be.counters()
        assert got["rows"] == 0 and c["status"] == 0 and c["births"] == 0
        assert eng.get_engine_metrics()["total_live"] == 0
        eng.close()


def test_engine_mechanics_path_in_the_step(cuda):
    """The step's contact stage through k_contact_mech (OlcMechanics enabled
    with the plain law's parameters: necrotic factor 1, no adhesion,
    overdamped) reproduces the oracle's plain step, so the state and column
    plumbing of the extended kernel is the plain kernel's; a necrotic factor
    of 0.3 then changes the positions of agents touching necrotic ones."""
    import ctypes as C

    import oracle
    from oncolytica_b200 import _lib

    spec = _parity_spec()
    eng = W.build_engine(spec)
    x = (np.arange(spec.field_dims[0], dtype=np.float32) + 0.5) / spec.field_dims[0]
    eng.chemistry.column("o2")[...] = np.clip(2.2 * x - 0.6, 0.0, 1.0)[:, None, None]
    eng.sync_to_device()
    be = eng._backend_impl
    m = _lib.OlcMechanics(state_field=be.layout.col_index("state"), necrotic_factor=1.0, adhesion_stiffness=0.0,
                          adhesion_range=0.0, velocity_field=-1, damping=1.0, max_speed=8.0, enabled=1)
    be._check(be.lib.olc_set_mechanics(be.handle, C.byref(m)))
    for step in range(3):
        snap = be.snapshot()
        orc = oracle.TumourOracle.from_snapshot(spec, snap, spec.capacity)
        eng.run_step()
        orc.step(nthreads=4)
        got = be.snapshot()
        n = got["rows"]
        assert n == orc.rows
        for a, key in (("pos.x", "x"), ("pos.y", "y"), ("pos.z", "z")):
            np.testing.assert_allclose(got["cols"][a], orc.bufs[key][:n], rtol=0, atol=1e-4)
    assert (got["cols"]["state"] == 3).any()
    snap = be.snapshot()
    orc = oracle.TumourOracle.from_snapshot(spec, snap, spec.capacity)
    m.necrotic_factor = 0.3
    be._check(be.lib.olc_set_mechanics(be.handle, C.byref(m)))
    eng.run_step()
    orc.step(nthreads=4)
    got = be.snapshot()
    n = got["rows"]
    np.testing.assert_array_equal(got["cols"]["state"], orc.bufs["state"][:n])
    moved = np.abs(got["cols"]["pos.x"] - orc.bufs["x"][:n]) > 1e-3
    assert moved.any(), "a necrotic factor of 0.3 must change some contacts"


def test_engine_active_motion_in_the_step(cuda):
    """Chemotaxis and random motility through Engine.setup_contact: one step
    from the same state with and without them keeps rows, states and life
    flags; every live non-necrotic agent's RNG is two xorshift32 draws further
    (the random direction), necrotic ones draw nothing, and positions move."""
    spec = _parity_spec()

    def run(**kw):
        eng, sim = W.configure_engine(spec)
        eng.setup_contact(radius="radius", stiffness=spec.stiffness, mobility=spec.mobility,
                          max_disp=spec.max_disp, margin=spec.margin, **kw)
        eng.load_model(sim)
        x = (np.arange(spec.field_dims[0], dtype=np.float32) + 0.5) / spec.field_dims[0]
        eng.chemistry.column("o2")[...] = np.clip(2.0 * x - 1.0, 0.0, 1.0)[:, None, None]  # no O2 below mid-x
        eng.sync_to_device()
        eng.run_step()
        snap = eng._backend_impl.snapshot()
        snap["births"] = eng._backend_impl.counters()["births"]
        return snap

    plain = run()
    moved = run(chemotaxis=(2.0, 0.5), motility=0.3)
    assert plain["births"] == moved["births"] > 0
    assert plain["rows"] == moved["rows"]
    np.testing.assert_array_equal(plain["life"], moved["life"])
    np.testing.assert_array_equal(plain["cols"]["state"], moved["cols"]["state"])

    def two_draws(s):
        s = s.astype(np.uint64)
        for _ in range(2):
            s ^= (s << 13) & 0xFFFFFFFF
            s ^= s >> 17
            s ^= (s << 5) & 0xFFFFFFFF
        return s.astype(np.uint32)

    # the contact stage moves the rows that entered the step; this step's
    # children (appended after them) keep the RNG their parents gave them
    entered = np.arange(plain["rows"]) < plain["rows"] - plain["births"]
    live = (plain["life"] == 0) & entered
    active = live & (plain["cols"]["state"] != 3)
    np.testing.assert_array_equal(moved["cols"]["_rng_state"][active], two_draws(plain["cols"]["_rng_state"][active]))
    np.testing.assert_array_equal(moved["cols"]["_rng_state"][~entered], plain["cols"]["_rng_state"][~entered])
    nec = live & (plain["cols"]["state"] == 3)
    assert nec.any()
    np.testing.assert_array_equal(moved["cols"]["_rng_state"][nec], plain["cols"]["_rng_state"][nec])
    assert np.abs(moved["cols"]["pos.x"][active] - plain["cols"]["pos.x"][active]).max() > 1e-3


def test_vessel_holds_its_voxels(cuda):
    """Engine.setup_vessel: the O2 voxels inside the vessel cylinder hold 1.0
    after every step (eager and graph steps alike), and the field around it
    is richer than without the vessel."""
    spec = _parity_spec()

    def run(vessel, graphs):
        eng, sim = W.configure_engine(spec)
        if vessel:
            eng.setup_vessel(center=(100.0, 100.0), radius=15.0, fields=("o2",))
        eng.load_model(sim)
        eng.chemistry.column("o2")[...] = 0.2
        eng.sync_to_device()
        eng.set_graphs(graphs)
        eng.run_steps(3)
        return eng, eng._backend_impl.snapshot()["fields"]["o2"]

    eng, o2 = run(True, False)
    idx = eng.vessel_voxels()
    assert len(idx) > 0 and np.all(o2[idx] == np.float32(1.0))
    _, o2_graphs = run(True, True)
    np.testing.assert_array_equal(o2_graphs, o2)
    _, o2_plain = run(False, False)
    assert o2.sum() > o2_plain.sum()


def test_plain_small_full_size_step_parity(cuda):
    """The plain workload at its own size (10,000 agents in a 256 um domain,
    one 64^3 O2 field with 79 substeps, 10 um bins decoupled from the field
    grid): five steps, each from the device state, against the oracle: rows,
    life flags and the integer and volume columns bit-exact, the field and the
    pending sink bit-exact, positions to 1e-4 um."""
    import oracle

    spec = W.PLAIN_SMALL
    eng = W.build_engine(spec)
    be = eng._backend_impl
    births = 0
    for step in range(5):
        snap = be.snapshot()
        orc = oracle.TumourOracle.from_snapshot(spec, snap, spec.capacity)
        eng.run_step()
        orc.step(nthreads=4)
        got = be.snapshot()
        n = got["rows"]
        assert n == orc.rows, step
        np.testing.assert_array_equal(got["life"], orc.dead[:n])
        for col, key in (("state", "state"), ("_rng_state", "rng"), ("volume", "volume"), ("radius", "radius")):
            np.testing.assert_array_equal(got["cols"][col], orc.bufs[key][:n], err_msg=f"{col} step {step}")
        for a, key in (("pos.x", "x"), ("pos.y", "y"), ("pos.z", "z")):
            np.testing.assert_allclose(got["cols"][a], orc.bufs[key][:n], rtol=0, atol=1e-4)
        np.testing.assert_array_equal(got["fields"]["o2"], orc.o2.ravel())
        np.testing.assert_array_equal(got["sinks"]["o2"], orc.o2_sink.ravel())
        births += int(orc.t.births)
    assert spec.n_agents == 10_000 and tuple(spec.field_dims) == (64, 64, 64) and births > 0


def test_scale_workload_full_size_step_parity(cuda):
    """The scale workload at its own size (1,000,000 agents in a 400 um ball,
    two 256^3 fields with 83 + 21 substeps, 100^3 bins and 21-bit keys): two
    steps, each from the device state, against the oracle on every host
    thread: rows, life flags, integer and volume columns, both fields and the
    pending sink bit-exact, positions to 1e-4 um."""
    import os

    import oracle

    spec = W.SCALE
    eng = W.build_engine(spec)
    be = eng._backend_impl
    threads = max(1, os.cpu_count() or 1)
    for step in range(2):
        snap = be.snapshot()
        orc = oracle.TumourOracle.from_snapshot(spec, snap, spec.capacity)
        eng.run_step()
        orc.step(nthreads=threads)
        got = be.snapshot()
        n = got["rows"]
        assert n == orc.rows, step
        np.testing.assert_array_equal(got["life"], orc.dead[:n])
        for col, key in (("state", "state"), ("_rng_state", "rng"), ("volume", "volume"), ("radius", "radius")):
            np.testing.assert_array_equal(got["cols"][col], orc.bufs[key][:n], err_msg=f"{col} step {step}")
        for a, key in (("pos.x", "x"), ("pos.y", "y"), ("pos.z", "z")):
            np.testing.assert_allclose(got["cols"][a], orc.bufs[key][:n], rtol=0, atol=1e-4)
        np.testing.assert_array_equal(got["fields"]["o2"], orc.o2.ravel())
        np.testing.assert_array_equal(got["fields"]["drug"], orc.drug.ravel())
        np.testing.assert_array_equal(got["sinks"]["o2"], orc.o2_sink.ravel())
    assert n >= spec.n_agents * 0.9 and tuple(spec.field_dims) == (256, 256, 256)
    eng.close()


def test_tumour_long_run_statistics(cuda):
    """Independent 60-step runs (GPU vs oracle, same seed): population counts
    within 1 % and radial profiles within 3 % of the live count."""
    import oracle

    spec = W.scaled(W.PLAIN_SMALL, n_agents=4000, domain=160.0, ball_radius=40.0, field_dims=(40, 40, 40),
                    capacity=40_000, seed=11, uptake=0.5)
    eng = W.build_engine(spec)
    st = W.initial_state(spec)
    o2, _ = W.initial_fields(spec)
    orc = oracle.TumourOracle(spec, st, o2, None, spec.capacity)
    for _ in range(60):
        eng.run_step()
        orc.step(nthreads=4)
    eng.sync_to_host()
    cols = eng.cells.columns()
    live_g = len(cols["state"])
    live_o = orc.live_agents()
    assert abs(live_g - len(live_o["state"])) <= 0.01 * live_g
    for s in (1, 2, 3):
        a = int((cols["state"] == s).sum())
        b = int((live_o["state"] == s).sum())
        assert abs(a - b) <= max(5, 0.02 * live_g), (s, a, b)
    c = np.array(spec.center)
    rg = np.linalg.norm(np.stack([cols["pos.x"], cols["pos.y"], cols["pos.z"]], 1) - c, axis=1)
    ro = np.linalg.norm(np.stack([live_o["x"], live_o["y"], live_o["z"]], 1) - c, axis=1)
    hg, _ = np.histogram(rg, bins=16, range=(0, 80))
    ho, _ = np.histogram(ro, bins=16, range=(0, 80))
    assert np.abs(hg - ho).max() <= 0.03 * live_g


def test_plain_workload_full_run_statistics(cuda):
    """The plain workload as configured (10,000 agents in a 60 um ball, a 256
    um domain, one 64^3 O2 field with 79 substeps, dt 0.1 h) for its full 100
    steps, the GPU and the oracle running independently from the same seed:
    live and per-state counts within 1 %, radial histograms of the live agents
    within 3 % of the live count in every bin, and the O2 fields within 1e-3
    relative L2.  The runs do not share states after step 0, so this checks
    the trajectory as a whole, not step by step (positions of children differ
    by an ulp of cos/sin, and the divergence grows through the contact law)."""
    import oracle

    spec = W.PLAIN_SMALL
    assert spec.n_agents == 10_000 and tuple(spec.field_dims) == (64, 64, 64) and spec.steps == 100
    eng = W.build_engine(spec)
    eng.set_graphs(True)
    st = W.initial_state(spec)
    o2, _ = W.initial_fields(spec)
    orc = oracle.TumourOracle(spec, st, o2, None, spec.capacity)
    for _ in range(spec.steps):
        orc.step(nthreads=0)
    eng.run_steps(spec.steps)
    be = eng._backend_impl
    assert be.counters()["status"] == 0
    eng.sync_to_host()
    cols = eng.cells.columns()
    live_g = len(cols["state"])
    live_o = orc.live_agents()
    assert live_g > 1.2 * spec.n_agents, "the run should grow"
    assert abs(live_g - len(live_o["state"])) <= 0.01 * live_g, (live_g, len(live_o["state"]))
    for s in (1, 2, 3):
        a = int((cols["state"] == s).sum())
        b = int((live_o["state"] == s).sum())
        assert abs(a - b) <= max(5, 0.01 * live_g), (s, a, b)
    c = np.array(spec.center)
    rg = np.linalg.norm(np.stack([cols["pos.x"], cols["pos.y"], cols["pos.z"]], 1) - c, axis=1)
    ro = np.linalg.norm(np.stack([live_o["x"], live_o["y"], live_o["z"]], 1) - c, axis=1)
    hg, _ = np.histogram(rg, bins=20, range=(0, 100))
    ho, _ = np.histogram(ro, bins=20, range=(0, 100))
    assert np.abs(hg - ho).max() <= 0.03 * live_g, (hg, ho)
    fo = be._field_values(0, be._current()[1]).astype(np.float64)
    ref = orc.o2.ravel().astype(np.float64)
    assert np.linalg.norm(fo - ref) / np.linalg.norm(ref) <= 1e-3


def test_graph_steps_match_eager_steps(cuda):
    """Steps replayed from cached CUDA graphs give bit-identical state,
    counters, reductions and metrics to eager steps, across parity states,
    metric collection, a params update and a host re-upload."""
    spec = W.scaled(_parity_spec(), n_agents=8000, capacity=60_000)
    engines = [W.build_engine(spec) for _ in range(2)]
    engines[1].set_graphs(True)

    def run(eng, k):
        if k == 3:
            eng.update_params(death_k=0.25)
        if k == 5:
            eng.sync_to_host()
            eng.sync_to_device()
        eng.run_steps(2, collect_metrics=(k % 2 == 1))

    for k in range(8):
        for eng in engines:
            run(eng, k)
        a, b = (e._backend_impl.snapshot() for e in engines)
        assert a["rows"] == b["rows"], k
        np.testing.assert_array_equal(a["life"], b["life"])
        for col in a["cols"]:
            np.testing.assert_array_equal(a["cols"][col], b["cols"][col], err_msg=f"{col} round {k}")
        for f in a["fields"]:
            np.testing.assert_array_equal(a["fields"][f], b["fields"][f])
        ca, cb = (e._backend_impl.counters() for e in engines)
        assert ca == cb, k
        if k % 2 == 1:
            assert engines[0].get_reductions() == engines[1].get_reductions()
            ma, mb = (e.get_metrics() for e in engines)
            assert {k: getattr(ma, k) for k in metric_fields(type(ma))} == \
                   {k: getattr(mb, k) for k in metric_fields(type(mb))}


@pytest.mark.parametrize("storage,code", [("bf16", 1), ("f16", 2), ("bf16_sr", 3), ("f16_sr", 4)])
def test_tumour_step_parity_16bit_fields(cuda, storage, code):
    """16-bit field storage through the engine: each step from an identical
    state gives the oracle's field bits and residuals (reaction + substeps,
    oracle.diffuse16), and the agent phase, run by the oracle on those field
    values, gives the same agents, life flags and uptake sink."""
    import oracle

    spec = W.scaled(_parity_spec(), storage=storage)
    eng = W.build_engine(spec)
    x = (np.arange(spec.field_dims[0], dtype=np.float32) + 0.5) / spec.field_dims[0]
    eng.chemistry.column("o2")[...] = np.clip(2.2 * x - 0.6, 0.0, 1.0)[:, None, None]
    eng.sync_to_device()
    be = eng._backend_impl
    shp = tuple(spec.field_dims[::-1])
    # what the elements hold: BF16 fields default to three offsets, FP16 to values
    e_o2, e_dr = be.field_codec("o2")[1], be.field_codec("drug")[1]
    assert (e_o2, e_dr) == ((2, 2) if code in (1, 3) else (0, 0))
    for step in range(4):
        snap = be.snapshot()
        k = be.counters()["steps"]  # the step count salts stochastic rounding, with the field's index
        o2_bits, o2_res = oracle.diffuse16(snap["fields"]["o2"].reshape(shp), snap["sinks"]["o2"].reshape(shp),
                                           snap["residuals"]["o2"].reshape(shp), spec.dx, spec.dt, spec.D_o2, 0.0,
                                           spec.bnd_o2, spec.S_o2, code, step=k, field=0, encoding=e_o2)
        dr_bits, dr_res = oracle.diffuse16(snap["fields"]["drug"].reshape(shp), None,
                                           snap["residuals"]["drug"].reshape(shp), spec.dx, spec.dt, spec.D_drug,
                                           spec.decay_drug, spec.bnd_drug, spec.S_drug, code, step=k, field=1,
                                           encoding=e_dr)
        fsnap = dict(snap)
        fsnap["fields"] = {"o2": oracle.from_bits16(o2_bits, code, e_o2, spec.bnd_o2).ravel(),
                           "drug": oracle.from_bits16(dr_bits, code, e_dr, spec.bnd_drug).ravel()}
        fsnap["sinks"] = {"o2": np.zeros(int(np.prod(shp)), np.float32)}
        orc = oracle.TumourOracle.from_snapshot(spec, fsnap, spec.capacity)
        orc.agents_part(nthreads=4)
        eng.run_step()
        got = be.snapshot()
        np.testing.assert_array_equal(got["fields"]["o2"], o2_bits.ravel(), err_msg=f"o2 bits step {step}")
        np.testing.assert_array_equal(got["residuals"]["o2"], o2_res.ravel(), err_msg=f"o2 residual step {step}")
        np.testing.assert_array_equal(got["fields"]["drug"], dr_bits.ravel(), err_msg=f"drug bits step {step}")
        np.testing.assert_array_equal(got["residuals"]["drug"], dr_res.ravel())
        n = got["rows"]
        assert n == orc.rows, step
        np.testing.assert_array_equal(got["life"], orc.dead[:n])
        for col, key in (("state", "state"), ("_rng_state", "rng"), ("volume", "volume"), ("radius", "radius")):
            np.testing.assert_array_equal(got["cols"][col], orc.bufs[key][:n], err_msg=f"{col} step {step}")
        for a, key in (("pos.x", "x"), ("pos.y", "y"), ("pos.z", "z")):
            np.testing.assert_allclose(got["cols"][a], orc.bufs[key][:n], rtol=0, atol=1e-4)
        np.testing.assert_array_equal(got["sinks"]["o2"], orc.o2_sink.ravel())


def test_queued_readbacks_match_waiting_steps(cuda):
    """Steps whose metrics are read one step late (run_step(collect_metrics=True,
    wait=False), the next step queued before the previous result is taken)
    give every step's metrics and counters exactly as waiting steps do, with
    a parameter changed before each step (the pinned upload ring keeps each
    upload's bytes until its copy ran); both engines end in the same state."""
    from oncolytica_b200 import _lib

    spec = W.scaled(_parity_spec(), n_agents=5000)
    a, b = W.build_engine(spec), W.build_engine(spec)
    for eng in (a, b):
        eng.set_graphs(True)
    want, got, pend = [], [], None
    for step in range(12):
        growth = 0.05 + 0.01 * (step % 5)
        a.update_params(growth=growth)
        a.run_step(collect_metrics=True)
        want.append((metric_fields_values(a.get_metrics()), a._backend_impl.counters()["agent_steps"]))
        b.update_params(growth=growth)
        h = b.run_step(collect_metrics=True, wait=False)
        assert h is not None
        if pend is not None:
            got.append((pend.result(), pend.counters["agent_steps"]))
        pend = h
    got.append((pend.result(), pend.counters["agent_steps"]))
    assert got == want
    assert metric_fields_values(b.get_metrics()) == want[-1][0]
    sa, sb = a._backend_impl.snapshot(), b._backend_impl.snapshot()
    assert sa["rows"] == sb["rows"]
    for k in ("o2", "drug"):
        np.testing.assert_array_equal(sa["fields"][k], sb["fields"][k])

    # a ticket whose slot a later queue reused is refused, not misread
    be = b._backend_impl
    import ctypes as C

    tickets = []
    for _ in range(_lib.READBACK_SLOTS + 1):
        t = C.c_uint64()
        assert be.lib.olc_queue_readback(be.handle, be._stream(), C.byref(t)) == _lib.OLC_OK
        tickets.append(t.value)
    c = _lib.OlcCounters()
    assert be.lib.olc_take_readback(be.handle, tickets[0], None, 0, C.byref(c)) == _lib.OLC_ERR_STATE
    assert be.lib.olc_take_readback(be.handle, tickets[-1], None, 0, C.byref(c)) == _lib.OLC_OK
    assert c.status == 0 and c.agent_steps == want[-1][1]
    a.close()
    b.close()


def metric_fields_values(m) -> dict:
    return {k: int(getattr(m, k)) for k in metric_fields(type(m))}
