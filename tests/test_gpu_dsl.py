"""Rule-translator parity on the GPU: the CUDA kernels NVRTC builds from a
model's rules against the rule interpreter (oracle/dsl_interp.py) running the
same Python rules, step by step from identical device snapshots.  Integer
columns, RNG states, life flags, children counts and every float that is
computed with + - * / sqrt are bit-exact; positions placed with cos/sin get
1e-4."""
from __future__ import annotations

import numpy as np
import pytest

import oncolytica_b200 as ol
from test_translator import GCell, GChem, GSim, GTissue

pytestmark = pytest.mark.gpu


def _compare(got, ref, float_exact=(), float_tol=(), tol=1e-4):
    assert got["rows"] == ref["rows"]
    n = got["rows"]
    np.testing.assert_array_equal(got["life"], ref["life"][:n])
    for col, a in got["cols"].items():
        b = ref["cols"][col][:n]
        if a.dtype.kind in "iu":
            np.testing.assert_array_equal(a, b, err_msg=col)
        elif col in float_tol:
            np.testing.assert_allclose(a, b, rtol=0, atol=tol, err_msg=col)
        else:
            np.testing.assert_array_equal(a, b, err_msg=col)


def test_rich_model_matches_interpreter(cuda):
    import dsl_interp

    rng = np.random.default_rng(21)
    eng = ol.Engine(backend="cuda", max_agents=20_000)
    eng.setup_geometry((20, 20, 20), 2.0)
    eng.setup_tissue(GTissue)
    eng.tissue.column("capacity")[...] = rng.integers(2, 12, size=eng.tissue_shape)
    eng.setup_chemistry(GChem)
    eng.chemistry.column("pdgf")[...] = rng.uniform(0, 300, size=eng.chemistry_shape).astype(np.float32)
    n = 1500
    pos = rng.uniform(0.0, 40.0, size=(n, 3)).astype(np.float32)
    eng.cells.add_arrays(GCell, pos=pos, kind=rng.integers(0, 2, n), clock=rng.uniform(0.5, 1.0, n),
                         p_pot=rng.uniform(0.0, 60.0, n))
    eng.load_model(GSim())
    be = eng._backend_impl
    total_births = 0
    for step in range(4):
        snap = be.snapshot()
        it = dsl_interp.Interpreter(eng._sim, dsl_interp.engine_cfg(eng), snap)
        ref = dsl_interp.step(it, eng, collect=True)
        eng.run_step(collect_metrics=True)
        got = be.snapshot()
        _compare(got, it.snapshot(), float_tol=("pos.x", "pos.y", "pos.z"))
        m = eng.get_metrics()
        assert m.count == ref["metrics"]["count"]
        assert abs(float(m.total) - float(ref["metrics"]["total"])) <= 1e-4 * max(1.0, abs(float(m.total)))
        total_births += ref["births"]
    assert total_births > 0


class MCell(ol.Cell):
    pos: ol.vec3
    age: ol.i32 = 0
    tag: ol.f32 = 0.0


class MChem(ol.Chemistry):
    c: ol.f32 = 0.0


class MTissue(ol.Tissue):
    pass


class MMetrics(ol.Metrics):
    n: ol.i32 = 0


class MParams(ol.Params):
    pass


class TwoRuleSim(ol.Simulation[MTissue, MChem, MCell, MMetrics, MParams]):
    @ol.cell_rule
    def a_first(self, cell: MCell):
        cell.age += 1
        if cell.age % 3 == 0:
            cell.die()
            return
        if cell.age % 2 == 0:
            cell.divide(MCell(pos=cell.pos, age=100))

    @ol.cell_rule
    def b_second(self, cell: MCell):
        cell.tag += 1.0
        if cell.age == 4:
            cell.divide(MCell(pos=cell.pos + ol.vec3(0.5), age=200))

    @ol.metric_rule
    def count(self, cell: MCell, m: MMetrics):
        m.n += 1


def test_two_rules_deaths_and_children_match_interpreter(cuda):
    import dsl_interp

    rng = np.random.default_rng(5)
    eng = ol.Engine(backend="cuda", max_agents=50_000)
    eng.setup_geometry((16, 16, 16), 1.0)
    n = 3000
    eng.cells.add_arrays(MCell, pos=rng.uniform(0, 16, size=(n, 3)), age=rng.integers(0, 6, n))
    eng.load_model(TwoRuleSim())
    be = eng._backend_impl
    for _ in range(5):
        snap = be.snapshot()
        it = dsl_interp.Interpreter(eng._sim, dsl_interp.engine_cfg(eng), snap)
        ref = dsl_interp.step(it, eng, collect=True)
        eng.run_step(collect_metrics=True)
        _compare(be.snapshot(), it.snapshot())
        assert eng.get_metrics().n == ref["metrics"]["n"]


def test_capacity_overflow_sets_status_and_drops_children(cuda):
    eng = ol.Engine(backend="cuda", max_agents=120)
    eng.setup_geometry((8, 8, 8), 1.0)
    eng.cells.add_arrays(MCell, pos=np.full((100, 3), 4.0), age=np.ones(100, np.int32))
    eng.load_model(TwoRuleSim())
    eng.run_step()  # every agent turns 2 and divides once: 100 children, room for 20
    c = eng._backend_impl.counters()
    assert c["n_agents"] == 120
    assert c["status"] & 0x1
