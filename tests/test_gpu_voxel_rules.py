"""Tissue and chemistry rules on the GPU (Kernel_TissueRule_i /
Kernel_ChemRule_i from the translator) against the rule interpreter
(oracle/dsl_interp.py) running the same Python rules, step by step from
identical device snapshots: counts, crowding flags and agent kinds exact;
field and energy values to 1e-6 relative (the interpreter sums some Python
float locals in double where the kernels sum in FP32)."""
from __future__ import annotations

import numpy as np
import pytest

import oncolytica_b200 as ol
import voxel_model as VM

pytestmark = pytest.mark.gpu


def _engine(seed=3, n=2000):
    rng = np.random.default_rng(seed)
    eng = ol.Engine(backend="cuda", max_agents=20_000)
    eng.setup_geometry((12, 12, 12), 10.0)  # chemistry tied: 6^3 voxels of 20 um
    eng.setup_tissue(VM.VTissue)
    eng.tissue.column("capacity")[...] = rng.integers(1, 5, size=eng.tissue_shape)
    eng.setup_chemistry(VM.VChem)
    eng.chemistry.column("pdgf")[...] = rng.uniform(0.0, 1.0, size=eng.chemistry_shape).astype(np.float32)
    eng.chemistry.column("glu")[...] = 1.0
    # a dense corner so that some bins hold more than two agents
    pos = np.concatenate([rng.uniform(0.0, 120.0, size=(n, 3)), rng.uniform(20.0, 40.0, size=(n // 2, 3))])
    eng.cells.add_arrays(VM.VCell, pos=pos.astype(np.float32), kind=rng.integers(0, 2, len(pos)))
    eng.load_model(VM.VoxelSim())
    return eng


def test_voxel_rules_match_interpreter(cuda):
    import dsl_interp

    eng = _engine()
    be = eng._backend_impl
    kinds = [k for _, k in be.program.kernels]
    assert 2 in kinds and 3 in kinds
    crowded_seen = 0
    for step in range(3):
        snap = be.snapshot()
        it = dsl_interp.Interpreter(eng._sim, dsl_interp.engine_cfg(eng), snap)
        ref = dsl_interp.step(it, eng, collect=True)
        eng.run_step(collect_metrics=True)
        got = be.snapshot()
        exp = it.snapshot()
        assert got["rows"] == exp["rows"]
        n = got["rows"]
        np.testing.assert_array_equal(got["cols"]["kind"], exp["cols"]["kind"][:n])
        for a in ("pos.x", "pos.y", "pos.z"):
            np.testing.assert_array_equal(got["cols"][a], exp["cols"][a][:n])
        np.testing.assert_allclose(got["cols"]["energy"], exp["cols"]["energy"][:n], rtol=1e-6, atol=1e-6)
        for f in ("pdgf", "glu"):
            np.testing.assert_allclose(got["fields"][f], exp["fields"][f], rtol=1e-6, atol=1e-6, err_msg=f)
        for k in ("density", "crowded", "capacity"):
            np.testing.assert_array_equal(got["tissue"][k], exp["tissue"][k], err_msg=k)
        assert eng.get_metrics().active == ref["metrics"]["active"]
        crowded_seen += int(got["tissue"]["crowded"].sum())
    assert crowded_seen > 0, "the case should exercise the crowding branch"
    # the host grids follow the device after sync_to_host
    eng.sync_to_host()
    np.testing.assert_array_equal(np.asarray(eng.tissue.column("density")), got["tissue"]["density"])


def test_voxel_rules_with_graphs_match_eager(cuda):
    a, b = _engine(seed=7), _engine(seed=7)
    b.set_graphs(True)
    a.run_steps(4)
    b.run_steps(4)
    sa, sb = a._backend_impl.snapshot(), b._backend_impl.snapshot()
    for k in sa["cols"]:
        np.testing.assert_array_equal(sa["cols"][k], sb["cols"][k], err_msg=k)
    for k in sa["fields"]:
        np.testing.assert_array_equal(sa["fields"][k], sb["fields"][k], err_msg=k)
    for k in sa["tissue"]:
        np.testing.assert_array_equal(sa["tissue"][k], sb["tissue"][k], err_msg=k)


class ItTissue(ol.Tissue):
    pass


class ItChem(ol.Chemistry):
    drug_conc: ol.f32 = 0.0


class ItCell(ol.Cell):
    pos: ol.vec3


class ItMetrics(ol.Metrics):
    pass


class ItParams(ol.Params):
    pass


class ItChemSim(ol.Simulation[ItTissue, ItChem, ItCell, ItMetrics, ItParams]):
    @ol.chemistry_rule(iterations=3)
    def diffuse(self, chem: ItChem):
        chem.drug_conc += 1.0  # runs 3 times per step


@pytest.mark.parametrize("tissue_shape", [(2, 2, 2), (16, 12, 8)])
def test_chemistry_rule_iterations_add_three_per_step(cuda, tissue_shape):
    """The reference's framework/tests/test_oncolytica.py:407-435 on the CUDA
    path: @chemistry_rule(iterations=3) adding 1.0 runs three times per step,
    so every chemistry voxel holds 3.0 after one step (and 6.0 after two)."""
    eng = ol.Engine(backend="cuda", max_agents=64)
    eng.setup_geometry(tissue_shape=tissue_shape)
    eng.load_model(ItChemSim())
    eng.chemistry.column("drug_conc")[...] = 0.0
    eng.sync_to_device()
    eng.run_step()
    eng.sync_to_host()
    vals = np.asarray(eng.chemistry.column("drug_conc"))
    assert vals.size == int(np.prod(eng.chemistry_shape)) and vals.size >= 1
    np.testing.assert_array_equal(vals, np.full(vals.shape, 3.0, np.float32))
    eng.run_step()
    eng.sync_to_host()
    np.testing.assert_array_equal(np.asarray(eng.chemistry.column("drug_conc")), 6.0)
