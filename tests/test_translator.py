"""The rule translator on CPU: rules translate to CUDA C that NVRTC compiles
for sm_100a (no GPU needed), and unsupported constructs raise
CompilationError with the offending line."""
from __future__ import annotations

import ctypes as C
from types import SimpleNamespace

import pytest

import oncolytica_b200 as ol
from oncolytica_b200 import _lib
from oncolytica_b200 import workloads as W
from oncolytica_b200.compiler.emit_cuda import make_layout, pack_params, translate_model


def _translate(sim_cls, radius=None):
    sim = sim_cls()
    rules = {"cell": [], "metric": []}
    for name in dir(sim):
        m = getattr(sim, name, None)
        kind = getattr(m, "_rule_type", None)
        if kind in rules:
            rules[kind].append(m)
    sim._engine = SimpleNamespace(_cell_rules=rules["cell"], _metric_rules=rules["metric"])
    layout = make_layout(sim._spec, radius)
    return translate_model(sim, layout, radius)


def _nvrtc_ok(prog):
    log = C.create_string_buffer(1 << 16)
    rc = _lib.load().olc_nvrtc_check(prog.source.encode(), _lib.CSRC_DIR.encode(), log, len(log))
    assert rc == 0, log.value.decode()[:3000]


def test_tumour_models_compile():
    for cls in (W.TumourSim, W.TumourDrugSim):
        prog = _translate(cls, "radius")
        assert [k for k, _ in prog.kernels] == ["Kernel_CellRule_0", "Kernel_MetricRule_0"]
        # a solo handle's metric rule adds into per-block shared words
        assert f"#define OLC_SOLO_METRIC_WORDS {len(prog.layout.metrics)}\n" in prog.source and "olc_s_metrics[k] = 0u" in prog.source
        assert prog.sink_fields == {"o2"}
        _nvrtc_ok(prog)


# ---- a model exercising helpers, tuples, neighbours, loops and casts ----

K_HILL: ol.f32 = 100.0
TYPE_A: ol.i32 = 1


class GTissue(ol.Tissue):
    capacity: ol.i32 = 10

    def crowded(self, n: ol.i32) -> ol.bool:
        return n >= self.capacity


class GChem(ol.Chemistry):
    pdgf: ol.f32 = 0.0


class GCell(ol.Cell):
    pos: ol.vec3
    kind: ol.i32 = 0
    clock: ol.f32 = 0.0
    moving: ol.bool = False
    p_pot: ol.f32 = 0.025

    def gamma(self, c: ol.f32) -> ol.f32:
        return c / (c + K_HILL)

    def phenotype(self, c: ol.f32, am: ol.bool) -> tuple[ol.f32, ol.f32]:
        g: ol.f32 = self.gamma(c)
        p: ol.f32 = self.p_pot * g
        m: ol.f32 = p * (0.1 if am else 1.0)
        return p, m

    def tick(self, p: ol.f32):
        self.clock += p
        if self.clock >= 1.0:
            self.clock -= 1.0
            self.spawn()

    def spawn(self):
        angle: ol.f32 = ol.random() * 6.2831853
        child: GCell = GCell(pos=self.pos + ol.vec3(ol.math.cos(angle), ol.math.sin(angle), 0.0), kind=self.kind)
        self.divide(child)


class GMetrics(ol.Metrics):
    count: ol.i32 = 0
    total: ol.f32 = 0.0


class GParams(ol.Params):
    am: ol.bool = False
    scale: ol.f32 = 2.0


class GSim(ol.Simulation[GTissue, GChem, GCell, GMetrics, GParams]):
    def clamp01(self, v: ol.f32) -> ol.f32:
        return ol.math.clamp(v, 0.0, 1.0)

    @ol.cell_rule
    def behave(self, cell: GCell):
        chem: GChem = self.chemistry_at(cell.pos)
        tissue: GTissue = self.tissue_at(cell.pos)
        p, m = cell.phenotype(chem.pdgf, self.params.am)
        active: ol.i32 = 0
        for nb in cell.neighbors:
            if nb.kind != 0:
                active += 1
            if active > 20:
                break
        total: ol.f32 = 0.0
        for i in range(3):
            total += float(i) * 0.5
        if not tissue.crowded(active):
            cell.tick(self.clamp01(p * self.params.scale + total))
        cell.moving = not cell.moving
        if cell.moving and m > 0.0:
            cell.pos.x = ol.math.clamp(cell.pos.x + m, 0.0, 100.0)
        q = 7 // 2 + 7 % 3
        if q == 5 and cell.kind == TYPE_A and chem.pdgf < -1.0:
            cell.die()

    @ol.metric_rule
    def collect(self, cell: GCell, mt: GMetrics):
        mt.count += 1
        mt.total += cell.clock


def test_rich_model_compiles():
    prog = _translate(GSim)
    src = prog.source
    assert "cell_phenotype" in src and "gtissue" not in src.lower().replace("tissue_t", "")
    assert "Tup_f32_f32" in src
    assert "olc_tissue_key" in src  # neighbour loop
    _nvrtc_ok(prog)


def test_params_blob_layout():
    prog = _translate(GSim)
    blob = pack_params(prog.layout, GParams(am=True, scale=3.0))
    assert len(blob) == 8
    import numpy as np

    assert np.frombuffer(blob[:4], np.int32)[0] == 1  # "am" sorts first
    assert np.frombuffer(blob[4:], np.float32)[0] == np.float32(3.0)


# ---- errors ----------------------------------------------------------------

class ECell(ol.Cell):
    pos: ol.vec3
    n: ol.i32 = 0


class EMetrics(ol.Metrics):
    c: ol.i32 = 0


class EParams(ol.Params):
    pass


def _err_sim(body):
    ns = {}
    src = ("class S(ol.Simulation[GTissue, GChem, ECell, EMetrics, EParams]):\n"
           "    @ol.cell_rule\n"
           "    def rule(self, cell: ECell):\n" + "".join("        " + line + "\n" for line in body.splitlines()))
    import linecache

    fname = f"<err-model-{abs(hash(src))}>"
    linecache.cache[fname] = (len(src), None, src.splitlines(True), fname)
    exec(compile(src, fname, "exec"), {**globals(), "ol": ol}, ns)
    return ns["S"]


@pytest.mark.parametrize("body,msg", [
    ("cell.n = 1.5", "float -> int"),
    ("x = undefined_name + 1", "unknown name"),
    ("for c in self.cells:\n    pass", ""),
    ("cell.n = len([1])", ""),
    ("with open('f') as f:\n    pass", "unsupported statement"),
])
def test_unsupported_constructs_raise(body, msg):
    with pytest.raises(ol.CompilationError, match=msg):
        _translate(_err_sim(body))


def test_batched_translation_compiles():
    """Batched mode adds a `_sim` column after `_rng_state`, gives rule bodies
    a per-simulation view and still compiles for sm_100a."""
    for cls, radius in ((W.TumourDrugSim, "radius"), (GSim, None)):
        sim = cls()
        rules = {"cell": [], "metric": []}
        for name in dir(sim):
            m = getattr(sim, name, None)
            kind = getattr(m, "_rule_type", None)
            if kind in rules:
                rules[kind].append(m)
        sim._engine = SimpleNamespace(_cell_rules=rules["cell"], _metric_rules=rules["metric"])
        layout = make_layout(sim._spec, radius, batched=True)
        assert [c for c, _, _ in layout.cell_cols][-2:] == ["_rng_state", "_sim"]
        assert layout.cell_cols[layout.rng_col][0] == "_rng_state"
        prog = translate_model(sim, layout, radius)
        assert "typedef OlcSimView OlcP;" in prog.source
        assert "OLC_SOLO_METRIC_WORDS" not in prog.source
        assert "olc_sim_view(P, sim)" in prog.source
        _nvrtc_ok(prog)


# ---- tissue and chemistry rules ---------------------------------------------

def _translate_all(sim_cls, tissue_shape=(12, 12, 12), vs=10.0, chem_shape=None, chem_vs=None, batched=False):
    sim = sim_cls()
    rules = {"cell": [], "metric": [], "tissue": [], "chemistry": []}
    for name in dir(sim):
        m = getattr(sim, name, None)
        kind = getattr(m, "_rule_type", None)
        if kind in rules:
            rules[kind].append(m)
    sim._engine = SimpleNamespace(_cell_rules=rules["cell"], _metric_rules=rules["metric"],
                                  _tissue_rules=rules["tissue"], _chemistry_rules=rules["chemistry"],
                                  tissue_shape=tissue_shape, tissue_voxel_size=vs,
                                  chemistry_shape=chem_shape or tuple(t // 2 for t in tissue_shape),
                                  chemistry_voxel_size=chem_vs or 2.0 * vs)
    return translate_model(sim, make_layout(sim._spec, None, batched=batched), None)


def test_batched_chemistry_rules_compile():
    """Chemistry rules in batched mode: one kernel over the batch's field
    tiles, each member through its own view; tissue rules and .tissues loops
    are refused there (members have no tissue grids)."""
    import chem_model as CM
    import voxel_model as VM

    prog = _translate_all(CM.ChemSim, batched=True)
    assert dict(prog.kernels)["Kernel_ChemRule_0"] == 3
    assert "olc_sim_view(P, t.x)" in prog.source and "P.vtiles" in prog.source
    _nvrtc_ok(prog)
    with pytest.raises(ol.CompilationError, match="tissue"):
        _translate_all(VM.VoxelSim, batched=True)


def test_voxel_rules_compile():
    import voxel_model as VM

    prog = _translate_all(VM.VoxelSim)
    kinds = dict(prog.kernels)
    assert kinds["Kernel_TissueRule_0"] == 2 and kinds["Kernel_ChemRule_0"] == 3
    assert prog.iterations[[k for k, _ in prog.kernels].index("Kernel_ChemRule_0")] == 2
    src = prog.source
    assert "olc_store_tissue" in src and "olc_store_chem" in src and "olc_chem_voxel" in src
    _nvrtc_ok(prog)


def test_chemistry_cells_need_the_tied_grids():
    import voxel_model as VM

    with pytest.raises(ol.CompilationError, match="tied"):
        _translate_all(VM.VoxelSim, chem_shape=(8, 8, 8), chem_vs=15.0)


class RTissue(ol.Tissue):
    a: ol.f32 = 0.0


class RandSim(ol.Simulation[RTissue, GChem, GCell, GMetrics, GParams]):
    @ol.tissue_rule
    def noisy(self, t: RTissue):
        t.a = ol.random()


def test_voxel_rules_have_no_rng():
    with pytest.raises(ol.CompilationError, match="no RNG state"):
        _translate_all(RandSim, tissue_shape=(20, 20, 20), vs=2.0)


def test_vessel_voxels_are_the_cylinder():
    import numpy as np

    eng = ol.Engine(backend="cuda", max_agents=16)
    eng.setup_geometry((20, 20, 20), 5.0)  # chemistry 10^3 voxels of 10 um
    eng.setup_vessel(center=(42.0, 57.0), radius=12.0)
    idx = eng.vessel_voxels()
    nx, ny, nz = eng.chemistry_shape
    want = [(z * ny + y) * nx + x for z in range(1, nz - 1) for y in range(1, ny - 1) for x in range(1, nx - 1)
            if (x * 10.0 + 5.0 - 42.0) ** 2 + (z * 10.0 + 5.0 - 57.0) ** 2 <= 144.0]
    assert idx.tolist() == sorted(want) and len(want) > 0
    assert idx.dtype == np.uint32
    # a vessel across a corner of the grid: its face voxels stay Dirichlet
    eng.setup_vessel(center=(5.0, 5.0), radius=25.0)
    v = eng.vessel_voxels().astype(np.int64)
    x, y, z = v % nx, v // nx % ny, v // (nx * ny)
    assert len(v) > 0 and x.min() == 1 and z.min() == 1 and y.min() == 1 and y.max() == ny - 2


from conftest import REFERENCE  # noqa: E402

_REFERENCE_GBM = __import__("os").path.join(REFERENCE, "framework", "examples", "gbm_model.py")


@pytest.mark.skipif(not __import__("os").path.exists(_REFERENCE_GBM), reason="no reference checkout here")
def test_reference_gbm_example_translates(tmp_path, monkeypatch):
    """The reference's own example model (framework/examples/gbm_model.py),
    with only its import line pointed at this package: its set-up runs through
    this Engine's API (setup_geometry keywords, tissue/chemistry sample(),
    cells.add), and its chemistry rule (helper methods looping over .cells and
    .neighbors, tuple returns), cell rule (neighbours, divide with keyword
    constructor, die, log/atan2/cos/sin) and metric rule translate to kernels
    that NVRTC compiles.  Read from the reference checkout when it is present;
    the model is not part of this repository."""
    import importlib
    import random
    import sys

    src = open(_REFERENCE_GBM, encoding="utf-8").read()
    assert "import oncolytica as ol" in src
    (tmp_path / "ref_gbm_model.py").write_text(src.replace("import oncolytica as ol", "import oncolytica_b200 as ol"))
    monkeypatch.syspath_prepend(str(tmp_path))
    G = importlib.import_module("ref_gbm_model")
    try:
        random.seed(42)
        eng = ol.Engine(backend="cuda")
        eng.setup_geometry(tissue_shape=(40, 40, 2), tissue_voxel_size=15.0, cell_diameter=10.0)
        eng.setup_tissue(G.BrainTissue)
        eng.setup_chemistry(G.BrainChem)
        G._init_tissue(eng)
        G._init_chemistry(eng)
        G._init_cells(eng)
        assert len(eng.cells) == 100 and tuple(eng.chemistry_shape) == (20, 20, 1)
        prog = _translate_all(G.MultiscaleGBM, tissue_shape=(40, 40, 2), vs=15.0)
        assert sorted(k for k, _ in prog.kernels) == ["Kernel_CellRule_0", "Kernel_ChemRule_0", "Kernel_MetricRule_0"]
        _nvrtc_ok(prog)
    finally:
        sys.modules.pop("ref_gbm_model", None)
