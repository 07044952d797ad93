"""A cell-rule model whose decisions are pinned against the reference's own
CPU backend (tests/golden/make_cpu_rules_golden.py runs this file's text with
its import line pointed at the reference package and records every step;
tests/test_gpu_pinned_rules.py runs it here).  It reads a static chemistry
field and a tissue column through chemistry_at / tissue_at, counts ages,
switches kinds, dies and divides with keyword constructors, and keeps a float
energy whose decisions stay far from their thresholds (so FP32 here and
Python's doubles there decide alike).  It has no neighbour loops (the
reference CPU updates agents in place, so its neighbour reads would see this
step's values), no random draws (the reference CPU's random() is Python's
generator) and no divide(): the reference CPU's agent list hands agents
appended during a rule pass to that same pass (AgentList.__iter__ walks the
growing list), while the reference GPU path, which this package follows, runs
children from the next step; births are pinned by the reference's divide test
instead (tests/golden/make_golden.py)."""
import oncolytica_b200 as ol

KIND_A: ol.i32 = 0
KIND_B: ol.i32 = 1


class PTissue(ol.Tissue):
    stiff: ol.i32 = 0


class PChem(ol.Chemistry):
    nutrient: ol.f32 = 0.0


class PCell(ol.Cell):
    pos: ol.vec3
    uid: ol.i32 = 0
    age: ol.i32 = 0
    kind: ol.i32 = 0
    energy: ol.f32 = 1.0


class PMetrics(ol.Metrics):
    n: ol.i32 = 0
    n_b: ol.i32 = 0
    age_sum: ol.i32 = 0


class PParams(ol.Params):
    pass


class PinnedSim(ol.Simulation[PTissue, PChem, PCell, PMetrics, PParams]):
    @ol.cell_rule
    def live(self, cell: PCell):
        chem: PChem = self.chemistry_at(cell.pos)
        t: PTissue = self.tissue_at(cell.pos)
        cell.age += 1
        cell.energy = cell.energy * 0.75 + chem.nutrient * 0.25
        if t.stiff > 0 and cell.age % 4 == 0:
            cell.kind = 1 - cell.kind
        if cell.energy < 0.3 and cell.age > 2:
            cell.die()
            return
        if cell.kind == KIND_A and cell.age % 3 == 0:
            cell.energy = cell.energy * 0.5 + 0.125

    @ol.metric_rule
    def census(self, cell: PCell, m: PMetrics):
        m.n += 1
        m.age_sum += cell.age
        if cell.kind == KIND_B:
            m.n_b += 1
