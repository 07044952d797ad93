"""A model with tissue and chemistry rules (the DSL surface of the
reference's GBM example, framework/examples/gbm_model.py: a chemistry rule
over voxel neighbours and the agents of the voxel, a tissue rule counting its
agents), shared by the translator test (CPU) and the parity test (GPU)."""
from __future__ import annotations

import oncolytica_b200 as ol

SECRETE: ol.f32 = 0.4
CONSUME: ol.f32 = 0.04
D_PDGF: ol.f32 = 0.02
DECAY: ol.f32 = 0.995
KIND_ACTIVE: ol.i32 = 1


class VTissue(ol.Tissue):
    density: ol.f32 = 0.0
    crowded: ol.i32 = 0
    capacity: ol.i32 = 3

    def is_crowded(self, n: ol.i32) -> ol.bool:
        return n >= self.capacity


class VChem(ol.Chemistry):
    pdgf: ol.f32 = 0.0
    glu: ol.f32 = 1.0

    def laplacian(self) -> ol.f32:
        lap: ol.f32 = 0.0
        for nb in self.neighbors:
            lap += nb.pdgf - self.pdgf
        return lap

    def source(self) -> tuple[ol.f32, ol.f32]:
        # seeded from a field so that the CPU interpreter sums in float32 too
        sec: ol.f32 = self.pdgf * 0.0
        con: ol.f32 = self.pdgf * 0.0
        for c in self.cells:
            if c.kind == KIND_ACTIVE:
                sec += SECRETE
            con += CONSUME
        return sec, con

    def tissue_load(self) -> ol.f32:
        d: ol.f32 = 0.0
        for t in self.tissues:
            d += t.density
        return d

    def step_pdgf(self):
        sec, con = self.source()
        lap: ol.f32 = self.laplacian()
        new_val: ol.f32 = (self.pdgf + sec - con + D_PDGF * lap) * DECAY
        self.pdgf = ol.math.clamp(new_val, 0.0, 1000.0)
        self.glu = self.glu - 0.001 * self.tissue_load()


class VCell(ol.Cell):
    pos: ol.vec3
    kind: ol.i32 = 0
    energy: ol.f32 = 1.0


class VMetrics(ol.Metrics):
    active: ol.i32 = 0


class VParams(ol.Params):
    gain: ol.f32 = 0.1


class VoxelSim(ol.Simulation[VTissue, VChem, VCell, VMetrics, VParams]):

    @ol.tissue_rule
    def census(self, t: VTissue):
        d: ol.f32 = 0.0
        for c in t.cells:
            d += 1.0
        t.density = d
        n: ol.i32 = 0
        for nb in t.neighbors:
            if nb.density > 2.0:
                n += 1
        t.crowded = 1 if t.is_crowded(n) else 0

    @ol.chemistry_rule(iterations=2)
    def pdgf(self, chem: VChem):
        chem.step_pdgf()

    @ol.cell_rule
    def live(self, cell: VCell):
        chem: VChem = self.chemistry_at(cell.pos)
        tis: VTissue = self.tissue_at(cell.pos)
        cell.energy = cell.energy + chem.pdgf * self.params.gain - tis.density * 0.01
        if chem.pdgf > 0.5 and tis.crowded == 0:
            cell.kind = KIND_ACTIVE

    @ol.metric_rule
    def count(self, cell: VCell, m: VMetrics):
        if cell.kind == KIND_ACTIVE:
            m.active += 1
