"""A model whose chemistry rule runs in batched and served mode: the voxel's
Moore-neighbour Laplacian, secretion by the agents of its 2 x 2 x 2 tissue
voxels (.cells, the reference's tied grids) and decay, three iterations per
step; a cell rule that reads the field back, grows, divides and dies (after
the reference's GBM example, framework/examples/gbm_model.py)."""
import oncolytica_b200 as ol

SECRETE: ol.f32 = 0.25
D_F: ol.f32 = 0.05


class CTissue(ol.Tissue):
    pass


class CChem(ol.Chemistry):
    signal: ol.f32 = 0.0

    def laplacian(self) -> ol.f32:
        lap: ol.f32 = 0.0
        for nb in self.neighbors:
            lap += nb.signal - self.signal
        return lap

    def secretion(self) -> ol.f32:
        s: ol.f32 = self.signal * 0.0
        for c in self.cells:
            if c.kind == 1:
                s += SECRETE
        return s


class CCell(ol.Cell):
    pos: ol.vec3
    kind: ol.i32 = 0
    energy: ol.f32 = 0.5


class CMetrics(ol.Metrics):
    n: ol.i32 = 0


class CParams(ol.Params):
    pass


class ChemSim(ol.Simulation[CTissue, CChem, CCell, CMetrics, CParams]):
    @ol.chemistry_rule(iterations=3)
    def spread(self, chem: CChem):
        chem.signal = (chem.signal + D_F * chem.laplacian() + chem.secretion()) * 0.98

    @ol.cell_rule
    def respond(self, cell: CCell):
        chem: CChem = self.chemistry_at(cell.pos)
        cell.energy += chem.signal * 0.01
        if cell.energy > 1.0:
            cell.energy = cell.energy * 0.5
            cell.divide(CCell(pos=cell.pos + ol.vec3(0.5, 0.25, 0.0), kind=1 - cell.kind, energy=cell.energy))
        elif cell.energy < 0.05:
            cell.die()

    @ol.metric_rule
    def count(self, cell: CCell, m: CMetrics):
        m.n += 1
