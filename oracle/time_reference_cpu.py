"""Times the reference's own CPU backend (CPUBackend, pure Python, one core)
on the plain workload expressed in the reference's rule DSL, and writes
oracle/reference_cpu_backend.json, which bench.py reports beside the C
oracle's timing.

This is a CPU baseline only (test infrastructure, like the rest of oracle/):
it runs where a checkout of the reference exists, because the reference does
not travel with this repository:

    python oracle/time_reference_cpu.py [/path/to/reference]

The reference path: the first argument, else $OLC_REFERENCE, else a directory
named "reference" beside this repository.

The model follows the plain workload's rule (workloads.TumourSim): divide
above twice the volume if O2 > 0.3, quiescent if 0.1 < O2 <= 0.3, necrotic if
O2 <= 0.1, volume growth 0.05/h; the reference has no built-in diffusion, so
O2 diffuses through its chemistry-rule mechanism (framework/src/oncolytica/cpu/
_decorators.py:33-39, CPUBackend.run_step's iterations loop,
framework/src/oncolytica/cpu/_cpu_backend.py:58-63): one chemistry-rule call
per voxel and iteration, over the voxel's Moore neighbours and its cells for
the uptake.  The reference ties its chemistry grid to half the tissue grid, so
the agent phase and one chemistry iteration are timed separately and the
plain workload's step (10,000 agents, 80 iterations over 64^3 voxels) is
extrapolated from them; the JSON says so.
"""
from __future__ import annotations

import json
import os
import platform
import random
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REF = (sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OLC_REFERENCE")
       or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
sys.path.insert(0, os.path.join(REF, "framework", "src"))

import oncolytica as ol  # noqa: E402  (the reference package)

PROLIF, QUIESC, NECROTIC = 1, 2, 3


class RTissue(ol.Tissue):
    pass


class RChem(ol.Chemistry):
    o2: ol.f32 = 1.0

    def uptake(self) -> ol.f32:
        u: ol.f32 = 0.0
        for c in self.cells:
            if c.state != 3:
                u += 0.02
        return u

    def laplacian(self) -> ol.f32:
        lap: ol.f32 = 0.0
        for nb in self.neighbors:
            lap += nb.o2 - self.o2
        return lap


class RCell(ol.Cell):
    pos: ol.vec3
    radius: ol.f32 = 5.0
    volume: ol.f32 = 1.0
    state: ol.i32 = 1


class RMetrics(ol.Metrics):
    live: ol.i32 = 0


class RParams(ol.Params):
    pass


class CellsOnly(ol.Simulation[RTissue, RChem, RCell, RMetrics, RParams]):
    @ol.cell_rule
    def cycle(self, cell: RCell):
        chem: RChem = self.chemistry_at(cell.pos)
        if cell.state == 3:
            return
        o2: ol.f32 = chem.o2
        if o2 <= 0.1:
            cell.state = 3
            return
        if o2 <= 0.3:
            cell.state = 2
            return
        cell.state = 1
        cell.volume += 0.05 * cell.volume * 0.1
        if cell.volume > 2.0:
            half: ol.f32 = cell.volume * 0.5
            cell.volume = half
            d: ol.vec3 = ol.random_dir()
            off: ol.vec3 = d * (cell.radius * 0.5)
            child: RCell = RCell(pos=cell.pos + off, radius=cell.radius, volume=half, state=1)
            cell.pos = cell.pos - off
            cell.divide(child)


class ChemOnly(ol.Simulation[RTissue, RChem, RCell, RMetrics, RParams]):
    @ol.chemistry_rule(iterations=2)
    def diffuse(self, chem: RChem):
        # r = D dt_sub / dx^2 per neighbour pair (26 Moore neighbours here)
        chem.o2 = ol.math.clamp(chem.o2 + 0.0064 * chem.laplacian() - 0.00125 * chem.uptake() * chem.o2, 0.0, 1.0)


def _engine(sim, tissue_shape, voxel, n_agents, seed=0):
    random.seed(seed)
    eng = ol.Engine(backend="cpu")
    eng.setup_geometry(tissue_shape=tissue_shape, tissue_voxel_size=voxel, cell_diameter=10.0)
    eng.setup_tissue(RTissue)
    eng.setup_chemistry(RChem)
    c = [d * voxel * 0.5 for d in tissue_shape]
    for _ in range(n_agents):
        while True:
            p = [random.uniform(-1.0, 1.0) for _ in range(3)]
            if p[0] ** 2 + p[1] ** 2 + p[2] ** 2 <= 1.0:
                break
        eng.cells.add(RCell(pos=ol.vec3(c[0] + 60.0 * p[0], c[1] + 60.0 * p[1], c[2] + 60.0 * p[2]),
                            volume=random.uniform(1.0, 2.0)))
    eng.load_model(sim)
    return eng


def main() -> None:
    n_agents, steps = 10_000, 3
    # the agent phase: the plain workload's 10,000 agents in a 256 um domain
    # (10 um tissue bins, as the workload's contact bins)
    t0 = time.perf_counter()
    eng = _engine(CellsOnly(), (26, 26, 26), 10.0, n_agents)
    t_setup_agents = time.perf_counter() - t0
    agent_times, agents = [], []
    for _ in range(steps):
        agents.append(len(eng.cells._data))
        t0 = time.perf_counter()
        eng.run_step()
        agent_times.append(time.perf_counter() - t0)
    # chemistry iterations: a 32^3 chemistry grid (tissue 64^3, tied at half
    # resolution), two iterations per step, with the agents depositing uptake
    t0 = time.perf_counter()
    chem = _engine(ChemOnly(), (64, 64, 64), 4.0, n_agents)
    t_setup_chem = time.perf_counter() - t0
    chem_times = []
    for _ in range(2):
        t0 = time.perf_counter()
        chem.run_step()
        chem_times.append(time.perf_counter() - t0)
    vox = 32 ** 3
    t_agent = min(agent_times)
    t_iter = min(chem_times) / 2
    vox_per_s = vox / t_iter
    # the plain workload's step: agent phase + 80 substeps over 64^3 voxels
    t_step = t_agent + 80 * (64 ** 3) / vox_per_s
    rec = {
        "kind": "reference", "cores": 1,
        "value": n_agents / t_step, "unit": "agent-steps/s",
        "voxel_updates_per_s": vox_per_s, "agent_phase_agent_steps_per_s": agents[agent_times.index(t_agent)] / t_agent,
        "sample": (f"the reference's CPUBackend (pure Python, one core): agent phase of {n_agents} agents timed over "
                   f"{steps} steps (best {t_agent:.3f} s), one chemistry iteration over 32^3 voxels timed over two "
                   f"steps of two iterations (best {t_iter:.3f} s); the plain workload's step (10,000 agents, 80 "
                   "substeps over 64^3 voxels) extrapolated from them"),
        "extrapolated": True,
        "setup_s": {"agents": t_setup_agents, "chemistry_grid": t_setup_chem},
        "agent_phase_s": agent_times, "chemistry_step_s_two_iterations": chem_times,
        "host": {"machine": platform.machine(), "processor": platform.processor() or platform.machine(),
                 "python": platform.python_version(), "cpus": os.cpu_count()},
        "measured_where": "the build container (the reference checkout does not travel to the GPU box)",
        "script": "oracle/time_reference_cpu.py",
    }
    with open(os.path.join(HERE, "reference_cpu_backend.json"), "w") as fh:
        json.dump(rec, fh, indent=1)
    print(json.dumps(rec, indent=1))


if __name__ == "__main__":
    main()
