"""Generates the golden fixtures in this directory from the reference itself.

Run in a container that has the reference checked out (it imports the
reference's Python package from REF_SRC; nothing at test time does):

    python tests/golden/make_golden.py [/path/to/reference]

Fixtures:
  morton_keys.json     keys from framework/src/oncolytica/core/runtime/_geometry.py:14-47
                       (get_chemical_voxel_key, get_tissue_voxel_key, voxel_table_size)
  sort_contract.npz    the inputs and per-key id sets of framework/tests/test_gpu.py:17-61
                       (N = 10,000, 50^3 bins, voxel 2.0, random.seed(42)), keys computed by
                       the reference's get_tissue_voxel_key on the float32 positions
  cpu_lifecycle.json   framework/tests/test_oncolytica.py:58-93 run on the reference's
                       CPUBackend: live-cell count and metric per step
"""


import json
import os
import random
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout: the first argument, else $OLC_REFERENCE, else a
# directory named "reference" beside this repository
REF = (sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OLC_REFERENCE")
       or os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(HERE))), "reference"))
REF_SRC = os.path.join(REF, "framework", "src")


def main() -> None:
    sys.path.insert(0, REF_SRC)
    from oncolytica.core.runtime import _geometry as geo  # reference module

    # ---- Morton keys ---------------------------------------------------
    rng = random.Random(1234)
    coords = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 1), (2, 3, 5), (7, 8, 9),
              (119, 119, 119), (239, 239, 239), (240, 240, 240), (25, 25, 25), (26, 26, 26),
              (99, 99, 99), (100, 100, 100), (49, 49, 49), (50, 50, 50), (255, 0, 511), (511, 511, 511)]
    coords += [(rng.randrange(0, 241), rng.randrange(0, 241), rng.randrange(0, 241)) for _ in range(400)]
    tissue = [[c[0], c[1], c[2], geo.get_tissue_voxel_key(*c)] for c in coords]
    chem = [[c[0], c[1], c[2], geo.get_chemical_voxel_key(*c)] for c in coords if max(c) < 512]
    dims = [(2, 2, 2), (10, 10, 10), (26, 26, 26), (50, 50, 50), (100, 100, 100), (120, 64, 32),
            (40, 40, 2), (64, 64, 64), (240, 240, 240), (52, 52, 52)]
    table = [[d[0], d[1], d[2], geo.voxel_table_size(d)] for d in dims]
    with open(os.path.join(HERE, "morton_keys.json"), "w") as fh:
        json.dump({"source": "framework/src/oncolytica/core/runtime/_geometry.py:14-47",
                   "tissue": tissue, "chemical": chem, "voxel_table_size": table}, fh)

    # ---- sort contract (test_gpu.py:17-61) -----------------------------
    N, GDIM, VS = 10_000, (50, 50, 50), 2.0
    random.seed(42)
    pos = np.zeros((N, 3), dtype=np.float32)
    for i in range(N):
        p = [random.uniform(0, GDIM[j] * VS * 0.99) for j in range(3)]
        pos[i] = p
    keys = np.array([geo.get_tissue_voxel_key(*(int(float(x) / VS) for x in pos[i])) for i in range(N)],
                    dtype=np.uint32)
    np.savez_compressed(os.path.join(HERE, "sort_contract.npz"), pos=pos, keys=keys,
                        dims=np.array(GDIM, dtype=np.int32), vs=np.float32(VS),
                        n_table=np.uint32(geo.voxel_table_size(GDIM)))

    # ---- CPU lifecycle (test_oncolytica.py:58-93) ----------------------
    import oncolytica as ol

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

    def run(initial_health, collect_at):
        engine = ol.Engine(backend="cpu")
        for i in range(5):
            cell = MyCell()
            cell.pos = ol.vec3(50.0, 50.0, 50.0) + 5.0 * ol.vec3(float(i))
            if initial_health is not None:
                cell.health = initial_health
            engine.cells.add(cell)
        engine.load_model(BasicSim())
        steps = []
        for s in range(11):
            collect = (s + 1) in collect_at
            engine.run_step(collect_metrics=collect)
            alive = sum(1 for c in engine.cells._data if getattr(c, "_alive", True))
            rec = {"step": s + 1, "alive_after": alive, "rows": len(engine.cells._data)}
            if collect:
                rec["metric_alive_cells"] = int(engine.get_metrics().alive_cells)
            steps.append(rec)
        return steps

    # A: the reference test as written (health defaults to 0.0, metrics at step 10)
    # B: health 100, so the cells live for 9 steps and die in step 10
    with open(os.path.join(HERE, "cpu_lifecycle.json"), "w") as fh:
        json.dump({"source": "framework/tests/test_oncolytica.py:58-93 on CPUBackend "
                             "(framework/src/oncolytica/cpu/_cpu_backend.py:36-70)",
                   "A_default_health": run(None, {10}),
                   "B_health_100": run(100.0, set())}, fh, indent=1)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
