"""Generates cpu_rules.json from the reference itself: tests/pinned_model.py's
rules run on the reference's CPUBackend (framework/src/oncolytica/cpu/
_cpu_backend.py:36-70) from a seeded initial state, every live agent and the
metrics recorded after each step.  Run in a container that has the reference
checked out (nothing at test time imports the reference):

    python tests/golden/make_cpu_rules_golden.py [/path/to/reference]

The model text is tests/pinned_model.py with its import line pointed at the
reference package, so both sides run the same rules.
"""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout: the first argument, else $OLC_REFERENCE, else a
# directory named "reference" beside this repository
REF = (sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OLC_REFERENCE")
       or os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(HERE))), "reference"))

TISSUE = (16, 16, 16)
VOXEL = 2.0
STEPS = 12
N = 240


def initial_state(seed: int = 17) -> dict:
    """Agents at voxel centres plus multiples of 1/8 (exact in FP32 and far
    from voxel faces), static nutrient and stiffness grids."""
    rng = np.random.default_rng(seed)
    cells = rng.integers(1, TISSUE[0] - 2, size=(N, 3))
    pos = cells * VOXEL + 0.5 + rng.integers(0, 8, size=(N, 3)) * 0.125
    chem_shape = tuple(d // 2 for d in TISSUE)
    nutrient = rng.choice([0.0, 0.5, 1.0, 2.0], size=chem_shape)
    stiff = rng.integers(0, 2, size=TISSUE)
    energy = rng.choice([0.5, 1.0, 1.5], size=N)
    kind = rng.integers(0, 2, size=N)
    return {"pos": pos.tolist(), "uid": list(range(N)), "energy": energy.tolist(), "kind": kind.tolist(),
            "nutrient": nutrient.tolist(), "stiff": stiff.tolist()}


def main() -> None:
    sys.path.insert(0, os.path.join(REF, "framework", "src"))
    src = open(os.path.join(HERE, "..", "pinned_model.py")).read()
    src = src.replace("import oncolytica_b200 as ol", "import oncolytica as ol")
    # the reference's validator reads rule sources from their file
    tmp = tempfile.mkdtemp()
    with open(os.path.join(tmp, "pinned_model_ref.py"), "w") as fh:
        fh.write(src)
    sys.path.insert(0, tmp)
    import pinned_model_ref as mod
    ol = mod.ol
    st = initial_state()
    eng = ol.Engine(backend="cpu")
    eng.setup_geometry(tissue_shape=TISSUE, tissue_voxel_size=VOXEL, cell_diameter=1.0)
    eng.setup_tissue(mod.PTissue)
    eng.setup_chemistry(mod.PChem)
    nut = np.array(st["nutrient"])
    for i, j, k in np.ndindex(nut.shape):
        eng.chemistry.sample(i, j, k).nutrient = float(nut[i, j, k])
    stiff = np.array(st["stiff"])
    for i, j, k in np.ndindex(stiff.shape):
        eng.tissue.sample(i, j, k).stiff = int(stiff[i, j, k])
    for p, u, e, kd in zip(st["pos"], st["uid"], st["energy"], st["kind"]):
        eng.cells.add(mod.PCell(pos=ol.vec3(*p), uid=u, age=0, kind=kd, energy=e))
    eng.load_model(mod.PinnedSim())
    steps, margin = [], 1e9
    for s in range(STEPS):
        eng.run_step(collect_metrics=True)
        # the reference's metrics accumulate over steps and its metric pass
        # walks agents that died in this step too (AgentList.__iter__ does not
        # skip them); the live agents are recorded beside them
        live = [c for c in eng.cells._data if getattr(c, "_alive", True)]
        margin = min([margin] + [abs(c.energy - 0.3) for c in live])
        m = eng.get_metrics()
        steps.append({"step": s + 1,
                      "agents": sorted([[int(c.uid), int(c.age), int(c.kind), float(c.energy),
                                         float(c.pos.x), float(c.pos.y), float(c.pos.z)] for c in live]),
                      "died": sorted(int(c.uid) for c in eng.cells._data if not getattr(c, "_alive", True)),
                      "metrics": {"n": int(m.n), "n_b": int(m.n_b), "age_sum": int(m.age_sum)}})
    assert margin > 1e-4, f"an energy came within {margin} of its threshold: pick another seed"
    with open(os.path.join(HERE, "cpu_rules.json"), "w") as fh:
        json.dump({"source": "tests/pinned_model.py on the reference's CPUBackend "
                             "(framework/src/oncolytica/cpu/_cpu_backend.py:36-70)",
                   "tissue_shape": TISSUE, "tissue_voxel_size": VOXEL, "initial": st, "steps": steps,
                   "energy_threshold_margin": margin}, fh)
    print("cpu_rules.json:", STEPS, "steps,", len(steps[-1]["agents"]), "agents at the end, margin", margin)


if __name__ == "__main__":
    main()
