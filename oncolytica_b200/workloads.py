"""Built-in workloads: the tumour-spheroid model of the benchmark configurations,
written in the rule DSL, and seeded synthetic initial states.

Configurations (units: µm, hours):
  * ``plain_small`` — 256 µm cube, 64^3 O2 field (dx 4 µm, D 2000, Dirichlet
    1.0, initial 1.0), 10,000 spheres of radius 5 µm uniform in a 60 µm ball,
    volume growth 0.05/h, 10 µm contact bins, dt 0.1 h, 100 steps, FP32.
  * ``scale`` — 1 mm cube, 1,000,000 agents in a 400 µm ball, radii U(4, 6),
    two 256^3 fields: O2 (D 2000) and drug (D 500, decay 0.1/h, boundary source
    1.0); death probability 0.02 * drug per step from the agent RNG; 1,000 steps.
The rule: divide when the volume exceeds 2x (normalised V0 = 1) if O2 > 0.3;
quiescent if 0.1 < O2 <= 0.3; necrotic if O2 <= 0.1; live non-necrotic cells
deposit an uptake rate of 0.02 /h into their O2 voxel.  No public dataset
exists for these; all inputs are generated here from numpy's default_rng(seed).
"""
from __future__ import annotations

import math
from typing import Any
from dataclasses import dataclass, field, replace

import numpy as np

import oncolytica_b200 as ol
from oncolytica_b200.engine import Engine, stable_substeps

PROLIFERATING: ol.i32 = 1
QUIESCENT: ol.i32 = 2
NECROTIC: ol.i32 = 3


class TumourTissue(ol.Tissue):
    pass


class O2Chem(ol.Chemistry):
    o2: ol.f32 = 1.0


class O2DrugChem(ol.Chemistry):
    o2: ol.f32 = 1.0
    drug: ol.f32 = 0.0


class TumourCell(ol.Cell):
    pos: ol.vec3
    radius: ol.f32 = 5.0
    volume: ol.f32 = 1.0
    state: ol.i32 = 1


class TumourMetrics(ol.Metrics):
    live: ol.i32 = 0
    proliferating: ol.i32 = 0
    quiescent: ol.i32 = 0
    necrotic: ol.i32 = 0


class TumourParams(ol.Params):
    dt: ol.f32 = 0.1
    growth: ol.f32 = 0.05
    v_div: ol.f32 = 2.0
    o2_necrotic: ol.f32 = 0.1
    o2_quiescent: ol.f32 = 0.3
    uptake: ol.f32 = 0.02
    death_k: ol.f32 = 0.0


class TumourSim(ol.Simulation[TumourTissue, O2Chem, TumourCell, TumourMetrics, TumourParams]):
    """Oxygen-limited growth (plain_small)."""

    @ol.cell_rule
    def cycle(self, cell: TumourCell):
        chem: O2Chem = self.chemistry_at(cell.pos)
        if cell.state == NECROTIC:
            return
        o2: ol.f32 = chem.o2
        if o2 <= self.params.o2_necrotic:
            cell.state = NECROTIC
            return
        self.sink_at(cell.pos).o2 += self.params.uptake
        if o2 <= self.params.o2_quiescent:
            cell.state = QUIESCENT
            return
        cell.state = PROLIFERATING
        cell.volume += self.params.growth * cell.volume * self.params.dt
        if cell.volume > self.params.v_div:
            half: ol.f32 = cell.volume * 0.5
            cell.volume = half
            d: ol.vec3 = ol.random_dir()
            off: ol.vec3 = d * (cell.radius * 0.5)
            child: TumourCell = TumourCell(pos=cell.pos + off, radius=cell.radius, volume=half,
                                           state=PROLIFERATING)
            cell.pos = cell.pos - off
            cell.divide(child)

    @ol.metric_rule
    def census(self, cell: TumourCell, m: TumourMetrics):
        m.live += 1
        if cell.state == PROLIFERATING:
            m.proliferating += 1
        elif cell.state == QUIESCENT:
            m.quiescent += 1
        else:
            m.necrotic += 1


class TumourDrugSim(ol.Simulation[TumourTissue, O2DrugChem, TumourCell, TumourMetrics, TumourParams]):
    """Oxygen-limited growth with drug-induced death (scale)."""

    @ol.cell_rule
    def cycle(self, cell: TumourCell):
        chem: O2DrugChem = self.chemistry_at(cell.pos)
        if cell.state == NECROTIC:
            return
        o2: ol.f32 = chem.o2
        if o2 <= self.params.o2_necrotic:
            cell.state = NECROTIC
            return
        if ol.random() < self.params.death_k * chem.drug:
            cell.die()
            return
        self.sink_at(cell.pos).o2 += self.params.uptake
        if o2 <= self.params.o2_quiescent:
            cell.state = QUIESCENT
            return
        cell.state = PROLIFERATING
        cell.volume += self.params.growth * cell.volume * self.params.dt
        if cell.volume > self.params.v_div:
            half: ol.f32 = cell.volume * 0.5
            cell.volume = half
            d: ol.vec3 = ol.random_dir()
            off: ol.vec3 = d * (cell.radius * 0.5)
            child: TumourCell = TumourCell(pos=cell.pos + off, radius=cell.radius, volume=half,
                                           state=PROLIFERATING)
            cell.pos = cell.pos - off
            cell.divide(child)

    @ol.metric_rule
    def census(self, cell: TumourCell, m: TumourMetrics):
        m.live += 1
        if cell.state == PROLIFERATING:
            m.proliferating += 1
        elif cell.state == QUIESCENT:
            m.quiescent += 1
        else:
            m.necrotic += 1


@dataclass
class TumourSpec:
    """All numbers of one tumour-spheroid configuration."""

    name: str
    n_agents: int
    domain: float
    ball_radius: float
    field_dims: tuple
    bin_size: float = 10.0
    r_lo: float = 5.0
    r_hi: float = 5.0
    has_drug: bool = False
    dt: float = 0.1
    steps: int = 100
    growth: float = 0.05
    v_div: float = 2.0
    v_lo: float = 1.0
    v_hi: float = 2.0
    o2_necrotic: float = 0.1
    o2_quiescent: float = 0.3
    uptake: float = 0.02
    death_k: float = 0.0
    D_o2: float = 2000.0
    bnd_o2: float = 1.0
    init_o2: float = 1.0
    D_drug: float = 500.0
    decay_drug: float = 0.1
    bnd_drug: float = 1.0
    init_drug: float = 0.0
    stiffness: float = 1.0
    mobility: float = 10.0
    max_disp: float = 1.0
    margin: float = 0.1
    seed: int = 0
    capacity: int = 0
    tissue_dims: tuple = field(default=())
    storage: str = "f32"      # field storage: "f32", "bf16" or "f16"
    encoding: str = "auto"    # 16-bit element encoding (Engine.setup_diffusion)

    def __post_init__(self) -> None:
        if not self.tissue_dims:
            nb = int(math.ceil(self.domain / self.bin_size))
            nb += nb % 2
            self.tissue_dims = (nb, nb, nb)
        if not self.capacity:
            self.capacity = max(4 * self.n_agents, 1024)

    @property
    def dx(self) -> float:
        return self.domain / self.field_dims[0]

    @property
    def S_o2(self) -> int:
        return stable_substeps(self.D_o2, self.dt, self.dx)

    @property
    def S_drug(self) -> int:
        return stable_substeps(self.D_drug, self.dt, self.dx) if self.has_drug else 0

    @property
    def center(self) -> tuple:
        c = self.domain * 0.5
        return (c, c, c)

    def voxel_updates_per_step(self) -> int:
        nv = int(np.prod(self.field_dims))
        return nv * (self.S_o2 + (self.S_drug if self.has_drug else 0))


PLAIN_SMALL = TumourSpec(name="plain_small", n_agents=10_000, domain=256.0, ball_radius=60.0,
                         field_dims=(64, 64, 64), steps=100)
SCALE = TumourSpec(name="scale", n_agents=1_000_000, domain=1000.0, ball_radius=400.0, field_dims=(256, 256, 256),
                   r_lo=4.0, r_hi=6.0, has_drug=True, death_k=0.02, steps=1000)
CONFIGS = {s.name: s for s in (PLAIN_SMALL, SCALE)}


def batched_specs(n_sims: int = 512, seed: int = 0, g_choices: tuple = (32, 48, 64, 96, 128),
                  n_range: tuple = (1e3, 2e5), density: float = 3.73e-3, steps: int = 0) -> list:
    """Members of a parameter sweep (the batched configuration): per member a
    grid G from ``g_choices`` (domain G * 4 um, dx = 4 um, 10 um bins), an agent
    count log-uniform in ``n_range`` capped so the ball of radius 0.4 * domain is
    no denser than the scale workload (``density`` agents per um^3), D_O2 ~
    U(1000, 3000), uptake ~ U(0.01, 0.04), drug decay ~ U(0.05, 0.2), and seed
    ``seed + k``.  Drawn from numpy default_rng(seed).  Agent capacity: twice
    the start, or for a run of ``steps`` steps the serving mix's rule (the
    population doubling every 300 steps, 50 % headroom)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_sims):
        g = int(rng.choice(g_choices))
        domain = 4.0 * g
        ball = 0.4 * domain
        n_max = max(100, int(density * (4.0 / 3.0) * math.pi * ball ** 3))
        n = int(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1]))))
        n = max(100, min(n, n_max))
        out.append(TumourSpec(name=f"sweep_{k}", n_agents=n, domain=domain, ball_radius=ball, field_dims=(g, g, g),
                              r_lo=4.0, r_hi=6.0, has_drug=True, D_o2=float(rng.uniform(1000.0, 3000.0)),
                              uptake=float(rng.uniform(0.01, 0.04)), decay_drug=float(rng.uniform(0.05, 0.2)),
                              death_k=0.02, seed=seed + k,
                              capacity=(int(1.5 * n * 2.0 ** (steps / 300.0)) + 8192) if steps else 2 * n + 1024))
    return out


def serving_schedule(rate: float = 20.0, duration: float = 120.0, seed: int = 0, steps_range: tuple = (100, 1000),
                     storage: str = "f32") -> list:
    """Requests of the serving mix: a Poisson process of ``rate`` requests/s
    over ``duration`` s; each request is one simulation drawn like a member of
    the batched sweep (``batched_specs``) with a step count uniform in
    ``steps_range``.  Its agent capacity (its solo run's max_agents, reserved on
    admission) allows the population to double every 300 steps with 50 %
    headroom: the largest domains grew about 6x in 900 steps.  Returns
    (arrival s, spec, steps) triples in arrival order, from numpy
    default_rng(seed)."""
    rng = np.random.default_rng(seed)
    times, t = [], 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > duration:
            break
        times.append(t)
    specs = batched_specs(len(times), seed=seed + 7919) if times else []
    steps = rng.integers(steps_range[0], steps_range[1] + 1, size=len(times))
    return [(tt, replace(sp, storage=storage, capacity=int(1.5 * sp.n_agents * 2.0 ** (n / 300.0)) + 8192,
                         name=f"request_{k}"), int(n))
            for k, (tt, sp, n) in enumerate(zip(times, specs, steps))]


def scaled(spec: TumourSpec, **kw) -> TumourSpec:
    """A copy with some numbers changed (smaller test cases)."""
    out = replace(spec, **kw)
    if "domain" in kw or "bin_size" in kw:
        out.tissue_dims = ()
        out.__post_init__()
    return out


def initial_state(spec: TumourSpec) -> dict:
    """Agents uniform in the ball (rejection sampling), radii U(r_lo, r_hi),
    volumes U(v_lo, v_hi), all proliferating, RNG states seeded from the index."""
    from oncolytica_b200.backend import seed_rng

    rng = np.random.default_rng(spec.seed)
    n = spec.n_agents
    pts = np.zeros((0, 3))
    while len(pts) < n:
        cand = rng.uniform(-1.0, 1.0, size=(max(2 * (n - len(pts)), 1024), 3))
        cand = cand[np.einsum("ij,ij->i", cand, cand) <= 1.0]
        pts = np.concatenate([pts, cand])
    pos = (np.asarray(spec.center) + pts[:n] * spec.ball_radius).astype(np.float32)
    radius = (rng.uniform(spec.r_lo, spec.r_hi, size=n) if spec.r_hi > spec.r_lo
              else np.full(n, spec.r_lo)).astype(np.float32)
    volume = rng.uniform(spec.v_lo, spec.v_hi, size=n).astype(np.float32)
    return {"x": pos[:, 0].copy(), "y": pos[:, 1].copy(), "z": pos[:, 2].copy(), "radius": radius,
            "volume": volume, "state": np.full(n, int(PROLIFERATING), np.int32),
            "rng": seed_rng(spec.seed, np.arange(n, dtype=np.uint32))}


def initial_fields(spec: TumourSpec) -> tuple[np.ndarray, np.ndarray | None]:
    """O2 (and drug) fields indexed [z, y, x] with the Dirichlet faces set."""
    def make(init, bnd):
        f = np.full(spec.field_dims[::-1], init, np.float32)
        f[0], f[-1] = bnd, bnd
        f[:, 0], f[:, -1] = bnd, bnd
        f[:, :, 0], f[:, :, -1] = bnd, bnd
        return f

    o2 = make(spec.init_o2, spec.bnd_o2)
    drug = make(spec.init_drug, spec.bnd_drug) if spec.has_drug else None
    return o2, drug


def build_engine(spec: TumourSpec, state: dict | None = None) -> Engine:
    """An Engine loaded with the tumour model and the initial state of ``spec``."""
    eng, sim = configure_engine(spec, state)
    eng.load_model(sim)
    return eng


def build_batch(specs: list, states: list | None = None, max_agents: int | None = None):
    """A BatchEngine running the tumour model for every spec (one member each)."""
    from oncolytica_b200.batch import BatchEngine

    states = states if states is not None else [None] * len(specs)
    pairs = [configure_engine(sp, st) for sp, st in zip(specs, states)]
    cap = max_agents if max_agents is not None else sum(sp.capacity for sp in specs)
    return BatchEngine([e for e, _ in pairs], [s for _, s in pairs], max_agents=cap)


def configure_engine(spec: TumourSpec, state: dict | None = None) -> tuple[Engine, Any]:
    """An Engine set up for ``spec`` (geometry, fields, contact, agents) and the
    model instance carrying its parameters, not yet loaded."""
    state = state if state is not None else initial_state(spec)
    eng = Engine(backend="cuda", max_agents=spec.capacity)
    eng.setup_geometry(tissue_shape=tuple(spec.tissue_dims), tissue_voxel_size=spec.bin_size)
    eng.setup_domain((0.0, 0.0, 0.0), (spec.domain,) * 3)
    eng.dt = spec.dt
    eng.seed = spec.seed
    chem_cls = O2DrugChem if spec.has_drug else O2Chem
    eng.setup_chemistry(chem_cls, shape=tuple(spec.field_dims), voxel_size=spec.dx)
    eng.chemistry.column("o2")[...] = spec.init_o2
    eng.setup_diffusion("o2", diffusion=spec.D_o2, boundary=spec.bnd_o2, substeps=spec.S_o2, storage=spec.storage,
                        encoding=spec.encoding)
    if spec.has_drug:
        eng.chemistry.column("drug")[...] = spec.init_drug
        eng.setup_diffusion("drug", diffusion=spec.D_drug, decay=spec.decay_drug, boundary=spec.bnd_drug,
                            substeps=spec.S_drug, storage=spec.storage, encoding=spec.encoding)
    eng.setup_contact(radius="radius", stiffness=spec.stiffness, mobility=spec.mobility, max_disp=spec.max_disp,
                      margin=spec.margin)
    eng.cells.add_arrays(TumourCell, **{"pos.x": state["x"], "pos.y": state["y"], "pos.z": state["z"],
                                        "radius": state["radius"], "volume": state["volume"],
                                        "state": state["state"], "_rng_state": state["rng"]})
    sim = TumourDrugSim() if spec.has_drug else TumourSim()
    sim._params = TumourParams(dt=float(spec.dt), growth=float(spec.growth), v_div=float(spec.v_div),
                               o2_necrotic=float(spec.o2_necrotic), o2_quiescent=float(spec.o2_quiescent),
                               uptake=float(spec.uptake), death_k=float(spec.death_k))
    return eng, sim
