"""Engine: the reference's orchestrator API (framework/src/oncolytica/core/runtime/_engine.py)
with the CUDA backend as its only implementation.

Reference API kept: ``Engine(backend, max_agents)``, ``setup_geometry``,
``setup_tissue``, ``setup_chemistry``, ``setup_params``, ``update_params``,
``load_model``, ``run_step(collect_metrics)``, ``get_metrics``,
``sync_to_host``, ``step``, ``cells``, ``tissue``, ``chemistry``.

Extensions (no reference counterpart): a chemistry grid decoupled from the
bin grid (``setup_chemistry(cls, shape=, voxel_size=)``), built-in diffusion
of chemistry fields (``setup_diffusion``), built-in contact mechanics
(``setup_contact``), ``dt``, ``seed``, ``setup_domain``, ``sync_to_device``,
``run_steps``, ``get_reductions``.
"""
from __future__ import annotations

import inspect
import math

import numpy as np
from dataclasses import dataclass
from typing import Any, Optional, Type

from oncolytica_b200._containers import AgentList, Grid
from oncolytica_b200._errors import CompilationError
from oncolytica_b200._types import Cell, Chemistry, Simulation, Tissue


@dataclass
class DiffusionSpec:
    diffusion: float
    decay: float = 0.0
    boundary: float = 0.0
    substeps: Optional[int] = None
    storage: str = "f32"   # "f32", "bf16", "f16", "bf16_sr" or "f16_sr": element type (and rounding) of the field
    encoding: str = "auto"  # 16-bit elements: "value", "deficit", "offset3" or "auto" (_fieldcodec.resolve)


STORAGE_CODES = {"f32": 0, "bf16": 1, "f16": 2, "bf16_sr": 3, "f16_sr": 4}


@dataclass
class ContactSpec:
    radius: str | float = "radius"
    stiffness: float = 1.0
    mobility: float = 10.0
    max_disp: float = 1.0
    margin: float = 0.1
    # the engine's extras (tumor_sim.wgsl:505-628); defaults leave them off
    necrotic_factor: float = 1.0
    adhesion_stiffness: float = 0.0
    adhesion_range: float = 0.0
    velocity: str | None = None
    damping: float = 1.0
    max_speed: float | None = None
    state: str | None = "state"
    # active motion: one (chemotaxis_o2, chemotaxis_glucose, move_prob) record,
    # or a species table selected by an i32 cell field
    species: tuple = ()
    species_field: str | None = None
    chemo_fields: tuple = (None, None)
    chemo_force: float = 2.0
    motility_impulse: float = 0.4

    @property
    def motion(self) -> bool:
        return any(any(v != 0.0 for v in rec) for rec in self.species)

    @property
    def mechanics(self) -> bool:
        return self.necrotic_factor != 1.0 or self.adhesion_stiffness != 0.0 or self.velocity is not None or \
            self.motion


def stable_substeps(D: float, dt: float, dx: float, margin: float = 1.05) -> int:
    """Smallest S with D*dt/(S*dx^2) <= 1/6 (explicit 7-point FTCS), times a margin."""
    if D <= 0.0 or dt <= 0.0:
        return 1
    return max(1, int(math.ceil(6.0 * D * dt / (dx * dx) * margin)))


class Engine:
    """Holds the model state and dispatches steps to the CUDA backend."""

    def __init__(self, backend: str = "cuda", max_agents: int = 1024 * 256):
        if backend == "gpu":
            backend = "cuda"
        if backend != "cuda":
            raise ValueError(f"Unknown backend {backend!r}: oncolytica_b200 runs the step on CUDA only "
                             f"(backend='cuda'; 'gpu' is accepted as an alias).")
        self.backend = backend
        self.max_agents = int(max_agents)
        # geometry defaults (reference _engine.py:34-39)
        self.tissue_voxel_size: float = 1.4
        self.chemistry_voxel_size: float = 2.8
        self.cell_diameter: float = 1.0
        self.tissue_shape: Optional[tuple[int, int, int]] = (64, 64, 64)
        self.chemistry_shape: Optional[tuple[int, int, int]] = (32, 32, 32)
        self.domain_lo: Optional[tuple[float, float, float]] = None
        self.domain_hi: Optional[tuple[float, float, float]] = None
        self.dt: float = 1.0
        self.seed: int = 0
        # replay each step as one CUDA graph (same results; fewer launch gaps)
        self.use_graphs: bool = False
        # device status word (capacity overflow, a bounded wait that gave up,
        # a second divide() in one call): checked every this many steps and
        # after every collected step; "raise" (DeviceStatusError), "warn" or
        # "ignore".  The reference drops overflowing children silently.
        self.status_check_every: int = 64
        self.on_device_status: str = "raise"
        self._step = 0
        self.cells = AgentList(self)
        self.tissue: Optional[Grid] = None
        self.chemistry: Optional[Grid] = None
        self._metrics = None
        self._sim: Optional[Simulation] = None
        self._tissue_rules: list = []
        self._chemistry_rules: list = []
        self._cell_rules: list = []
        self._metric_rules: list = []
        self._diffusion: dict[str, DiffusionSpec] = {}
        self._vessel: tuple | None = None
        self._contact: Optional[ContactSpec] = None
        self._tissue_class = None
        self._chem_class = None
        self._backend_impl = None

    # ---- state initialisation ---------------------------------------------
    def setup_params(self, params: Any) -> None:
        self._sim._params = params
        if self._backend_impl is not None:
            self._backend_impl.upload_params()

    def update_params(self, **kwargs: Any) -> None:
        """Changes parameter values; unlike the reference (whose uniforms are
        packed once), the new values reach the device before the next step."""
        for name, value in kwargs.items():
            self._sim._params._validate_field(name, value)
        for name, value in kwargs.items():
            object.__setattr__(self._sim._params, name, value)
        if self._backend_impl is not None:
            self._backend_impl.upload_params()

    def setup_geometry(self, tissue_shape: tuple[int, int, int] = (120, 120, 120), tissue_voxel_size: float = 1.4,
                       cell_diameter: float = 1.0) -> None:
        self._validate_geometry(tissue_shape)
        self.tissue_shape = tuple(tissue_shape)
        self.chemistry_shape = (tissue_shape[0] // 2, tissue_shape[1] // 2, tissue_shape[2] // 2)
        self.cell_diameter = cell_diameter
        self.tissue_voxel_size = float(tissue_voxel_size)
        self.chemistry_voxel_size = 2.0 * float(tissue_voxel_size)

    @staticmethod
    def _validate_geometry(tissue_shape) -> None:
        if not isinstance(tissue_shape, (list, tuple)) or len(tissue_shape) != 3:
            raise TypeError(f"tissue_shape must be a tuple of 3 ints, got {tissue_shape!r}")
        for i, dim in enumerate(tissue_shape):
            if not isinstance(dim, int) or isinstance(dim, bool):
                raise TypeError(f"tissue_shape component {i} must be int, got {type(dim).__name__!r}")
            if dim <= 0:
                raise ValueError(f"tissue_shape component {i} must be positive, got {dim}")
            if dim > 240:
                raise ValueError(f"tissue_shape component {i} must be ≤ 240, got {dim}")
            if dim % 2 != 0:
                raise ValueError(f"tissue_shape component {i} must be even, got {dim}")

    def setup_tissue(self, tissue_class: Type) -> None:
        if not (isinstance(tissue_class, type) and issubclass(tissue_class, Tissue)):
            raise ValueError(f"tissue_class must be a subclass of ol.Tissue, got {tissue_class}")
        self._tissue_class = tissue_class
        self.tissue = Grid(tissue_class, self.tissue_shape, self)

    def setup_chemistry(self, chemistry_class: Type, shape: Optional[tuple[int, int, int]] = None,
                        voxel_size: Optional[float] = None) -> None:
        """Chemistry grid.  Without ``shape``/``voxel_size`` it is the
        reference's tied grid (tissue/2 at twice the voxel size)."""
        if not (isinstance(chemistry_class, type) and issubclass(chemistry_class, Chemistry)):
            raise ValueError(f"chemistry_class must be a subclass of ol.Chemistry, got {chemistry_class}")
        if shape is not None:
            if len(shape) != 3 or any(int(s) < 3 for s in shape):
                raise ValueError("chemistry shape must be 3 ints >= 3")
            self.chemistry_shape = tuple(int(s) for s in shape)
        if voxel_size is not None:
            if voxel_size <= 0:
                raise ValueError("chemistry voxel_size must be > 0")
            self.chemistry_voxel_size = float(voxel_size)
        self._chem_class = chemistry_class
        self.chemistry = Grid(chemistry_class, self.chemistry_shape, self)

    def setup_diffusion(self, field: str, diffusion: float, decay: float = 0.0, boundary: float = 0.0,
                        substeps: Optional[int] = None, storage: str = "f32", encoding: str = "auto") -> None:
        """Built-in diffusion of one chemistry field: per step an implicit sink
        (rates deposited with ``self.sink_at(pos).field += k``), then S explicit
        7-point substeps with the outer faces pinned to ``boundary``
        (engine tumor_sim.wgsl:387-446; substeps as chemistry_rule(iterations=S)).
        ``storage`` "bf16" or "f16" keeps the field in 16 bits: updates run in
        FP32, and uptake and decay are applied once per step with a per-voxel
        FP32 rounding residual carried to the next step; "bf16_sr" and
        "f16_sr" round the substeps stochastically (reproducible hash bits) so
        that small diffusion increments are not lost to the short mantissa and
        rounding errors do not accumulate a bias (no counterpart in the
        reference, whose fields are FP32).  ``encoding`` says what a 16-bit
        element holds: "value"; "deficit" (boundary - value, for fields that
        stay near their boundary value, like O2); "offset3" (the value minus
        the nearest of 0, b/2 and b: fine near all three); "auto" picks
        "offset3" for BF16 fields with 0 < b <= 4 and "value" otherwise
        (_fieldcodec.resolve).  Encoded fields are clamped to [0, boundary]
        (FP32 and value-encoded fields at 0 only), so a BF16 field whose
        values may exceed its boundary value needs ``encoding="value"``."""
        from oncolytica_b200._fieldcodec import ENCODINGS

        if storage not in STORAGE_CODES:
            raise ValueError(f"storage must be one of {sorted(STORAGE_CODES)}, got {storage!r}")
        if encoding != "auto" and encoding not in ENCODINGS:
            raise ValueError(f"encoding must be 'auto' or one of {sorted(ENCODINGS)}, got {encoding!r}")
        self._diffusion[field] = DiffusionSpec(float(diffusion), float(decay), float(boundary), substeps, storage,
                                               encoding)

    def field_encoding(self, field: str) -> int:
        """The OLC_ENC_* code a diffusing field's 16-bit elements use (0 for
        FP32 fields and static fields), resolving "auto" from the field's
        storage, decay, boundary and current host values."""
        from oncolytica_b200._fieldcodec import resolve

        spec = self._diffusion.get(field)
        if spec is None:
            return 0
        mean = None
        if self.chemistry is not None and field in self.chemistry._fields:
            vals = np.asarray(self.chemistry.column(field), dtype=np.float64)
            mean = float(vals.mean()) if vals.size else None
        return resolve(spec.encoding, STORAGE_CODES[spec.storage], spec.decay, spec.boundary, mean)

    def setup_contact(self, radius: str | float = "radius", stiffness: float = 1.0, mobility: float = 10.0,
                      max_disp: float = 1.0, margin: float = 0.1, necrotic_factor: float = 1.0,
                      adhesion_stiffness: float = 0.0, adhesion_range: float = 0.0, velocity: str | None = None,
                      damping: float = 1.0, max_speed: float | None = None, state: str | None = "state",
                      chemotaxis: tuple = (0.0, 0.0), motility: float = 0.0, species: list | None = None,
                      species_field: str | None = None, chemotactic_fields: tuple | None = None,
                      chemo_force: float = 2.0, motility_impulse: float = 0.4) -> None:
        """Built-in Hertz-like contact repulsion over the 27 bins
        (engine tumor_sim.wgsl:505-628), overdamped.  The engine's other terms
        are optional: `necrotic_factor` scales repulsion when either agent's
        `state` is 3 (the engine uses 0.3); `adhesion_stiffness` and
        `adhesion_range` add the cosine adhesion between non-necrotic agents;
        `velocity` names an ol.vec3 cell field for the engine's damped velocity
        integration (`damping`, speed cap `max_speed`, default 0.8 x bin size)
        in place of the overdamped move.  Active motion of non-necrotic agents
        (tumor_sim.wgsl:584-604): `chemotaxis` = (O2, glucose) coefficients on
        the gradients of `chemotactic_fields` (default: the first two chemistry
        fields) times `chemo_force`, and random motility `motility` times
        `motility_impulse` along a direction drawn from the agent's RNG; or a
        `species` table of (chemotaxis_o2, chemotaxis_glucose, move_prob)
        records selected by the i32 cell field `species_field`."""
        if adhesion_stiffness != 0.0 and not adhesion_range > 0.0:
            raise ValueError("adhesion_stiffness needs adhesion_range > 0")
        if species is None:
            table = (tuple(float(v) for v in (*chemotaxis, motility)),)
        else:
            table = tuple(tuple(float(v) for v in rec) for rec in species)
            if not 1 <= len(table) <= 8 or any(len(rec) != 3 for rec in table):
                raise ValueError("species: 1 to 8 records of (chemotaxis_o2, chemotaxis_glucose, move_prob)")
        self._contact = ContactSpec(radius, float(stiffness), float(mobility), float(max_disp), float(margin),
                                    float(necrotic_factor), float(adhesion_stiffness), float(adhesion_range),
                                    velocity, float(damping), None if max_speed is None else float(max_speed),
                                    state, table, species_field,
                                    tuple(chemotactic_fields) if chemotactic_fields is not None else (None, None),
                                    float(chemo_force), float(motility_impulse))

    def setup_vessel(self, center: tuple[float, float], radius: float, value: float = 1.0,
                     fields: tuple | None = None) -> None:
        """The engine's vessel (engine/assets/shaders/tumor_sim.wgsl:375-385,
        425-428): interior chemistry voxels whose centre lies within `radius`
        of the axis parallel to y through (x, z) = `center` are held at
        `value` after every diffusion substep of `fields` (default: every FP32
        diffusing field).  Face voxels keep the Dirichlet boundary value, as
        the engine tests the faces before the vessel."""
        if radius <= 0.0:
            raise ValueError("setup_vessel: radius must be positive")
        self._vessel = (float(center[0]), float(center[1]), float(radius), float(value),
                        tuple(fields) if fields is not None else None)

    def vessel_voxels(self) -> np.ndarray:
        """x-fastest indices of the interior chemistry voxels inside the vessel."""
        cx, cz, r, _, _ = self._vessel
        nx, ny, nz = (int(v) for v in self.chemistry_shape)
        dx = float(self.chemistry_voxel_size)
        lo = self.domain_lo or (0.0, 0.0, 0.0)
        xs = lo[0] + (np.arange(nx) + 0.5) * dx
        zs = lo[2] + (np.arange(nz) + 0.5) * dx
        inside = (xs[None, :] - cx) ** 2 + (zs[:, None] - cz) ** 2 <= r * r  # [z][x]
        inside[[0, -1], :] = False
        inside[:, [0, -1]] = False
        z, x = np.nonzero(inside)
        y = np.arange(1, ny - 1)
        idx = (z[:, None] * ny + y[None, :]) * nx + x[:, None]
        return np.sort(idx.ravel()).astype(np.uint32)

    def setup_domain(self, lo: tuple[float, float, float], hi: tuple[float, float, float]) -> None:
        self.domain_lo = tuple(float(v) for v in lo)
        self.domain_hi = tuple(float(v) for v in hi)

    def substeps_for(self, field: str) -> int:
        spec = self._diffusion[field]
        if spec.substeps:
            return int(spec.substeps)
        return stable_substeps(spec.diffusion, self.dt, self.chemistry_voxel_size)

    @property
    def step(self) -> int:
        return self._step

    # ---- model loading ----------------------------------------------------
    def load_model(self, sim_instance: Any) -> None:
        self._prepare_model(sim_instance)
        from oncolytica_b200.backend import CudaBackend

        self._backend_impl = CudaBackend(self)
        self._backend_impl.compile(sim_instance)

    def _prepare_model(self, sim_instance: Any) -> None:
        """Rule discovery and model checks of load_model, without a backend
        (a BatchEngine drives many prepared engines through one handle)."""
        if not isinstance(sim_instance, Simulation):
            raise CompilationError(f"Expected an instance of 'ol.Simulation', got '{type(sim_instance).__name__}'.")
        self._sim = sim_instance
        self._metrics = sim_instance._spec.metrics_class(sim_instance)
        sim_instance._engine = self
        self._tissue_rules.clear()
        self._chemistry_rules.clear()
        self._cell_rules.clear()
        self._metric_rules.clear()
        # rule discovery by tag, in dir() order (reference _engine.py:130-147)
        for name in dir(sim_instance):
            if name.startswith("_"):
                continue
            try:
                method = getattr(sim_instance, name)
            except Exception:
                continue
            if not callable(method):
                continue
            kind = getattr(method, "_rule_type", None)
            {"tissue": self._tissue_rules, "chemistry": self._chemistry_rules, "cell": self._cell_rules,
             "metric": self._metric_rules}.get(kind, []).append(method)
        if self.tissue is None and self._tissue_class is None:
            self._tissue_class = sim_instance._spec.tissue_class
        if self.chemistry is None:
            self.setup_chemistry(sim_instance._spec.chemistry_class)
        for f in self._diffusion:
            if f not in self.chemistry._fields:
                raise CompilationError(f"setup_diffusion: chemistry class has no field {f!r}")

    # ---- execution ---------------------------------------------------------
    def run_step(self, collect_metrics: bool = False, wait: bool = True):
        """One step.  With ``collect_metrics`` the step's metric values reach
        the host: at once (``wait``, as the reference), or, with
        ``wait=False``, through the returned PendingReadback, whose
        ``result()`` (or the next get_metrics()) waits for that step's copies
        only, so the caller can queue the next step before reading this one."""
        if self._sim is None or self._backend_impl is None:
            raise RuntimeError("Engine.run_step() called before load_model().")
        self._step += 1
        return self._backend_impl.run_steps(1, collect_metrics=collect_metrics, wait=wait)

    def run_steps(self, n: int, collect_metrics: bool = False, wait: bool = True):
        """n steps enqueued back to back (metrics after the last when asked;
        ``wait`` as in run_step)."""
        if self._sim is None or self._backend_impl is None:
            raise RuntimeError("Engine.run_steps() called before load_model().")
        self._step += n
        return self._backend_impl.run_steps(n, collect_metrics=collect_metrics, wait=wait)

    def set_graphs(self, enable: bool) -> None:
        """Runs later steps through cached CUDA graphs of whole steps (no
        counterpart in the reference); results are identical to eager steps."""
        self.use_graphs = bool(enable)
        if self._backend_impl is not None:
            self._backend_impl.set_graphs(self.use_graphs)

    def get_metrics(self) -> Any:
        if self._backend_impl is not None and hasattr(self._backend_impl, "resolve_pending"):
            self._backend_impl.resolve_pending()
        return self._metrics

    def get_engine_metrics(self, **kw: Any) -> dict:
        """The engine's metrics set (engine/assets/shaders/tumor_sim.wgsl:248-361:
        counts, fractions, centroid, radii, mean field values, crowding) of the
        current state, computed on the device; keyword arguments name the
        columns and fields to read (CudaBackend.engine_metrics)."""
        if self._backend_impl is None:
            raise RuntimeError("Engine.get_engine_metrics() called before load_model().")
        return self._backend_impl.engine_metrics(**kw)

    def close(self) -> None:
        """Releases the device state now (the engine, its model instance and its
        backend refer to each other, so without this the memory is freed only
        when Python's cycle collector runs)."""
        if self._backend_impl is not None:
            self._backend_impl.close()
            self._backend_impl = None

    # ---- checkpoints ----------------------------------------------------------
    def state_dict(self) -> dict:
        """The device state as host arrays (CudaBackend.state_dict); resuming
        from it with load_state_dict continues bit for bit."""
        if self._backend_impl is None:
            raise RuntimeError("Engine.state_dict() called before load_model().")
        return self._backend_impl.state_dict()

    def load_state_dict(self, sd: dict) -> None:
        if self._backend_impl is None:
            raise RuntimeError("Engine.load_state_dict() called before load_model().")
        self._backend_impl.load_state_dict(sd)

    def export_bundle(self, export_dir: str, exact: bool = True) -> str:
        """Writes the current state as a bundle (config.json + .bin files, the
        reference's GpuBackend.export_bundle format) plus, with `exact`, a
        resume record; returns the path of config.json."""
        from oncolytica_b200.bundle import export_bundle

        return export_bundle(self, export_dir, exact=exact)

    def import_bundle(self, bundle_dir: str) -> None:
        """Loads a bundle written by export_bundle (exactly) or by the
        reference (through its recorded struct layout) into the loaded model."""
        from oncolytica_b200.bundle import import_bundle

        import_bundle(self, bundle_dir)

    def get_reductions(self) -> dict:
        return self._backend_impl.get_reductions()

    def sync_to_host(self) -> None:
        self._backend_impl.sync_to_host()

    def sync_to_device(self) -> None:
        self._backend_impl.sync_to_device()

    def _resolve_container_for(self, bound_method: Any) -> Any:
        sig = inspect.signature(bound_method)
        params = list(sig.parameters.values())
        if not params:
            return ()
        ann = params[0].annotation
        if isinstance(ann, type) and issubclass(ann, Cell):
            return self.cells
        return ()

    def __repr__(self) -> str:
        return f"Engine(backend={self.backend!r}, step={self._step}, cells={len(self.cells)})"
