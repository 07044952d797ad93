"""CudaBackend: the reference's backend protocol
(ISimulationBackend, framework/src/oncolytica/core/runtime/_backend.py:7-36)
implemented on libolc.so.

State lives on the device in torch tensors laid out as columns (one array per
scalar field, three per vec3), double-buffered for the sort permute and the
rule kernels; chemistry fields are float32 arrays (x fastest) with a ping-pong
partner and an optional sink.  torch owns the memory; libolc borrows the
pointers.  Replaces GpuBackend (framework/src/oncolytica/gpu/runtime/_gpu_backend.py).
"""
from __future__ import annotations

import ctypes as C
from typing import Any, Optional

import numpy as np

from oncolytica_b200 import _lib
from oncolytica_b200._errors import CompilationError
from oncolytica_b200.compiler.emit_cuda import make_layout, pack_params, translate_model
from oncolytica_b200.engine import STORAGE_CODES
from oncolytica_b200 import _fieldcodec

# torch element type of each field storage code (OLC_FIELD_F32 / BF16 / F16)
FIELD_DTYPES = {0: lambda t: t.float32, 1: lambda t: t.bfloat16, 2: lambda t: t.float16, 3: lambda t: t.bfloat16,
                4: lambda t: t.float16}


def seed_rng(seed: int, idx: np.ndarray) -> np.ndarray:
    """Initial RNG states: MurmurHash3 fmix32 of seed*golden + index, forced odd
    (the device and the oracle use the same function)."""
    with np.errstate(over="ignore"):
        h = np.uint32(seed & 0xFFFFFFFF) * np.uint32(0x9E3779B9) + idx.astype(np.uint32)
        h = h.astype(np.uint32)
        h ^= h >> np.uint32(16)
        h *= np.uint32(0x85EBCA6B)
        h ^= h >> np.uint32(13)
        h *= np.uint32(0xC2B2AE35)
        h ^= h >> np.uint32(16)
    return h | np.uint32(1)


class PendingReadback:
    """The results of a collected step whose copies are queued on the stream
    (``Engine.run_step(collect_metrics=True, wait=False)``): ``result()``
    waits for those copies only, checks the device status word they carry,
    writes the metric values into the engine's metrics object (unless a newer
    step's are already there) and returns them as a dict."""

    def __init__(self, backend: "CudaBackend", ticket: int):
        self._backend = backend
        self.ticket = ticket
        self._values: dict | None = None
        self.counters: dict | None = None

    def result(self) -> dict:
        if self._values is not None:
            return self._values
        be = self._backend
        if self in be._pending:
            be._pending.remove(self)
        words, c = be._take_readback(self.ticket)
        self._values = be._decode_metrics(words)
        self.counters = {"n_agents": c.n_agents, "births": c.births, "deaths": c.deaths, "status": c.status,
                         "steps": c.steps, "agent_steps": c.agent_steps}
        be._apply_metrics(self.ticket, self._values)
        be.status.report(c.status)
        return self._values


class CudaBackend:
    """ISimulationBackend on CUDA: compile / run_step / sync_to_host / sync_to_device / get_metrics."""

    def __init__(self, engine: Any) -> None:
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("oncolytica_b200 needs a CUDA device: the step has no CPU implementation")
        self.engine = engine
        self.torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.lib = _lib.load()
        self.handle = C.c_void_p()
        self.layout = None
        self.program = None
        self.cols_dev: list[tuple[Any, Any]] = []
        self.fields_dev: list[tuple[Any, Any, Any]] = []
        self.comp_dev: list[Any] = []
        self.tissue_dev = None
        self.tissue_pair = None
        self._params_dirty = True
        self._last_reductions: dict | None = None
        self._pending: list = []          # PendingReadback, oldest first
        self._applied_ticket = 0          # newest readback written into the engine's metrics
        self.status = _lib.StatusWatch(lambda: self.counters()["status"], "CudaBackend.run_steps",
                                       every=engine.status_check_every, policy=engine.on_device_status)

    # ---- helpers -------------------------------------------------------------
    def _check(self, rc: int) -> None:
        if rc != _lib.OLC_OK:
            raise _lib.OlcError(rc, _lib.last_error(self.handle))

    def _stream(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def _torch_dtype(self, dt):
        t = self.torch
        return t.float32 if dt == np.float32 else t.int32

    # ---- ISimulationBackend ---------------------------------------------------
    def compile(self, sim: Any) -> None:
        eng = self.engine
        spec = sim._spec
        contact = eng._contact
        radius_field = contact.radius if (contact and isinstance(contact.radius, str)) else None
        self.layout = L = make_layout(spec, radius_field)
        if eng._cell_rules or eng._metric_rules or eng._tissue_rules or eng._chemistry_rules:
            self.program = translate_model(sim, L, radius_field)
        cap = eng.max_agents
        tdims = tuple(int(v) for v in eng.tissue_shape)
        cdims = tuple(int(v) for v in eng.chemistry_shape)
        lo = eng.domain_lo or (0.0, 0.0, 0.0)
        hi = eng.domain_hi or tuple(d * eng.tissue_voxel_size for d in tdims)
        g = _lib.OlcGeom()
        g.tissue_dims[:] = tdims
        g.tissue_voxel_size = eng.tissue_voxel_size
        g.chem_dims[:] = cdims
        g.chem_voxel_size = eng.chemistry_voxel_size
        g.domain_lo[:] = lo
        g.domain_hi[:] = hi
        caps = _lib.OlcCaps()
        caps.max_agents = cap
        caps.n_agent_fields = len(L.cell_cols)
        caps.n_fields = len(L.chem_fields)
        state_col = -1
        for i, (col, _, dt) in enumerate(L.cell_cols):
            if col == "state" and dt == np.int32:
                state_col = i
        caps.state_field = state_col
        caps.radial_bin_width = eng.tissue_voxel_size
        caps.center[:] = tuple((a + b) * 0.5 for a, b in zip(lo, hi))
        caps.dt = eng.dt
        self._check(self.lib.olc_create(C.byref(g), C.byref(caps), C.byref(self.handle)))
        self.geom, self.caps = g, caps
        torch = self.torch
        for i, (col, _, dt) in enumerate(L.cell_cols):
            a = torch.zeros(cap, dtype=self._torch_dtype(dt), device=self.device)
            b = torch.zeros(cap, dtype=self._torch_dtype(dt), device=self.device)
            self.cols_dev.append((a, b))
            self._check(self.lib.olc_bind_agent_column(self.handle, i, C.c_void_p(a.data_ptr()),
                                                       C.c_void_p(b.data_ptr())))
        nvox = int(np.prod(cdims))
        sinks = self.program.sink_fields if self.program else set()
        self.comp_dev = []
        # what each field's 16-bit elements hold (OLC_ENC_*), fixed at load
        self.field_enc = [eng.field_encoding(name) for name in L.chem_fields]
        for i, name in enumerate(L.chem_fields):
            spec_d = eng._diffusion.get(name)
            storage = STORAGE_CODES[spec_d.storage] if spec_d is not None else 0
            fdt = FIELD_DTYPES[storage](torch)
            a = torch.zeros(nvox, dtype=fdt, device=self.device)
            b = torch.zeros(nvox, dtype=fdt, device=self.device)
            s = torch.zeros(nvox, dtype=torch.float32, device=self.device) if name in sinks else None
            comp = torch.zeros(nvox, dtype=torch.float32, device=self.device) if storage else None
            self.fields_dev.append((a, b, s))
            self.comp_dev.append(comp)
            d = _lib.OlcDiffusion()
            d.storage = storage
            d.encoding = self.field_enc[i]
            if spec_d is None:
                if name in sinks:
                    raise ValueError(f"sink_at(...).{name} needs Engine.setup_diffusion({name!r}, ...)")
                d.substeps = 0  # static field: read by rules, never updated
            else:
                d.diffusion = spec_d.diffusion
                d.decay = spec_d.decay
                d.boundary = spec_d.boundary
                d.substeps = eng.substeps_for(name)
                d.has_sink = int(s is not None)
            self._check(self.lib.olc_bind_field_ex(self.handle, i, C.c_void_p(a.data_ptr()),
                                                   C.c_void_p(b.data_ptr()),
                                                   C.c_void_p(s.data_ptr()) if s is not None else None,
                                                   C.c_void_p(comp.data_ptr()) if comp is not None else None,
                                                   C.byref(d)))
        ct = _lib.OlcContact()
        if contact is not None:
            ct.enabled = 1
            if radius_field is not None:
                ct.radius_field = L.col_index(radius_field)
                ct.radius_const = 0.0
            else:
                ct.radius_field = -1
                ct.radius_const = float(contact.radius)
            ct.stiffness, ct.mobility = contact.stiffness, contact.mobility
            ct.max_disp, ct.margin = contact.max_disp, contact.margin
        self._check(self.lib.olc_set_contact(self.handle, C.byref(ct)))
        self.pins_dev = None
        if eng._vessel is not None:
            _, _, _, value, names = eng._vessel
            if names is None:
                names = [n for n in L.chem_fields
                         if n in eng._diffusion and STORAGE_CODES[eng._diffusion[n].storage] == 0]
            idx = eng.vessel_voxels()
            self.pins_dev = self.torch.from_numpy(idx.view(np.int32).copy()).to(self.device)
            for name in names:
                if name not in L.chem_fields:
                    raise ValueError(f"setup_vessel: no chemistry field {name!r}")
                self._check(self.lib.olc_set_pinned(self.handle, L.chem_fields.index(name),
                                                    C.c_void_p(self.pins_dev.data_ptr()), len(idx), value))
        if contact is not None and contact.mechanics:
            m = _lib.OlcMechanics()
            m.enabled = 1
            m.state_field = -1
            if contact.state is not None:
                for i, (col, _, dt) in enumerate(L.cell_cols):
                    if col == contact.state and dt == np.int32:
                        m.state_field = i
                if m.state_field < 0 and contact.necrotic_factor != 1.0:
                    raise ValueError(f"setup_contact: no ol.i32 cell field {contact.state!r} for the necrotic test")
            m.necrotic_factor = contact.necrotic_factor
            m.adhesion_stiffness = contact.adhesion_stiffness
            m.adhesion_range = contact.adhesion_range
            m.velocity_field = -1
            if contact.velocity is not None:
                try:
                    m.velocity_field = L.col_index(f"{contact.velocity}.x")
                except KeyError:
                    raise ValueError(f"setup_contact: velocity needs an ol.vec3 cell field {contact.velocity!r}")
            m.damping = contact.damping
            m.max_speed = contact.max_speed if contact.max_speed is not None else 0.8 * eng.tissue_voxel_size
            m.species_field = m.rng_field = m.o2_field = m.glucose_field = -1
            if contact.motion:
                m.n_species = len(contact.species)
                for i, (a, b, c) in enumerate(contact.species):
                    m.species[i].chemotaxis_o2, m.species[i].chemotaxis_glucose, m.species[i].move_prob = a, b, c
                m.chemo_force = contact.chemo_force
                m.motility_impulse = contact.motility_impulse
                if contact.species_field is not None:
                    try:
                        m.species_field = L.col_index(contact.species_field)
                    except KeyError:
                        raise ValueError(f"setup_contact: no cell field {contact.species_field!r} for the species")
                if any(rec[2] != 0.0 for rec in contact.species):
                    m.rng_field = L.col_index("_rng_state")
                if any(rec[0] != 0.0 or rec[1] != 0.0 for rec in contact.species):
                    names = list(contact.chemo_fields)
                    if names == [None, None]:
                        names = (list(L.chem_fields) + [None, None])[:2]
                    for attr, name in zip(("o2_field", "glucose_field"), names):
                        if name is not None:
                            if name not in L.chem_fields:
                                raise ValueError(f"setup_contact: no chemistry field {name!r} for chemotaxis")
                            setattr(m, attr, L.chem_fields.index(name))
            self._check(self.lib.olc_set_mechanics(self.handle, C.byref(m)))
        if self.program is not None:
            names = (C.c_char_p * len(self.program.kernels))(*[k.encode() for k, _ in self.program.kernels])
            kinds = (C.c_int * len(self.program.kernels))(*[kind for _, kind in self.program.kernels])
            self._check(self.lib.olc_set_rule_source(self.handle, self.program.source.encode(), names, kinds,
                                                     len(self.program.kernels), _lib.CSRC_DIR.encode()))
            if any(kind >= 2 for _, kind in self.program.kernels):
                if any(kind == 3 for _, kind in self.program.kernels) and any(
                        d.storage != "f32" for d in eng._diffusion.values()):
                    raise CompilationError("chemistry rules need FP32 chemistry fields (setup_diffusion storage='f32')")
                its = (C.c_int * len(self.program.kernels))(*self.program.iterations)
                self._check(self.lib.olc_set_rule_iterations(self.handle, its, len(self.program.kernels)))
        self._check(self.lib.olc_set_user_metrics_size(self.handle, 4 * max(1, len(L.metrics))))
        self.upload_params()
        self.sync_to_device()
        self.set_graphs(self.engine.use_graphs)

    def upload_params(self) -> None:
        sim = self.engine._sim
        blob = pack_params(self.layout, sim._params)
        buf = C.create_string_buffer(blob, len(blob))
        self._check(self.lib.olc_set_params(self.handle, C.cast(buf, C.c_void_p), len(blob), self._stream()))

    def run_step(self, collect_metrics: bool = False, wait: bool = True) -> Optional["PendingReadback"]:
        return self.run_steps(1, collect_metrics, wait)

    def run_steps(self, n: int, collect_metrics: bool = False, wait: bool = True) -> Optional["PendingReadback"]:
        """n steps; the device status word is checked every
        ``Engine.status_check_every`` steps and with every collected step's
        results (StatusWatch: DeviceStatusError on new bits).  A collected
        step queues the copies of its metric accumulators and counters
        (olc_queue_readback); ``wait`` takes them at once, otherwise the
        returned PendingReadback takes them when asked, so that the caller
        can queue the next step first."""
        self.status.every = max(1, int(self.engine.status_check_every))
        self.status.policy = self.engine.on_device_status
        chunks = list(self.status.chunks(n))
        pend = None
        for i, k in enumerate(chunks):
            last = i == len(chunks) - 1
            self._check(self.lib.olc_step(self.handle, int(k), int(bool(collect_metrics and last)), self._stream()))
            if collect_metrics and last:
                pend = self._queue_readback()
                self.status.since = 0
            else:
                self.status.after(k)
        if pend is not None and wait:
            pend.result()
            return None
        return pend

    def _queue_readback(self) -> "PendingReadback":
        # a ticket must be taken before READBACK_SLOTS later ones are queued
        while len(self._pending) >= _lib.READBACK_SLOTS - 1:
            self._pending[0].result()
        t = C.c_uint64()
        self._check(self.lib.olc_queue_readback(self.handle, self._stream(), C.byref(t)))
        pend = PendingReadback(self, int(t.value))
        self._pending.append(pend)
        return pend

    def resolve_pending(self) -> None:
        """Takes every queued readback (oldest first)."""
        while self._pending:
            self._pending[0].result()

    def _take_readback(self, ticket: int) -> tuple:
        nm = max(1, len(self.layout.metrics))
        raw = (C.c_uint32 * nm)()
        c = _lib.OlcCounters()
        self._check(self.lib.olc_take_readback(self.handle, ticket, C.cast(raw, C.c_void_p), 4 * nm, C.byref(c)))
        return np.frombuffer(bytes(raw), dtype=np.uint32), c

    def _decode_metrics(self, words) -> dict:
        out = {}
        for name, (slot, ty) in self.layout.metrics.items():
            w = words[slot:slot + 1]
            if ty == "f32":
                out[name] = np.float32(w.view(np.float32)[0])
            elif ty == "u32":
                out[name] = int(w[0])
            elif ty == "bool":
                out[name] = bool(w.view(np.int32)[0])
            else:
                out[name] = int(w.view(np.int32)[0])
        return out

    def _apply_metrics(self, ticket: int, values: dict) -> None:
        """Writes a readback's metric values into the engine's metrics object
        unless a newer readback has already been written there."""
        if ticket < self._applied_ticket:
            return
        self._applied_ticket = ticket
        m = self.engine._metrics
        for name, v in values.items():
            object.__setattr__(m, name, v)
        self._last_reductions = None

    def get_metrics(self) -> Any:
        self.resolve_pending()
        return self.engine._metrics

    def counters(self) -> dict:
        c = _lib.OlcCounters()
        self._check(self.lib.olc_read_counters(self.handle, C.byref(c), self._stream()))
        return {"n_agents": c.n_agents, "births": c.births, "deaths": c.deaths, "status": c.status,
                "steps": c.steps, "agent_steps": c.agent_steps}

    def set_graphs(self, enable: bool) -> None:
        self._check(self.lib.olc_set_graphs(self.handle, int(bool(enable))))

    # ---- tuning (olc.h OlcTuning; oncolytica_b200.autotune measures it) -------
    def set_tuning(self, stencil_tile=(8, 8), contact_variant: int = _lib.OLC_CONTACT_FLAT,
                   batch_tile_depth: int = 16, stencil_pair=(0, 0), l2_keep_pct: int = 0) -> None:
        """Kernel shapes and variants (olc_set_tuning): the FP32 stencil tile
        (rows, planes), the contact walk, the batched tile depth,
        ``stencil_pair`` = (threads per CTA, planes per CTA) of the
        two-substeps-per-pass kernel ((0, 0): one substep per pass), and the
        share of an FP32 field's planes kept in L2 across substeps by
        eviction hints (``l2_keep_pct``, 0: none)."""
        t = _lib.OlcTuning(int(stencil_tile[0]), int(stencil_tile[1]), int(contact_variant), int(batch_tile_depth),
                           int(stencil_pair[0]), int(stencil_pair[1]), int(l2_keep_pct))
        self._check(self.lib.olc_set_tuning(self.handle, C.byref(t)))

    def get_tuning(self) -> dict:
        t = _lib.OlcTuning()
        self._check(self.lib.olc_get_tuning(self.handle, C.byref(t)))
        return {"stencil_tile": (t.stencil_tile_y, t.stencil_tile_z), "contact_variant": t.contact_variant,
                "batch_tile_depth": t.batch_tile_depth,
                "stencil_pair": (t.stencil_pair_threads, t.stencil_pair_planes), "l2_keep_pct": t.stencil_l2_keep_pct}

    def has_tma_fields(self) -> bool:
        """Whether a diffusing FP32 field takes the TMA substep (the tuned tile)."""
        eng = self.engine
        return any(STORAGE_CODES[d.storage] == 0 and eng.substeps_for(n) > 0 for n, d in eng._diffusion.items())

    def mech_enabled(self) -> bool:
        c = self.engine._contact
        return bool(c is not None and c.mechanics)

    def set_profiling(self, enable: bool) -> None:
        self._check(self.lib.olc_set_profiling(self.handle, int(bool(enable))))

    def profile(self) -> dict:
        p = _lib.OlcProfile()
        self._check(self.lib.olc_read_profile(self.handle, C.byref(p)))
        return {k: getattr(p, k) for k, _ in _lib.OlcProfile._fields_}

    def get_reductions(self) -> dict:
        r = _lib.OlcReductions()
        self._check(self.lib.olc_read_reductions(self.handle, C.byref(r), self._stream()))
        n = len(self.layout.chem_fields)
        return {"n_live": r.n_live, "state_counts": list(r.state_counts), "radial_hist": list(r.radial_hist),
                "sum_pos": list(r.sum_pos), "sum_r2": r.sum_r2, "max_r": r.max_r,
                "field_mass": {f: r.field_mass[i] for i, f in enumerate(self.layout.chem_fields)},
                "field_min": {f: r.field_min[i] for i, f in enumerate(self.layout.chem_fields[:n])},
                "field_max": {f: r.field_max[i] for i, f in enumerate(self.layout.chem_fields[:n])}}

    def engine_metrics(self, state: str | None = "state", energy: str | None = None, speed: str | None = None,
                       csc: str | None = None, o2: str | None = None, glucose: str | None = None,
                       hypoxia_threshold: float = 0.1, crowd_threshold: int = 12) -> dict:
        """The engine's 23 metrics (engine/src/sim/readback.rs:25-50) of the
        current state, computed on the device (olc_engine_metrics).  Column
        and field names select what the engine reads from its fixed cell
        struct; a name the model lacks reads as absent (zero).  By default O2
        is the first chemistry field and glucose the second."""
        L = self.layout

        def col(name, dtype):
            if name is None:
                return -1
            for i, (c, _, dt) in enumerate(L.cell_cols):
                if c == name and dt == dtype:
                    return i
            return -1

        def field(name, default):
            if name is None:
                return default if default < len(L.chem_fields) else -1
            return L.chem_fields.index(name) if name in L.chem_fields else -1

        sp = _lib.OlcEngineMetricsSpec()
        sp.state_field = col(state, np.int32)
        sp.energy_field = col(energy, np.float32)
        sp.speed_field = col(None if speed is None else f"{speed}.x", np.float32)  # a vec3: x, y, z columns
        sp.csc_field = col(csc, np.int32)
        sp.o2_field = field(o2, 0)
        sp.glucose_field = field(glucose, 1)
        sp.hypoxia_threshold = hypoxia_threshold
        sp.crowd_threshold = int(crowd_threshold)
        sp.center[:] = tuple(self.caps.center)
        out = (C.c_double * _lib.OLC_ENGINE_METRICS)()
        self._check(self.lib.olc_engine_metrics(self.handle, C.byref(sp), out, self._stream()))
        return dict(zip(_lib.ENGINE_METRIC_NAMES, list(out)))

    def _current(self) -> tuple[int, int]:
        a, f = C.c_int(), C.c_int()
        self._check(self.lib.olc_current_buffers(self.handle, C.byref(a), C.byref(f)))
        return a.value, f.value

    def sync_to_device(self) -> None:
        """Host agents and fields -> device (replaces _gpu_backend.py:353-371)."""
        torch = self.torch
        eng = self.engine
        L = self.layout
        cols = eng.cells.columns(L.cell_class)
        n = len(next(iter(cols.values()))) if cols else 0
        if n > eng.max_agents:
            raise _lib.OlcError(_lib.OLC_ERR_CAPACITY, f"{n} agents exceed max_agents={eng.max_agents}")
        rng = cols.get("_rng_state", np.zeros(n, np.uint32)).astype(np.uint32)
        zero = rng == 0
        if zero.any():
            rng = rng.copy()
            rng[zero] = seed_rng(eng.seed, np.nonzero(zero)[0].astype(np.uint32))
        ab, fb = self._current()
        self.torch.cuda.synchronize(self.device)
        for i, (col, _, dt) in enumerate(L.cell_cols):
            host = rng if col == "_rng_state" else cols[col]
            arr = np.ascontiguousarray(host.astype(dt))
            if dt == np.uint32:
                arr = arr.view(np.int32)
            if n:
                self.cols_dev[i][ab][:n].copy_(torch.from_numpy(arr))
        for i, name in enumerate(L.chem_fields):
            host = np.asarray(eng.chemistry.column(name), dtype=np.float32)
            spec_d = eng._diffusion.get(name)
            if spec_d is not None:
                host = host.copy(order="F")
                b = np.float32(spec_d.boundary)
                host[0, :, :] = host[-1, :, :] = b
                host[:, 0, :] = host[:, -1, :] = b
                host[:, :, 0] = host[:, :, -1] = b
            flat = np.ascontiguousarray(host.ravel(order="F"))
            if eng._vessel is not None and spec_d is not None and (eng._vessel[4] is None or name in eng._vessel[4]) \
                    and STORAGE_CODES[spec_d.storage] == 0:
                flat = flat.copy()
                flat[eng.vessel_voxels()] = np.float32(eng._vessel[3])
            cur = (fb >> i) & 1
            dst = self.fields_dev[i][cur]
            if dst.dtype == torch.float32:
                dst.copy_(torch.from_numpy(flat))
            else:  # 16-bit elements of the field's encoding, rounded to nearest even
                bits = _fieldcodec.encode(flat, self._storage_code(i), self.field_enc[i], self._boundary(i))
                dst.view(torch.int16).copy_(torch.from_numpy(bits.view(np.int16)))
            if self.fields_dev[i][2] is not None:
                self.fields_dev[i][2].zero_()
            if self.comp_dev[i] is not None:
                self.comp_dev[i].zero_()
        self._upload_tissue()
        self.torch.cuda.synchronize(self.device)
        self._check(self.lib.olc_set_agent_count(self.handle, n, self._stream()))

    @property
    def _tissue_rules(self) -> bool:
        return self.program is not None and any(kind == 2 for _, kind in self.program.kernels)

    def _tissue_keys(self):
        from oncolytica_b200._geometry import get_tissue_voxel_key, voxel_table_size

        dims = self.engine.tissue_shape
        ix, iy, iz = np.meshgrid(*(np.arange(d) for d in dims), indexing="ij")
        keys = np.asarray(get_tissue_voxel_key(ix.ravel(), iy.ravel(), iz.ravel()), dtype=np.int64)
        return keys, voxel_table_size(dims)

    def _read_tissue(self) -> None:
        """Tissue rules' results back into the host Tissue grid."""
        eng = self.engine
        L = self.layout
        cur = C.c_int()
        self._check(self.lib.olc_current_tissue(self.handle, C.byref(cur)))
        packed = self.tissue_pair[cur.value].cpu().numpy()
        keys, _ = self._tissue_keys()
        shape = tuple(eng.tissue_shape)
        for i, (name, t) in enumerate(L.tissue_fields.items()):
            col = eng.tissue.column(name)
            raw = packed[i, keys]
            if col.dtype == np.float32:
                col[...] = raw.reshape(shape)
            else:
                col[...] = raw.view(np.int32).reshape(shape).astype(col.dtype)

    def _upload_tissue(self) -> None:
        """Tissue grid columns packed by tissue (Morton) key for tissue_at();
        with tissue rules, two such buffers (the rules write the other one)."""
        eng = self.engine
        L = self.layout
        if eng.tissue is None or not L.tissue_fields:
            return
        from oncolytica_b200._geometry import get_tissue_voxel_key, voxel_table_size

        dims = eng.tissue_shape
        v = voxel_table_size(dims)
        ix, iy, iz = np.meshgrid(*(np.arange(d) for d in dims), indexing="ij")
        keys = np.asarray(get_tissue_voxel_key(ix.ravel(), iy.ravel(), iz.ravel()), dtype=np.int64)
        packed = np.zeros((len(L.tissue_fields), v), dtype=np.float32)
        for i, name in enumerate(L.tissue_fields):
            col = np.asarray(eng.tissue.column(name))
            if col.dtype == np.float32:
                packed[i, keys] = col.ravel(order="C")
            else:
                packed[i].view(np.int32)[keys] = col.astype(np.int32).ravel(order="C")
        self.tissue_dev = self.torch.from_numpy(packed).to(self.device)
        if self._tissue_rules:
            self.tissue_pair = (self.tissue_dev, self.tissue_dev.clone())
            self._check(self.lib.olc_bind_tissue_pair(self.handle, C.c_void_p(self.tissue_pair[0].data_ptr()),
                                                      C.c_void_p(self.tissue_pair[1].data_ptr()),
                                                      len(L.tissue_fields), v * 4))
            return
        self._check(self.lib.olc_bind_tissue(self.handle, C.c_void_p(self.tissue_dev.data_ptr()),
                                             len(L.tissue_fields), v * 4))

    def sync_to_host(self) -> None:
        """Device -> host agents (live only) and fields (replaces _gpu_backend.py:373-405)."""
        eng = self.engine
        L = self.layout
        cnt = self.counters()
        rows = cnt["n_agents"]
        ab, fb = self._current()
        self.torch.cuda.synchronize(self.device)
        cols = {}
        life = self._life(rows)
        keep = life == 0
        for i, (col, _, dt) in enumerate(L.cell_cols):
            a = self.cols_dev[i][ab][:rows].cpu().numpy()
            if dt == np.uint32:
                a = a.view(np.uint32)
            cols[col] = a[keep].copy()
        eng.cells._set_columns(cols, L.cell_class)
        for i, name in enumerate(L.chem_fields):
            flat = self._field_values(i, fb)
            eng.chemistry.column(name)[...] = flat.reshape(eng.chemistry_shape, order="F")
        if self._tissue_rules and eng.tissue is not None and L.tissue_fields:
            self._read_tissue()

    def _storage_code(self, i: int) -> int:
        spec_d = self.engine._diffusion.get(self.layout.chem_fields[i])
        return STORAGE_CODES[spec_d.storage] if spec_d is not None else 0

    def _boundary(self, i: int) -> float:
        spec_d = self.engine._diffusion.get(self.layout.chem_fields[i])
        return float(spec_d.boundary) if spec_d is not None else 0.0

    def field_codec(self, name: str) -> tuple[int, int, float]:
        """(storage code, encoding code, boundary value) of a field's elements."""
        i = self.layout.chem_fields.index(name)
        return self._storage_code(i), self.field_enc[i], self._boundary(i)

    def _field_values(self, i: int, fb: int) -> np.ndarray:
        """Field i as float32 on the host; for 16-bit storage the stored value
        plus its FP32 rounding residual (what the next reaction continues from),
        decoded from the field's encoding."""
        cur = (fb >> i) & 1
        t = self.fields_dev[i][cur]
        if self.comp_dev[i] is None:
            return t.cpu().numpy()
        bits = t.cpu().view(self.torch.int16).numpy().view(np.uint16)
        return _fieldcodec.decode(bits, self._storage_code(i), self.field_enc[i], self._boundary(i),
                                  self.comp_dev[i].cpu().numpy())

    def _life(self, rows: int) -> np.ndarray:
        buf = (C.c_uint8 * max(rows, 1))()
        self._check(self.lib.olc_read_life(self.handle, C.cast(buf, C.c_void_p), rows, self._stream()))
        return np.frombuffer(bytes(buf), dtype=np.uint8)[:rows]

    def snapshot(self) -> dict:
        """Raw device state: every row in use (dead rows included, in device
        order) with its life flag, the current fields and their sinks."""
        cnt = self.counters()
        rows = cnt["n_agents"]
        ab, fb = self._current()
        self.torch.cuda.synchronize(self.device)
        out = {"rows": rows, "life": self._life(rows).copy(), "cols": {}, "fields": {}, "sinks": {}}
        for i, (col, _, dt) in enumerate(self.layout.cell_cols):
            a = self.cols_dev[i][ab][:rows].cpu().numpy()
            out["cols"][col] = a.view(np.uint32).copy() if dt == np.uint32 else a.copy()
        for i, name in enumerate(self.layout.chem_fields):
            t = self.fields_dev[i][(fb >> i) & 1]
            out["fields"][name] = t.cpu().numpy().copy() if t.dtype == self.torch.float32 else \
                t.cpu().view(self.torch.int16).numpy().view(np.uint16).copy()
            s = self.fields_dev[i][2]
            out["sinks"][name] = s.cpu().numpy().copy() if s is not None else None
            c = self.comp_dev[i]
            if c is not None:
                out.setdefault("residuals", {})[name] = c.cpu().numpy().copy()
        if self._tissue_rules and self.engine.tissue is not None and self.layout.tissue_fields:
            # the tissue grid the rules update, as (X, Y, Z) arrays per field
            cur = C.c_int()
            self._check(self.lib.olc_current_tissue(self.handle, C.byref(cur)))
            packed = self.tissue_pair[cur.value].cpu().numpy()
            keys, _ = self._tissue_keys()
            shape = tuple(self.engine.tissue_shape)
            out["tissue"] = {}
            for i, (name, t) in enumerate(self.layout.tissue_fields.items()):
                raw = packed[i, keys]
                out["tissue"][name] = (raw if self.engine.tissue.column(name).dtype == np.float32
                                       else raw.view(np.int32)).reshape(shape).copy()
        return out

    # ---- checkpoints (no counterpart in the reference, which has no resume) ----
    def _layout_signature(self) -> dict:
        L = self.layout
        storages = []
        for i in range(len(L.chem_fields)):
            t = self.fields_dev[i][0]
            storages.append(str(t.dtype).replace("torch.", ""))
        return {"cols": [[c, np.dtype(dt).name] for c, _, dt in L.cell_cols],
                "fields": list(L.chem_fields), "field_dtypes": storages,
                "field_encodings": [int(e) for e in self.field_enc],
                "sinks": [self.fields_dev[i][2] is not None for i in range(len(L.chem_fields))],
                "chem_dims": [int(v) for v in self.geom.chem_dims], "tissue_dims": [int(v) for v in self.geom.tissue_dims],
                "max_agents": int(self.caps.max_agents)}

    def state_dict(self) -> dict:
        """Everything the next step reads, as host arrays: the live agents (in
        device order, every column including _rng_state), each field's current
        buffer as stored (FP32 values or 16-bit bit patterns), its pending sink
        and 16-bit residuals, the step counters and the parameters.
        load_state_dict() of this on an engine built the same way continues
        bit for bit as this one would: the next sort drops dead rows keeping
        the survivors' order, so storing the survivors compacted changes
        nothing."""
        torch = self.torch
        cnt = self.counters()
        rows = cnt["n_agents"]
        ab, fb = self._current()
        torch.cuda.synchronize(self.device)
        keep = self._life(rows) == 0
        cols = {}
        for i, (col, _, dt) in enumerate(self.layout.cell_cols):
            a = self.cols_dev[i][ab][:rows].cpu().numpy()
            cols[col] = (a.view(np.uint32) if dt == np.uint32 else a)[keep].copy()
        fields, sinks, residuals = {}, {}, {}
        for i, name in enumerate(self.layout.chem_fields):
            t = self.fields_dev[i][(fb >> i) & 1]
            fields[name] = t.cpu().numpy().copy() if t.dtype == torch.float32 else \
                t.cpu().view(torch.int16).numpy().view(np.uint16).copy()
            sk = self.fields_dev[i][2]
            sinks[name] = sk.cpu().numpy().copy() if sk is not None else None
            c = self.comp_dev[i]
            residuals[name] = c.cpu().numpy().copy() if c is not None else None
        ss = _lib.OlcStepState()
        self._check(self.lib.olc_get_step_state(self.handle, C.byref(ss), self._stream()))
        params = self.engine._sim._params
        tissue = None
        if self._tissue_rules and getattr(self, "tissue_pair", None) is not None:
            cur = C.c_int()
            self._check(self.lib.olc_current_tissue(self.handle, C.byref(cur)))
            tissue = self.tissue_pair[cur.value].cpu().numpy().copy()  # packed by tissue key
        return {"format": "oncolytica_b200.state/1", "layout": self._layout_signature(), "cols": cols,
                "fields": fields, "sinks": sinks, "residuals": residuals, "tissue": tissue,
                "step_state": {"steps": int(ss.steps), "agent_steps": int(ss.agent_steps),
                               "field_step": int(ss.field_step), "status": int(ss.status)},
                "engine_step": int(self.engine._step),
                "params": {k: getattr(params, k) for k in params.__dataclass_fields__}}

    def load_state_dict(self, sd: dict) -> None:
        """Writes a state_dict() into this engine's current buffers (the model,
        geometry, field storages and capacity must match)."""
        torch = self.torch
        if sd.get("format") != "oncolytica_b200.state/1":
            raise ValueError(f"not a checkpoint state: format {sd.get('format')!r}")
        mine = self._layout_signature()
        theirs = sd["layout"]
        theirs = dict(theirs)
        theirs.setdefault("field_encodings", [0] * len(theirs["fields"]))
        for k in ("cols", "fields", "field_dtypes", "field_encodings", "sinks", "chem_dims", "tissue_dims"):
            if [list(x) if isinstance(x, (list, tuple)) else x for x in theirs[k]] != \
                    [list(x) if isinstance(x, (list, tuple)) else x for x in mine[k]]:
                raise ValueError(f"checkpoint does not match this engine: {k} {theirs[k]} != {mine[k]}")
        L = self.layout
        n = len(sd["cols"]["pos.x"])
        if n > self.caps.max_agents:
            raise _lib.OlcError(_lib.OLC_ERR_CAPACITY, f"{n} agents exceed max_agents={self.caps.max_agents}")
        if sd.get("params"):
            p = self.engine._sim._params
            for k, v in sd["params"].items():
                object.__setattr__(p, k, v)
            self.upload_params()
        ab, fb = self._current()
        torch.cuda.synchronize(self.device)
        for i, (col, _, dt) in enumerate(L.cell_cols):
            a = np.ascontiguousarray(sd["cols"][col]).astype(dt, copy=False)
            if dt == np.uint32:
                a = a.view(np.int32)
            if n:
                self.cols_dev[i][ab][:n].copy_(torch.from_numpy(a))
        for i, name in enumerate(L.chem_fields):
            t = self.fields_dev[i][(fb >> i) & 1]
            raw = np.ascontiguousarray(sd["fields"][name])
            if t.dtype == torch.float32:
                t.copy_(torch.from_numpy(raw.astype(np.float32, copy=False)))
            else:
                t.view(torch.int16).copy_(torch.from_numpy(raw.astype(np.uint16, copy=False).view(np.int16)))
            sk = self.fields_dev[i][2]
            if sk is not None:
                v = sd["sinks"].get(name)
                sk.copy_(torch.from_numpy(np.ascontiguousarray(v, dtype=np.float32))) if v is not None else sk.zero_()
            c = self.comp_dev[i]
            if c is not None:
                v = sd["residuals"].get(name)
                c.copy_(torch.from_numpy(np.ascontiguousarray(v, dtype=np.float32))) if v is not None else c.zero_()
        if sd.get("tissue") is not None and getattr(self, "tissue_pair", None) is not None:
            cur = C.c_int()
            self._check(self.lib.olc_current_tissue(self.handle, C.byref(cur)))
            self.tissue_pair[cur.value].copy_(torch.from_numpy(np.ascontiguousarray(sd["tissue"])))
        torch.cuda.synchronize(self.device)
        self._check(self.lib.olc_set_agent_count(self.handle, n, self._stream()))
        ss = _lib.OlcStepState()
        st = sd["step_state"]
        ss.steps, ss.agent_steps = st["steps"], st["agent_steps"]
        ss.field_step, ss.status = st["field_step"], st["status"]
        self._check(self.lib.olc_set_step_state(self.handle, C.byref(ss), self._stream()))
        self.engine._step = int(sd.get("engine_step", st["steps"]))

    def field_tensor(self, name: str):
        """The device tensor currently holding chemistry field ``name`` (x fastest)."""
        _, fb = self._current()
        i = self.layout.chem_fields.index(name)
        return self.fields_dev[i][(fb >> i) & 1]

    def column_tensor(self, col: str):
        ab, _ = self._current()
        return self.cols_dev[self.layout.col_index(col)][ab]

    def close(self) -> None:
        """Destroys the library handle and drops the device tensors (their
        memory returns to torch's allocator)."""
        if self.handle:
            self.lib.olc_destroy(self.handle)
            self.handle = C.c_void_p()
        self._pending = []
        self.cols_dev, self.fields_dev, self.comp_dev = [], [], []
        self.tissue_dev = self.tissue_pair = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass
