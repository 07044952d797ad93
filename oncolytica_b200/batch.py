"""BatchEngine: many independent simulations of one model advanced together,
one launch per stage (libolc's batched mode; no counterpart in the
reference, which runs one simulation per engine).

Each member is an ordinary ``Engine`` configured as for a solo run
(geometry, chemistry, diffusion, contact, agents, dt, seed) and a model
instance of one shared model class carrying that member's ``Params``.  The
batch translates the model once, packs every member's agents and fields into
shared device buffers and steps them all with one handle.  Each member
reproduces its solo run bit for bit; ``sync_to_host`` writes the results back
into the member engines.
"""
from __future__ import annotations

import ctypes as C
from typing import Any, Sequence

import numpy as np

from oncolytica_b200 import _lib
from oncolytica_b200.backend import FIELD_DTYPES, seed_rng
from oncolytica_b200.engine import STORAGE_CODES
from oncolytica_b200 import _fieldcodec
from oncolytica_b200.compiler.emit_cuda import make_layout, pack_params, translate_model


class BatchEngine:
    """Drives ``engines[k]`` with model instance ``sims[k]`` in one batch."""

    def __init__(self, engines: Sequence[Any], sims: Sequence[Any], max_agents: int | None = None) -> None:
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("oncolytica_b200 needs a CUDA device: the step has no CPU implementation")
        if len(engines) == 0 or len(engines) != len(sims):
            raise ValueError("BatchEngine needs one model instance per engine")
        cls = type(sims[0])
        if any(type(s) is not cls for s in sims):
            raise ValueError("every member of a batch runs the same model class")
        self.torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.engines = list(engines)
        self.sims = list(sims)
        self.lib = _lib.load()
        self.handle = C.c_void_p()
        for eng, sim in zip(self.engines, self.sims):
            eng._prepare_model(sim)
        e0 = self.engines[0]
        for eng in self.engines[1:]:
            if eng.dt != e0.dt:
                raise ValueError("every member of a batch uses the same dt")
            if (eng._contact is None) != (e0._contact is None) or (eng._contact and eng._contact != e0._contact):
                raise ValueError("every member of a batch uses the same contact settings")
        self.max_agents = int(max_agents or sum(e.max_agents for e in self.engines))
        self.use_graphs = False
        self._step = 0
        self.status = _lib.StatusWatch(lambda: self.counters()["status"], "BatchEngine.run_steps",
                                       every=e0.status_check_every, policy=e0.on_device_status)
        self._compile()

    # ---- set-up ----------------------------------------------------------------
    def _check(self, rc: int) -> None:
        if rc != _lib.OLC_OK:
            raise _lib.OlcError(rc, _lib.last_error(self.handle))

    def _stream(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def _geom(self, eng) -> Any:
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
        return g

    def _compile(self) -> None:
        torch = self.torch
        e0, s0 = self.engines[0], self.sims[0]
        contact = e0._contact
        radius_field = contact.radius if (contact and isinstance(contact.radius, str)) else None
        self.layout = L = make_layout(s0._spec, radius_field, batched=True)
        self.program = (translate_model(s0, L, radius_field)
                        if (e0._cell_rules or e0._metric_rules or e0._chemistry_rules or e0._tissue_rules) else None)
        n = len(self.engines)
        geoms = (_lib.OlcGeom * n)(*[self._geom(e) for e in self.engines])
        caps = _lib.OlcCaps()
        caps.max_agents = self.max_agents
        caps.n_agent_fields = len(L.cell_cols)
        caps.n_fields = len(L.chem_fields)
        caps.state_field = -1
        for i, (col, _, dt) in enumerate(L.cell_cols):
            if col == "state" and dt == np.int32:
                caps.state_field = i
        caps.radial_bin_width = e0.tissue_voxel_size
        caps.dt = e0.dt
        self._check(self.lib.olc_create_batch(geoms, n, C.byref(caps), C.byref(self.handle)))
        offs = (C.c_uint64 * (n + 1))()
        self._check(self.lib.olc_batch_field_offsets(self.handle, offs))
        self.field_off = np.array(list(offs), dtype=np.int64)
        self.cols_dev = []
        for i, (col, _, dt) in enumerate(L.cell_cols):
            tdt = torch.float32 if dt == np.float32 else torch.int32
            a = torch.zeros(self.max_agents, dtype=tdt, device=self.device)
            b = torch.zeros(self.max_agents, dtype=tdt, device=self.device)
            self.cols_dev.append((a, b))
            self._check(self.lib.olc_bind_agent_column(self.handle, i, C.c_void_p(a.data_ptr()),
                                                       C.c_void_p(b.data_ptr())))
        nvox = int(self.field_off[-1])
        sinks = self.program.sink_fields if self.program else set()
        self.fields_dev = []
        self.comp_dev = []
        self.field_enc = []
        self.field_bval = []
        for i, name in enumerate(L.chem_fields):
            kinds = {e._diffusion[name].storage for e in self.engines if name in e._diffusion}
            if len(kinds) > 1:
                raise ValueError(f"every member of a batch stores field {name!r} with the same type")
            storage = STORAGE_CODES[kinds.pop()] if kinds else 0
            # what the 16-bit elements hold: one encoding (and, when encoded,
            # one boundary value) for every member
            encs = {e.field_encoding(name) for e in self.engines}
            if len(encs) > 1:
                raise ValueError(f"members resolve different encodings for field {name!r}; pass "
                                 "setup_diffusion(encoding=...) explicitly")
            enc = encs.pop()
            bvals = {float(e._diffusion[name].boundary) for e in self.engines if name in e._diffusion}
            if enc and len(bvals) > 1:
                raise ValueError(f"encoded field {name!r} needs one boundary value for every member")
            self.field_enc.append(enc)
            self.field_bval.append(bvals.pop() if bvals else 0.0)
            fdt = FIELD_DTYPES[storage](torch)
            a = torch.zeros(max(nvox, 1), dtype=fdt, device=self.device)
            b = torch.zeros(max(nvox, 1), dtype=fdt, device=self.device)
            s = torch.zeros(max(nvox, 1), dtype=torch.float32, device=self.device) if name in sinks else None
            comp = torch.zeros(max(nvox, 1), dtype=torch.float32, device=self.device) if storage else None
            self.fields_dev.append((a, b, s))
            self.comp_dev.append(comp)
            specs = (_lib.OlcDiffusion * n)()
            for k, eng in enumerate(self.engines):
                spec_d = eng._diffusion.get(name)
                d = specs[k]
                d.storage = storage
                d.encoding = enc
                if spec_d is None:
                    if name in sinks:
                        raise ValueError(f"sink_at(...).{name} needs Engine.setup_diffusion({name!r}, ...)")
                    d.substeps = 0
                else:
                    d.diffusion, d.decay, d.boundary = spec_d.diffusion, spec_d.decay, spec_d.boundary
                    d.substeps = eng.substeps_for(name)
                    d.has_sink = int(s is not None)
            self._check(self.lib.olc_bind_field_batch(self.handle, i, C.c_void_p(a.data_ptr()),
                                                      C.c_void_p(b.data_ptr()),
                                                      C.c_void_p(s.data_ptr()) if s is not None else None,
                                                      C.c_void_p(comp.data_ptr()) if comp is not None else None,
                                                      specs))
        ct = _lib.OlcContact()
        if contact is not None:
            ct.enabled = 1
            if radius_field is not None:
                ct.radius_field, ct.radius_const = L.col_index(radius_field), 0.0
            else:
                ct.radius_field, ct.radius_const = -1, float(contact.radius)
            ct.stiffness, ct.mobility = contact.stiffness, contact.mobility
            ct.max_disp, ct.margin = contact.max_disp, contact.margin
        self._check(self.lib.olc_set_contact(self.handle, C.byref(ct)))
        if self.program is not None:
            names = (C.c_char_p * len(self.program.kernels))(*[k.encode() for k, _ in self.program.kernels])
            kinds = (C.c_int * len(self.program.kernels))(*[kind for _, kind in self.program.kernels])
            self._check(self.lib.olc_set_rule_source(self.handle, self.program.source.encode(), names, kinds,
                                                     len(self.program.kernels), _lib.CSRC_DIR.encode()))
            if any(kind == 3 for _, kind in self.program.kernels):
                if any(d.storage != "f32" for e in self.engines for d in e._diffusion.values()):
                    from oncolytica_b200._errors import CompilationError

                    raise CompilationError("chemistry rules need FP32 chemistry fields (setup_diffusion storage='f32')")
                its = (C.c_int * len(self.program.kernels))(*self.program.iterations)
                self._check(self.lib.olc_set_rule_iterations(self.handle, its, len(self.program.kernels)))
        self.metrics_words = max(1, len(L.metrics))
        self._check(self.lib.olc_set_user_metrics_size(self.handle, 4 * self.metrics_words))
        self.upload_params()
        self.sync_to_device()

    def upload_params(self) -> None:
        blobs = [pack_params(self.layout, s._params) for s in self.sims]
        stride = len(blobs[0])
        raw = b"".join(blobs)
        buf = C.create_string_buffer(raw, len(raw))
        self._check(self.lib.olc_set_params_batch(self.handle, C.cast(buf, C.c_void_p), stride, self._stream()))

    def set_graphs(self, enable: bool) -> None:
        self.use_graphs = bool(enable)
        self._check(self.lib.olc_set_graphs(self.handle, int(self.use_graphs)))

    def set_tuning(self, stencil_tile=(8, 8), contact_variant: int = _lib.OLC_CONTACT_FLAT,
                   batch_tile_depth: int = 16, stencil_pair=(0, 0), l2_keep_pct: int = 0) -> None:
        """Kernel shapes and variants of the batch handle (olc_set_tuning)."""
        t = _lib.OlcTuning(int(stencil_tile[0]), int(stencil_tile[1]), int(contact_variant), int(batch_tile_depth),
                           int(stencil_pair[0]), int(stencil_pair[1]), int(l2_keep_pct))
        self._check(self.lib.olc_set_tuning(self.handle, C.byref(t)))

    def set_tile_depths(self, depths) -> None:
        """The batched FP32 substep tile depth of each member (8, 16, 32; 0 =
        the handle's); oncolytica_b200.autotune.tune_batch measures them."""
        arr = (C.c_int32 * len(self.engines))(*[int(d) for d in depths])
        self._check(self.lib.olc_set_batch_tile_depths(self.handle, arr, len(self.engines)))
        self.tile_depths = [int(d) for d in depths]

    def set_profiling(self, enable: bool) -> None:
        self._check(self.lib.olc_set_profiling(self.handle, int(bool(enable))))

    def profile(self) -> dict:
        p = _lib.OlcProfile()
        self._check(self.lib.olc_read_profile(self.handle, C.byref(p)))
        return {k: getattr(p, k) for k, _ in _lib.OlcProfile._fields_}

    # ---- stepping -------------------------------------------------------------
    def run_steps(self, n: int, collect_metrics: bool = False) -> None:
        self._step += n
        for eng in self.engines:
            eng._step += n
        chunks = list(self.status.chunks(n))
        for i, k in enumerate(chunks):
            last = i == len(chunks) - 1
            self._check(self.lib.olc_step(self.handle, int(k), int(bool(collect_metrics and last)), self._stream()))
            if collect_metrics and last:
                self._read_metrics()
            self.status.after(k, synced=collect_metrics and last)

    def run_step(self, collect_metrics: bool = False) -> None:
        self.run_steps(1, collect_metrics)

    def counters(self) -> dict:
        c = _lib.OlcCounters()
        self._check(self.lib.olc_read_counters(self.handle, C.byref(c), self._stream()))
        return {"n_agents": c.n_agents, "births": c.births, "deaths": c.deaths, "status": c.status,
                "steps": c.steps, "agent_steps": c.agent_steps}

    def _read_metrics(self) -> None:
        n = len(self.engines)
        raw = (C.c_uint32 * (n * self.metrics_words))()
        self._check(self.lib.olc_read_user_metrics_batch(self.handle, C.cast(raw, C.c_void_p), 4 * self.metrics_words,
                                                         self._stream()))
        words = np.frombuffer(bytes(raw), dtype=np.uint32).reshape(n, self.metrics_words)
        for k, eng in enumerate(self.engines):
            m = eng._metrics
            for name, (slot, ty) in self.layout.metrics.items():
                w = words[k, slot:slot + 1]
                if ty == "f32":
                    v = np.float32(w.view(np.float32)[0])
                elif ty == "u32":
                    v = int(w[0])
                elif ty == "bool":
                    v = bool(w.view(np.int32)[0])
                else:
                    v = int(w.view(np.int32)[0])
                object.__setattr__(m, name, v)

    def get_reductions(self) -> list[dict]:
        n = len(self.engines)
        rs = (_lib.OlcReductions * n)()
        self._check(self.lib.olc_read_reductions_batch(self.handle, rs, self._stream()))
        out = []
        for r in rs:
            out.append({"n_live": r.n_live, "state_counts": list(r.state_counts),
                        "radial_hist": list(r.radial_hist), "sum_pos": list(r.sum_pos), "sum_r2": r.sum_r2,
                        "max_r": r.max_r,
                        "field_mass": {f: r.field_mass[i] for i, f in enumerate(self.layout.chem_fields)},
                        "field_min": {f: r.field_min[i] for i, f in enumerate(self.layout.chem_fields)},
                        "field_max": {f: r.field_max[i] for i, f in enumerate(self.layout.chem_fields)}})
        return out

    # ---- state transfer ---------------------------------------------------------
    def _agent_buf(self) -> int:
        a, f = C.c_int(), C.c_int()
        self._check(self.lib.olc_current_buffers(self.handle, C.byref(a), C.byref(f)))
        return a.value

    def _field_parity(self) -> np.ndarray:
        n, nf = len(self.engines), len(self.layout.chem_fields)
        buf = (C.c_uint8 * max(1, n * nf))()
        self._check(self.lib.olc_read_field_parity(self.handle, buf, self._stream()))
        return np.frombuffer(bytes(buf), dtype=np.uint8)[:n * nf].reshape(n, max(nf, 1) if nf else 0)

    def _life(self, rows: int) -> np.ndarray:
        buf = (C.c_uint8 * max(rows, 1))()
        self._check(self.lib.olc_read_life(self.handle, C.cast(buf, C.c_void_p), rows, self._stream()))
        return np.frombuffer(bytes(buf), dtype=np.uint8)[:rows]

    def sync_to_device(self) -> None:
        """Every member's host agents and fields -> the shared device buffers
        (agents simulation-major; each member's RNG states seeded as in its solo run)."""
        torch = self.torch
        L = self.layout
        parts: dict[str, list] = {col: [] for col, _, _ in L.cell_cols}
        for k, eng in enumerate(self.engines):
            cols = eng.cells.columns(L.cell_class)
            n = len(next(iter(cols.values()))) if cols else 0
            rng = cols.get("_rng_state", np.zeros(n, np.uint32)).astype(np.uint32)
            zero = rng == 0
            if zero.any():
                rng = rng.copy()
                rng[zero] = seed_rng(eng.seed, np.nonzero(zero)[0].astype(np.uint32))
            for col, _, dt in L.cell_cols:
                if col == "_rng_state":
                    parts[col].append(rng)
                elif col == "_sim":
                    parts[col].append(np.full(n, k, np.uint32))
                else:
                    parts[col].append(np.asarray(cols[col]).astype(dt))
        total = sum(len(p) for p in parts[L.cell_cols[0][0]])
        if total > self.max_agents:
            raise _lib.OlcError(_lib.OLC_ERR_CAPACITY, f"{total} agents exceed the batch capacity {self.max_agents}")
        ab = self._agent_buf()
        torch.cuda.synchronize(self.device)
        for i, (col, _, dt) in enumerate(L.cell_cols):
            arr = np.ascontiguousarray(np.concatenate(parts[col]).astype(dt))
            if dt == np.uint32:
                arr = arr.view(np.int32)
            if total:
                self.cols_dev[i][ab][:total].copy_(torch.from_numpy(arr))
        par = self._field_parity()
        for i, name in enumerate(L.chem_fields):
            for k, eng in enumerate(self.engines):
                host = np.asarray(eng.chemistry.column(name), dtype=np.float32)
                spec_d = eng._diffusion.get(name)
                if spec_d is not None:
                    host = host.copy(order="F")
                    b = np.float32(spec_d.boundary)
                    host[0, :, :] = host[-1, :, :] = b
                    host[:, 0, :] = host[:, -1, :] = b
                    host[:, :, 0] = host[:, :, -1] = b
                flat = np.ascontiguousarray(host.ravel(order="F"))
                lo, hi = int(self.field_off[k]), int(self.field_off[k + 1])
                dst = self.fields_dev[i][int(par[k, i])][lo:hi]
                if dst.dtype == torch.float32:
                    dst.copy_(torch.from_numpy(flat))
                else:
                    bits = _fieldcodec.encode(flat, self._storage_code(name), self.field_enc[i], self.field_bval[i])
                    dst.view(torch.int16).copy_(torch.from_numpy(bits.view(np.int16)))
            if self.fields_dev[i][2] is not None:
                self.fields_dev[i][2].zero_()
            if self.comp_dev[i] is not None:
                self.comp_dev[i].zero_()
        torch.cuda.synchronize(self.device)
        self._check(self.lib.olc_set_agent_count(self.handle, total, self._stream()))

    def member_rows(self) -> tuple[np.ndarray, np.ndarray, int]:
        """(simulation index, life flag) of every row in use, and the row count."""
        rows = self.counters()["n_agents"]
        ab = self._agent_buf()
        self.torch.cuda.synchronize(self.device)
        sim = self.cols_dev[len(self.layout.cell_cols) - 1][ab][:rows].cpu().numpy().view(np.uint32)
        return sim, self._life(rows), rows

    def snapshot(self, k: int) -> dict:
        """Member k's raw device state in the form of CudaBackend.snapshot():
        its rows in device order (dead rows included), life flags, fields."""
        sim, life, rows = self.member_rows()
        sel = np.nonzero(sim == k)[0]
        ab = self._agent_buf()
        out = {"rows": len(sel), "life": life[sel].copy(), "cols": {}, "fields": {}}
        for i, (col, _, dt) in enumerate(self.layout.cell_cols):
            if col == "_sim":
                continue
            a = self.cols_dev[i][ab][:rows].cpu().numpy()
            out["cols"][col] = (a.view(np.uint32) if dt == np.uint32 else a)[sel].copy()
        par = self._field_parity()
        lo, hi = int(self.field_off[k]), int(self.field_off[k + 1])
        for i, name in enumerate(self.layout.chem_fields):
            t = self.fields_dev[i][int(par[k, i])][lo:hi]
            out["fields"][name] = t.cpu().numpy().copy() if t.dtype == self.torch.float32 else \
                t.cpu().view(self.torch.int16).numpy().view(np.uint16).copy()
            if self.comp_dev[i] is not None:
                out.setdefault("residuals", {})[name] = self.comp_dev[i][lo:hi].cpu().numpy().copy()
        return out

    def sync_to_host(self) -> None:
        """Device -> every member engine's agents (live rows) and fields."""
        L = self.layout
        sim, life, rows = self.member_rows()
        ab = self._agent_buf()
        host_cols = {}
        for i, (col, _, dt) in enumerate(L.cell_cols):
            a = self.cols_dev[i][ab][:rows].cpu().numpy()
            host_cols[col] = a.view(np.uint32) if dt == np.uint32 else a
        par = self._field_parity()
        for k, eng in enumerate(self.engines):
            keep = (sim == k) & (life == 0)
            cols = {col: host_cols[col][keep].copy() for col, _, _ in L.cell_cols if col != "_sim"}
            eng.cells._set_columns(cols, L.cell_class)
            lo, hi = int(self.field_off[k]), int(self.field_off[k + 1])
            for i, name in enumerate(L.chem_fields):
                t = self.fields_dev[i][int(par[k, i])][lo:hi]
                if self.comp_dev[i] is not None:
                    bits = t.cpu().view(self.torch.int16).numpy().view(np.uint16)
                    flat = _fieldcodec.decode(bits, self._storage_code(name), self.field_enc[i], self.field_bval[i],
                                              self.comp_dev[i][lo:hi].cpu().numpy())
                else:
                    flat = t.cpu().numpy()
                eng.chemistry.column(name)[...] = flat.reshape(eng.chemistry_shape, order="F")

    def _storage_code(self, name: str) -> int:
        for e in self.engines:
            if name in e._diffusion:
                return STORAGE_CODES[e._diffusion[name].storage]
        return 0

    def close(self) -> None:
        if self.handle:
            self.lib.olc_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass
