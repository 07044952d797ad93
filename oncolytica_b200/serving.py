"""Serving loop: simulation requests of different sizes join a running batch
as they arrive and leave it when done (continuous batching; no counterpart in
the reference, which runs one simulation per engine).

A request is what a solo run takes: an ``Engine`` configured as for that run
(geometry, chemistry grid, diffusion, contact, agents, dt, seed) with a model
instance carrying its ``Params``, and a step count.  ``ServingPool`` keeps
every admitted request's agents and fields resident on the device inside one
libolc pool handle (``olc_create_pool``): all residents advance together, one
launch per stage, and each reproduces its solo run bit for bit.

Admission is by free device memory.  At start the pool takes a fraction of
the free HBM as three arenas: agent rows (reserved per request by its engine's
``max_agents``, the same capacity its solo run has), bin-table entries and
field voxels (one range per request, the same range in every field buffer).
A queued request is admitted, first come first served with backfill, when a
slot and room in all three arenas are free; requests finish out of order, and
a finished request's result (live agents in device order, fields, reductions,
metrics) is copied out asynchronously before its memory returns to the arenas.

Host-side fault injection (``FaultInjector``) makes admissions fail as if the
device were out of memory or raised an error, so the queueing, rejection and
cancellation paths are testable without a GPU fault (``FakePoolDevice`` runs
the scheduler on the CPU).
"""
from __future__ import annotations

import collections
import ctypes as C
import time
from dataclasses import dataclass, field
from typing import Any, Callable, Iterable, Sequence

import numpy as np

from oncolytica_b200 import _fieldcodec, _lib
from oncolytica_b200.backend import FIELD_DTYPES, seed_rng
from oncolytica_b200.engine import STORAGE_CODES
from oncolytica_b200.compiler.emit_cuda import make_layout, pack_params, translate_model


class RequestError(ValueError):
    """A request the pool can never run (malformed, or larger than the pool)."""


class CapacityError(RuntimeError):
    """No room for the request right now (slots, rows or arenas are in use)."""


@dataclass
class SimRequest:
    """One simulation to run for ``steps`` steps from the engine's state."""

    engine: Any
    sim: Any
    steps: int
    return_state: bool = True
    request_id: int = -1
    arrival: float | None = None   # clock time of submission (set by submit when None)
    _payload: Any = field(default=None, repr=False, compare=False)  # host half of the admission


@dataclass
class SimResult:
    request_id: int
    status: str                    # "done", "cancelled", "rejected" or "failed"
    error: str | None = None
    steps: int = 0
    arrival: float = 0.0
    admitted: float | None = None
    finished: float | None = None
    agents: dict | None = None     # live rows in device order: column -> array
    fields: dict | None = None     # field -> FP32 values (16-bit: stored value + residual), chemistry shape
    field_bits: dict | None = None  # 16-bit fields: raw storage bits (uint16), flat x-fastest
    residuals: dict | None = None  # 16-bit fields: FP32 residuals, flat x-fastest
    reductions: dict | None = None
    metrics: dict | None = None
    voxel_updates: int = 0

    @property
    def ttc(self) -> float | None:
        """Time to completion: submission to result available."""
        return None if self.finished is None else self.finished - self.arrival


@dataclass
class Footprint:
    rows: int            # agent rows reserved (the request's max_agents)
    table: int           # bin-table entries
    voxels: int          # field voxels (per field buffer)


@dataclass
class _Resident:
    req: SimRequest
    member: Any
    admitted: float
    done: int = 0


# ---------------------------------------------------------------- fault injection
class FaultInjector:
    """Host-side faults for the admission path: ``oom[request_id] = k`` makes
    the next k admissions of that request fail as if the arenas were full;
    ``fail`` is a set of request ids whose admission raises a device error
    (the request fails; the pool keeps serving)."""

    def __init__(self, oom: dict | None = None, fail: Iterable[int] = ()) -> None:
        self.oom = dict(oom or {})
        self.fail = set(fail)
        self.events: list[tuple[str, int]] = []

    def before_admit(self, req: SimRequest) -> None:
        rid = req.request_id
        if rid in self.fail:
            self.events.append(("fail", rid))
            raise RuntimeError(f"injected device error admitting request {rid}")
        if self.oom.get(rid, 0) > 0:
            self.oom[rid] -= 1
            self.events.append(("oom", rid))
            raise CapacityError(f"injected out-of-memory admitting request {rid}")


# ---------------------------------------------------------------- scheduler
class ServingPool:
    """Continuous batching over a pool device (``PoolDevice`` on a GPU,
    ``FakePoolDevice`` in host-only tests)."""

    def __init__(self, device: Any, *, backfill: bool = True, depth: int = 2,
                 clock: Callable[[], float] = time.perf_counter, faults: FaultInjector | None = None) -> None:
        self.device = device
        self.backfill = bool(backfill)
        self.depth = max(1, int(depth))
        self.clock = clock
        self.faults = faults
        self.queue: collections.deque[SimRequest] = collections.deque()
        self.residents: dict[int, _Resident] = {}
        self.draining: list[tuple[_Resident, Any]] = []
        self.results: dict[int, SimResult] = {}
        self.rows_reserved = 0
        self.max_resident = 0
        self.peak_usage: dict = {}
        self.steps_run = 0
        self._next_id = 0
        self._inflight: collections.deque = collections.deque()
        # the device status word (capacity overflow, a bounded wait that gave
        # up) is read every status_every steps; new bits fail the requests on
        # the device then (they cannot be attributed to one member)
        self.status_every = _lib.StatusWatch.DEFAULT_EVERY
        self._status_seen = 0
        self._since_status = 0

    # ---- requests ---------------------------------------------------------
    def submit(self, req: SimRequest) -> int:
        if req.request_id < 0:
            req.request_id = self._next_id
        self._next_id = max(self._next_id, req.request_id + 1)
        if req.arrival is None:
            req.arrival = self.clock()
        try:
            if not isinstance(req.steps, (int, np.integer)) or req.steps < 1:
                raise RequestError(f"steps must be a positive integer, got {req.steps!r}")
            self.device.validate(req)
            fp = self.device.footprint(req)
            if not self.device.could_ever_fit(fp):
                raise RequestError(f"request needs {fp} but the pool holds {self.device.capacity()}")
        except RequestError as e:
            self._finish(req, "rejected", error=str(e))
            return req.request_id
        self.queue.append(req)
        return req.request_id

    def cancel(self, request_id: int) -> bool:
        """Drops a queued request, or retires a resident one between steps."""
        for req in list(self.queue):
            if req.request_id == request_id:
                self.queue.remove(req)
                self._finish(req, "cancelled")
                return True
        r = self.residents.pop(request_id, None)
        if r is None:
            return False
        self.device.retire(r.member)
        self.rows_reserved -= self.device.footprint(r.req).rows
        self._finish(r.req, "cancelled", admitted=r.admitted, steps=r.done)
        return True

    def _finish(self, req: SimRequest, status: str, error: str | None = None, admitted: float | None = None,
                steps: int = 0) -> SimResult:
        res = SimResult(request_id=req.request_id, status=status, error=error, steps=steps,
                        arrival=float(req.arrival), admitted=admitted, finished=self.clock())
        self.results[req.request_id] = res
        return res

    # ---- admission --------------------------------------------------------
    def _try_admit(self, req: SimRequest) -> bool:
        fp = self.device.footprint(req)
        if self.rows_reserved + fp.rows > self.device.capacity().rows:
            return False
        try:
            if self.faults is not None:
                self.faults.before_admit(req)
            member = self.device.admit(req)
        except CapacityError:
            return False
        except RequestError as e:
            self._finish(req, "rejected", error=str(e))
            return True
        except Exception as e:  # device error: the request fails, the pool goes on
            self._finish(req, "failed", error=str(e))
            return True
        self.rows_reserved += fp.rows
        self.residents[req.request_id] = _Resident(req, member, self.clock())
        self.max_resident = max(self.max_resident, len(self.residents))
        return True

    def admit(self) -> int:
        """Admits queued requests in arrival order; with backfill, a request
        that does not fit yet is passed over by later ones that do."""
        admitted = 0
        for req in list(self.queue):
            if self._try_admit(req):
                self.queue.remove(req)
                admitted += req.request_id in self.residents
            elif not self.backfill:
                break
        if admitted and hasattr(self.device, "usage"):
            u = self.device.usage()
            u["rows_reserved"] = self.rows_reserved
            for k, v in u.items():
                self.peak_usage[k] = max(self.peak_usage.get(k, 0), v)
        return admitted

    # ---- stepping ---------------------------------------------------------
    def step(self) -> list[SimResult]:
        """Admits what fits, advances every resident one step, starts the
        result copies of residents that finished and returns the results
        whose copies are complete."""
        self.admit()
        if self.residents:
            finishing = [r for r in self.residents.values() if r.done + 1 == r.req.steps]
            self.device.step(collect=bool(finishing))
            self.steps_run += 1
            for r in self.residents.values():
                r.done += 1
            for r in finishing:
                pending = self.device.finish(r.member, r.req)
                self.device.retire(r.member)
                del self.residents[r.req.request_id]
                self.rows_reserved -= self.device.footprint(r.req).rows
                self.draining.append((r, pending))
            self._inflight.append(self.device.fence())
            while len(self._inflight) > self.depth:
                self._inflight.popleft().synchronize()
            self._since_status += 1
            if self._since_status >= self.status_every:
                self._since_status = 0
                self._check_status()
        return self.poll()

    def _check_status(self) -> None:
        """Reads the device status word; bits not seen before fail every
        request whose steps ran since the last check: the residents and the
        results still being copied out."""
        read = getattr(self.device, "status", None)
        if read is None:
            return
        bits = int(read())
        new = bits & ~self._status_seen
        self._status_seen |= bits
        if not new:
            return
        msg = f"device status {bits:#x} during this request's steps: {_lib.status_names(new)}"
        for rid, r in list(self.residents.items()):
            self.device.retire(r.member)
            self.rows_reserved -= self.device.footprint(r.req).rows
            del self.residents[rid]
            self._finish(r.req, "failed", error=msg, admitted=r.admitted, steps=r.done)
        for r, pending in self.draining:
            pending.wait()
            self._finish(r.req, "failed", error=msg, admitted=r.admitted, steps=r.done)
        self.draining = []

    def poll(self, wait: bool = False) -> list[SimResult]:
        out, keep = [], []
        for r, pending in self.draining:
            if wait or pending.ready():
                res = self._finish(r.req, "done", admitted=r.admitted, steps=r.done)
                pending.fill(res)
                out.append(res)
            else:
                keep.append((r, pending))
        self.draining = keep
        return out

    @property
    def idle(self) -> bool:
        return not self.queue and not self.residents and not self.draining

    # An empty pool that admits nothing this many times in a row rejects the
    # head of the queue (only injected faults make an empty pool refuse a
    # request that could_ever_fit accepted).
    MAX_IDLE_TRIES = 64

    def _unstick(self, idle_tries: int) -> int:
        if self.residents or not self.queue:
            return 0
        if idle_tries + 1 < self.MAX_IDLE_TRIES:
            return idle_tries + 1
        self._finish(self.queue.popleft(), "rejected", error="not admitted by an empty pool")
        return 0

    def drain(self) -> list[SimResult]:
        """Runs until every submitted request has finished."""
        out, idle = [], 0
        while self.queue or self.residents:
            out += self.step()
            idle = self._unstick(idle)
        out += self.poll(wait=True)
        return out

    def serve(self, arrivals: Sequence[tuple[float, Callable[[], SimRequest]]],
              on_result: Callable[[SimResult], None] | None = None, prefetch: float = 0.0,
              workers: int = 2) -> list[SimResult]:
        """Replays an arrival schedule in real time: ``arrivals`` holds
        (seconds after start, request factory) in time order; each request is
        submitted when its time comes (its arrival is the scheduled time).
        With ``prefetch`` > 0, worker threads build the requests (the factory
        and the device's host-side ``prepare``) up to that many seconds ahead,
        as clients would send them ready-made.  Returns every result once all
        have finished."""
        import concurrent.futures as cf

        ex = cf.ThreadPoolExecutor(max(1, workers)) if prefetch > 0 else None
        futures: dict[int, Any] = {}
        prep = getattr(self.device, "prepare", None)

        def build(j: int) -> SimRequest:
            req = arrivals[j][1]()
            if prep is not None:
                try:
                    prep(req)
                except RequestError:
                    pass  # rejected on admission with the same message
            return req

        t0 = self.clock()
        i, idle, ahead = 0, 0, 0
        out: list[SimResult] = []
        while i < len(arrivals) or not self.idle:
            now = self.clock()
            if ex is not None:
                while ahead < len(arrivals) and t0 + arrivals[ahead][0] <= now + prefetch:
                    futures[ahead] = ex.submit(build, ahead)
                    ahead += 1
            while i < len(arrivals) and t0 + arrivals[i][0] <= now:
                req = futures.pop(i).result() if i in futures else arrivals[i][1]()
                req.arrival = t0 + arrivals[i][0]
                self.submit(req)
                if req.request_id in self.results:
                    out.append(self.results[req.request_id])  # rejected at submission
                i += 1
            got = self.step()
            idle = self._unstick(idle)
            if self.idle and i < len(arrivals):
                time.sleep(max(0.0, min(t0 + arrivals[i][0] - self.clock(), 0.05)))
            out += got
        out += self.poll(wait=True)
        if ex is not None:
            ex.shutdown(wait=True)
        if on_result is not None:
            for r in out:
                on_result(r)
        return out


# ---------------------------------------------------------------- GPU pool device
def _geom_of(eng) -> Any:
    tdims = tuple(int(v) for v in eng.tissue_shape)
    g = _lib.OlcGeom()
    g.tissue_dims[:] = tdims
    g.tissue_voxel_size = eng.tissue_voxel_size
    g.chem_dims[:] = tuple(int(v) for v in eng.chemistry_shape)
    g.chem_voxel_size = eng.chemistry_voxel_size
    g.domain_lo[:] = eng.domain_lo or (0.0, 0.0, 0.0)
    g.domain_hi[:] = eng.domain_hi or tuple(d * eng.tissue_voxel_size for d in tdims)
    return g


def _table_entries(tissue_dims) -> int:
    from oncolytica_b200._geometry import voxel_table_size

    return int(voxel_table_size(tuple(int(v) for v in tissue_dims)))


@dataclass
class _Member:
    slot: int
    field_off: int
    nvox: int
    substeps: tuple


class _PendingResult:
    def __init__(self, event, fill_fn) -> None:
        self.event = event
        self._fill = fill_fn

    def ready(self) -> bool:
        return self.event.query()

    def wait(self) -> None:
        self.event.synchronize()

    def fill(self, res: SimResult) -> None:
        self.event.synchronize()
        self._fill(res)


class PoolDevice:
    """The libolc pool on the current CUDA device, for one model.

    ``prototype`` is an (engine, sim) pair configured like the requests: it
    fixes the model, the chemistry fields and their storage, contact, dt and
    the metric layout; every request must match it.  Arena sizes are given
    directly or planned from a share of free HBM (``plan_arenas``)."""

    def __init__(self, prototype: tuple, *, max_slots: int, max_rows: int, table_entries: int,
                 field_voxels: int, max_tissue_dims: tuple, graphs: bool = False) -> None:
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("oncolytica_b200 needs a CUDA device: the step has no CPU implementation")
        self.torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.stream = torch.cuda.Stream(self.device)
        self.lib = _lib.load()
        self.handle = C.c_void_p()
        eng, sim = prototype
        eng._prepare_model(sim)
        self.proto_engine, self.model_cls = eng, type(sim)
        self.max_slots, self.max_rows = int(max_slots), int(max_rows)
        self.table_entries, self.field_voxels = int(table_entries), int(field_voxels)
        self.max_tissue_dims = tuple(int(v) for v in max_tissue_dims)
        self.time_steps = False
        self.step_events: list = []
        self._build(eng, sim)
        self.set_graphs(graphs)

    # ---- set-up -------------------------------------------------------------
    def _check(self, rc: int) -> None:
        if rc != _lib.OLC_OK:
            raise _lib.OlcError(rc, _lib.last_error(self.handle))

    def _s(self) -> C.c_void_p:
        return C.c_void_p(self.stream.cuda_stream)

    def _build(self, eng, sim) -> None:
        torch = self.torch
        contact = eng._contact
        self.contact = contact
        radius_field = contact.radius if (contact and isinstance(contact.radius, str)) else None
        self.layout = L = make_layout(sim._spec, radius_field, batched=True)
        self.program = (translate_model(sim, L, radius_field)
                        if (eng._cell_rules or eng._metric_rules or eng._chemistry_rules or eng._tissue_rules) else None)
        self.sinks = self.program.sink_fields if self.program else set()
        self.storage, self.encoding, self.bval = {}, {}, {}
        for name in L.chem_fields:
            d = eng._diffusion.get(name)
            self.storage[name] = STORAGE_CODES[d.storage] if d is not None else 0
            # what the 16-bit elements hold; every request must resolve the same
            self.encoding[name] = eng.field_encoding(name)
            self.bval[name] = float(d.boundary) if d is not None else 0.0
        caps = _lib.OlcCaps()
        caps.max_agents = self.max_rows
        caps.n_agent_fields = len(L.cell_cols)
        caps.n_fields = len(L.chem_fields)
        caps.state_field = -1
        for i, (col, _, dt) in enumerate(L.cell_cols):
            if col == "state" and dt == np.int32:
                caps.state_field = i
        caps.radial_bin_width = eng.tissue_voxel_size
        caps.dt = eng.dt
        self.dt = eng.dt
        cfg = _lib.OlcPoolConfig()
        cfg.max_slots = self.max_slots
        cfg.max_tissue_dims[:] = self.max_tissue_dims
        cfg.table_entries = self.table_entries
        cfg.field_voxels = max(self.field_voxels, 1)
        self._check(self.lib.olc_create_pool(C.byref(cfg), C.byref(caps), C.byref(self.handle)))
        with torch.cuda.stream(self.stream):
            self.cols_dev = []
            for i, (col, _, dt) in enumerate(L.cell_cols):
                tdt = torch.float32 if dt == np.float32 else torch.int32
                a = torch.zeros(self.max_rows, dtype=tdt, device=self.device)
                b = torch.zeros(self.max_rows, dtype=tdt, device=self.device)
                self.cols_dev.append((a, b))
                self._check(self.lib.olc_bind_agent_column(self.handle, i, C.c_void_p(a.data_ptr()),
                                                           C.c_void_p(b.data_ptr())))
            self.fields_dev, self.comp_dev = [], []
            nv = max(self.field_voxels, 1)
            for i, name in enumerate(L.chem_fields):
                st = self.storage[name]
                fdt = FIELD_DTYPES[st](torch)
                a = torch.zeros(nv, dtype=fdt, device=self.device)
                b = torch.zeros(nv, dtype=fdt, device=self.device)
                s = torch.zeros(nv, dtype=torch.float32, device=self.device) if name in self.sinks else None
                comp = torch.zeros(nv, dtype=torch.float32, device=self.device) if st else None
                self.fields_dev.append((a, b, s))
                self.comp_dev.append(comp)
                self._check(self.lib.olc_bind_field_pool(
                    self.handle, i, C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()),
                    C.c_void_p(s.data_ptr()) if s is not None else None,
                    C.c_void_p(comp.data_ptr()) if comp is not None else None, st, self.encoding[name],
                    C.c_float(self.bval[name])))
        self.stream.synchronize()
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
                if any(d.storage != "f32" for d in eng._diffusion.values()):
                    from oncolytica_b200._errors import CompilationError

                    raise CompilationError("chemistry rules need FP32 chemistry fields (setup_diffusion storage='f32')")
                its = (C.c_int * len(self.program.kernels))(*self.program.iterations)
                self._check(self.lib.olc_set_rule_iterations(self.handle, its, len(self.program.kernels)))
        # every chemistry-rule iteration writes every field's other buffer and
        # flips its parity (olc_sim.cu step_once_batch), as each substep does
        self.chem_flips = (sum(it for (_, kind), it in zip(self.program.kernels, self.program.iterations)
                               if kind == 3) if self.program is not None else 0)
        self.metrics_words = max(1, len(L.metrics))
        self._check(self.lib.olc_set_user_metrics_size(self.handle, 4 * self.metrics_words))
        self.sim_col = len(L.cell_cols) - 1

    def set_graphs(self, enable: bool) -> None:
        self._check(self.lib.olc_set_graphs(self.handle, int(bool(enable))))

    # ---- requests ---------------------------------------------------------
    def capacity(self) -> Footprint:
        return Footprint(self.max_rows, self.table_entries, self.field_voxels)

    def could_ever_fit(self, fp: Footprint) -> bool:
        return fp.rows <= self.max_rows and fp.table <= self.table_entries and fp.voxels <= self.field_voxels

    def footprint(self, req: SimRequest) -> Footprint:
        e = req.engine
        nvox = int(np.prod(e.chemistry_shape)) if self.layout.chem_fields else 0
        return Footprint(int(e.max_agents), _table_entries(e.tissue_shape), nvox)

    def validate(self, req: SimRequest) -> None:
        """Host checks: same model, dt, contact and field storage as the pool;
        grids within the pool's limits (the library re-checks on admission)."""
        e, sim = req.engine, req.sim
        if type(sim) is not self.model_cls:
            raise RequestError(f"model {type(sim).__name__} differs from the pool's {self.model_cls.__name__}")
        if e.dt != self.dt:
            raise RequestError(f"dt {e.dt} differs from the pool's {self.dt}")
        if (e._contact is None) != (self.contact is None) or (e._contact and e._contact != self.contact):
            raise RequestError("contact settings differ from the pool's")
        for i in range(3):
            if int(e.tissue_shape[i]) > self.max_tissue_dims[i]:
                raise RequestError(f"bin grid {tuple(e.tissue_shape)} exceeds the pool's {self.max_tissue_dims}")
        for name in self.layout.chem_fields:
            d = e._diffusion.get(name)
            st = STORAGE_CODES[d.storage] if d is not None else 0
            if st != self.storage[name]:
                raise RequestError(f"field {name!r} storage differs from the pool's")
            if e.field_encoding(name) != self.encoding[name] or (
                    self.encoding[name] and d is not None and float(d.boundary) != self.bval[name]):
                raise RequestError(f"field {name!r} encoding (or encoded boundary value) differs from the pool's")
            if name in self.sinks and d is None:
                raise RequestError(f"sink_at(...).{name} needs Engine.setup_diffusion({name!r}, ...)")
        if e.chemistry is not None and int(e.chemistry_shape[0]) % (8 if any(self.storage.values()) else 4):
            raise RequestError("chemistry x extent must be a multiple of 4 (8 for 16-bit fields)")
        if int(e.max_agents) < 1:
            raise RequestError("max_agents must be >= 1")

    def prepare(self, req: SimRequest) -> None:
        """Host half of an admission, safe to run on another thread ahead of
        time: model checks, agent columns (RNG states seeded as in a solo
        run) and initial grids (faces pinned to the boundary, x fastest) in
        pinned host memory, diffusion specs and the Params blob."""
        if getattr(req, "_payload", None) is not None:
            return
        torch = self.torch
        e, sim = req.engine, req.sim
        e._prepare_model(sim)
        L = self.layout
        cols = e.cells.columns(L.cell_class)
        n = len(next(iter(cols.values()))) if cols else 0
        if n > e.max_agents:
            raise RequestError(f"{n} agents exceed the request's max_agents={e.max_agents}")
        nf = len(L.chem_fields)
        specs = (_lib.OlcDiffusion * max(nf, 1))()
        substeps = []
        for i, name in enumerate(L.chem_fields):
            d = e._diffusion.get(name)
            sp = specs[i]
            sp.storage = self.storage[name]
            sp.encoding = self.encoding[name]
            if d is None:
                sp.substeps = 0
                substeps.append(0)
            else:
                sp.diffusion, sp.decay, sp.boundary = d.diffusion, d.decay, d.boundary
                sp.substeps = e.substeps_for(name)
                sp.has_sink = int(name in self.sinks)
                substeps.append(int(sp.substeps))
        rng = cols.get("_rng_state", np.zeros(n, np.uint32)).astype(np.uint32)
        zero = rng == 0
        if zero.any():
            rng = rng.copy()
            rng[zero] = seed_rng(e.seed, np.nonzero(zero)[0].astype(np.uint32))
        agents = {}
        if n:
            for i, (col, _, dt) in enumerate(L.cell_cols):
                if col == "_sim":
                    continue
                host = rng if col == "_rng_state" else np.asarray(cols[col]).astype(dt)
                arr = np.ascontiguousarray(host).view(np.int32 if dt != np.float32 else np.float32)
                agents[i] = torch.from_numpy(arr).pin_memory()
        fields = []
        for i, name in enumerate(L.chem_fields):
            host = np.asarray(e.chemistry.column(name), dtype=np.float32)
            d = e._diffusion.get(name)
            pin = torch.empty(host.size, dtype=torch.float32, pin_memory=True)
            flat = pin.numpy()
            out = flat.reshape(host.shape, order="F")  # x fastest, written in place
            if not np.shares_memory(out, flat):
                raise RuntimeError("pinned field staging is not a view")
            out[...] = host
            if d is not None:
                b = np.float32(d.boundary)
                out[0, :, :] = out[-1, :, :] = b
                out[:, 0, :] = out[:, -1, :] = b
                out[:, :, 0] = out[:, :, -1] = b
            if self.storage[name]:  # 16-bit elements of the field's encoding, rounded to nearest even
                bits = _fieldcodec.encode(flat, self.storage[name], self.encoding[name], self.bval[name])
                pin = torch.from_numpy(bits.view(np.int16)).pin_memory()
            fields.append(pin)
        blob = pack_params(L, sim._params)
        req._payload = {"n": n, "specs": specs, "substeps": tuple(substeps), "agents": agents, "fields": fields,
                        "blob": blob, "geom": _geom_of(e), "nvox": int(np.prod(e.chemistry_shape)) if nf else 0}

    def admit(self, req: SimRequest) -> _Member:
        """Device half of an admission: a slot and arena ranges, then the
        agents appended and the initial grids written, all on the pool's
        stream.  CapacityError (nothing taken) when the pool is full."""
        torch = self.torch
        self.prepare(req)
        P = req._payload
        L = self.layout
        buf = C.create_string_buffer(P["blob"], len(P["blob"]))
        slot, foff = C.c_int32(), C.c_uint64()
        rc = self.lib.olc_pool_admit(self.handle, C.byref(P["geom"]), P["specs"], C.cast(buf, C.c_void_p),
                                     len(P["blob"]), C.byref(slot), C.byref(foff), self._s())
        if rc == _lib.OLC_ERR_CAPACITY:
            raise CapacityError(_lib.last_error(self.handle))
        if rc == _lib.OLC_ERR_ARG:
            raise RequestError(_lib.last_error(self.handle))
        self._check(rc)
        n, nvox = P["n"], P["nvox"]
        m = _Member(int(slot.value), int(foff.value), nvox, P["substeps"])
        with torch.cuda.stream(self.stream):
            keep = []
            if n:
                ptrs = (C.c_void_p * len(L.cell_cols))()
                for i, pin in P["agents"].items():
                    dev = torch.empty(n, dtype=pin.dtype, device=self.device)
                    dev.copy_(pin, non_blocking=True)
                    keep.append(dev)
                    ptrs[i] = dev.data_ptr()
                self._check(self.lib.olc_pool_add_agents(self.handle, m.slot, ptrs, n, self._s()))
            for i, pin in enumerate(P["fields"]):
                dst = self.fields_dev[i][0][m.field_off:m.field_off + nvox]
                if dst.dtype == torch.float32:
                    dst.copy_(pin, non_blocking=True)
                else:  # encoded on the host (prepare), as a solo run's upload
                    dst.view(torch.int16).copy_(pin, non_blocking=True)
            for t in keep:
                t.record_stream(self.stream)
        req._payload = None  # pinned buffers return to torch's cache once the copies are done
        return m

    def step(self, collect: bool) -> None:
        if self.time_steps:
            a, b = self.torch.cuda.Event(enable_timing=True), self.torch.cuda.Event(enable_timing=True)
            a.record(self.stream)
            self._check(self.lib.olc_step(self.handle, 1, int(collect), self._s()))
            b.record(self.stream)
            self.step_events.append((a, b))
        else:
            self._check(self.lib.olc_step(self.handle, 1, int(collect), self._s()))

    def device_seconds(self) -> float:
        """Device time of the steps run since time_steps was set (each step
        from its first to its last kernel; idle gaps between steps excluded)."""
        self.stream.synchronize()
        return sum(a.elapsed_time(b) for a, b in self.step_events) / 1e3

    def fence(self):
        ev = self.torch.cuda.Event()
        ev.record(self.stream)
        return ev

    def finish(self, m: _Member, req: SimRequest) -> _PendingResult:
        """Starts the copies of a member's result (after its last, collected
        step); the pending result is complete when its event is."""
        torch = self.torch
        L = self.layout
        steps = req.steps
        with torch.cuda.stream(self.stream):
            red = torch.empty(C.sizeof(_lib.OlcReductions), dtype=torch.uint8, pin_memory=True)
            met = torch.empty(4 * self.metrics_words, dtype=torch.uint8, pin_memory=True)
            self._check(self.lib.olc_pool_copy_results(self.handle, m.slot, C.c_void_p(red.data_ptr()),
                                                       C.c_void_p(met.data_ptr()), self._s()))
            host_cols, count_h, fields_h = {}, None, []
            if req.return_state:
                rows = int(req.engine.max_agents)
                dst = (C.c_void_p * len(L.cell_cols))()
                devs = {}
                for i, (col, _, dt) in enumerate(L.cell_cols):
                    if col == "_sim":
                        continue
                    t = torch.empty(rows, dtype=torch.float32 if dt == np.float32 else torch.int32, device=self.device)
                    devs[col] = t
                    dst[i] = t.data_ptr()
                count = torch.zeros(1, dtype=torch.int32, device=self.device)
                self._check(self.lib.olc_pool_gather(self.handle, m.slot, dst, rows, C.c_void_p(count.data_ptr()),
                                                     self._s()))
                count_h = torch.empty(1, dtype=torch.int32, pin_memory=True)
                count_h.copy_(count, non_blocking=True)
                for col, t in devs.items():
                    h = torch.empty(rows, dtype=t.dtype, pin_memory=True)
                    h.copy_(t, non_blocking=True)
                    host_cols[col] = h
                    t.record_stream(self.stream)
                count.record_stream(self.stream)
                for i, name in enumerate(L.chem_fields):
                    par = (steps * (m.substeps[i] + self.chem_flips)) & 1
                    src = self.fields_dev[i][par][m.field_off:m.field_off + m.nvox]
                    h = torch.empty(m.nvox, dtype=src.dtype, pin_memory=True)
                    h.copy_(src, non_blocking=True)
                    c = None
                    if self.comp_dev[i] is not None:
                        c = torch.empty(m.nvox, dtype=torch.float32, pin_memory=True)
                        c.copy_(self.comp_dev[i][m.field_off:m.field_off + m.nvox], non_blocking=True)
                    fields_h.append((name, h, c))
            ev = torch.cuda.Event()
            ev.record(self.stream)
        shape = tuple(int(v) for v in req.engine.chemistry_shape)
        vox_per_step = m.nvox * sum(m.substeps)

        def fill(res: SimResult) -> None:
            r = _lib.OlcReductions.from_buffer_copy(bytes(red.numpy()))
            res.reductions = {
                "n_live": r.n_live, "state_counts": list(r.state_counts), "radial_hist": list(r.radial_hist),
                "sum_pos": list(r.sum_pos), "sum_r2": r.sum_r2, "max_r": r.max_r,
                "field_mass": {f: r.field_mass[i] for i, f in enumerate(L.chem_fields)},
                "field_min": {f: r.field_min[i] for i, f in enumerate(L.chem_fields)},
                "field_max": {f: r.field_max[i] for i, f in enumerate(L.chem_fields)}}
            words = met.numpy().view(np.uint32)
            res.metrics = {}
            for name, (slot, ty) in L.metrics.items():
                w = words[slot:slot + 1]
                res.metrics[name] = (float(w.view(np.float32)[0]) if ty == "f32" else
                                     int(w[0]) if ty == "u32" else bool(w.view(np.int32)[0]) if ty == "bool"
                                     else int(w.view(np.int32)[0]))
            res.voxel_updates = vox_per_step * steps
            if count_h is None:
                return
            k = int(count_h.numpy()[0])
            if k > int(req.engine.max_agents):
                res.status, res.error = "failed", (f"{k} agents exceed the request's max_agents="
                                                   f"{req.engine.max_agents} (its solo run would drop births)")
                k = int(req.engine.max_agents)
            res.agents = {}
            for col, _, dt in L.cell_cols:
                if col in host_cols:
                    a = host_cols[col].numpy()[:k]
                    res.agents[col] = (a.view(np.uint32) if dt == np.uint32 else a).copy()
            res.fields, res.field_bits, res.residuals = {}, {}, {}
            for name, h, c in fields_h:
                if c is None:
                    v = h.numpy().copy()
                else:
                    bits = h.view(torch.int16).numpy().view(np.uint16).copy()
                    res.field_bits[name] = bits
                    res.residuals[name] = c.numpy().copy()
                    v = _fieldcodec.decode(bits, self.storage[name], self.encoding[name], self.bval[name],
                                           res.residuals[name])
                res.fields[name] = v.reshape(shape, order="F")

        return _PendingResult(ev, fill)

    def retire(self, m: _Member) -> None:
        self._check(self.lib.olc_pool_retire(self.handle, m.slot, self._s()))

    def usage(self) -> dict:
        u = _lib.OlcPoolUsage()
        self._check(self.lib.olc_pool_usage(self.handle, C.byref(u)))
        return {k: getattr(u, k) for k, _ in _lib.OlcPoolUsage._fields_}

    def counters(self) -> dict:
        c = _lib.OlcCounters()
        self._check(self.lib.olc_read_counters(self.handle, C.byref(c), self._s()))
        return {"n_agents": c.n_agents, "status": c.status, "steps": c.steps, "agent_steps": c.agent_steps}

    def status(self) -> int:
        return self.counters()["status"]

    def close(self) -> None:
        if self.handle:
            self.stream.synchronize()
            self.lib.olc_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass


def row_bytes(n_cols: int) -> int:
    """Device bytes per agent row of a pool: two buffers of every 4-byte
    column, and the library's per-row scratch (life flag, keys in and out,
    sort values and their alternates, contact positions, birth look-back)."""
    return 8 * n_cols + 1 + 4 + 4 + 4 + 8 + 16 + 1


def voxel_bytes(storages: Sequence[int], sinks: Sequence[bool]) -> int:
    """Device bytes per field voxel of a pool (every field buffer)."""
    b = 0
    for st, sk in zip(storages, sinks):
        b += 2 * (4 if st == 0 else 2) + (4 if sk else 0) + (4 if st else 0)
    return b


def plan_arenas(budget_bytes: int, mix: Sequence[Footprint], n_cols: int, storages: Sequence[int],
                sinks: Sequence[bool]) -> dict:
    """Splits a byte budget into the three arenas in the proportions a
    representative request mix uses them."""
    rb, vb, tb = row_bytes(n_cols), voxel_bytes(storages, sinks), 8
    rows = sum(f.rows for f in mix)
    vox = sum(f.voxels for f in mix)
    tab = sum(f.table for f in mix)
    per_mix = rows * rb + vox * vb + tab * tb
    k = max(1.0, budget_bytes / max(per_mix, 1))
    return {"max_rows": int(min(rows * k, 1 << 30)), "field_voxels": int(vox * k), "table_entries": int(min(tab * k, (1 << 31) - 1))}


# ---------------------------------------------------------------- host-only device
class FakePoolDevice:
    """The pool device interface without a GPU, for scheduler tests: slots and
    arenas are counted (first fit), a step advances nothing, a finished
    request's result is ready at once and carries its step count."""

    class _Ev:
        def synchronize(self) -> None:
            pass

        def query(self) -> bool:
            return True

    def __init__(self, max_slots: int, max_rows: int, table_entries: int, field_voxels: int) -> None:
        self.cap = Footprint(max_rows, table_entries, field_voxels)
        self.max_slots = max_slots
        arena = _lib.load(build_if_missing=False)
        self.lib = arena
        self._tab = C.c_void_p()
        self._vox = C.c_void_p()
        _lib.check(arena.olc_arena_create(table_entries, C.byref(self._tab)))
        _lib.check(arena.olc_arena_create(field_voxels, C.byref(self._vox)))
        self.slots: dict[int, tuple] = {}
        self.log: list[tuple] = []
        self.steps = 0
        self.status_bits = 0  # the device status word a test sets

    def status(self) -> int:
        return self.status_bits

    def capacity(self) -> Footprint:
        return self.cap

    def could_ever_fit(self, fp: Footprint) -> bool:
        return fp.rows <= self.cap.rows and fp.table <= self.cap.table and fp.voxels <= self.cap.voxels

    def footprint(self, req: SimRequest) -> Footprint:
        return req.engine["footprint"]

    def validate(self, req: SimRequest) -> None:
        if req.engine.get("malformed"):
            raise RequestError("malformed request")

    def admit(self, req: SimRequest):
        fp = self.footprint(req)
        if len(self.slots) >= self.max_slots:
            raise CapacityError("no free slot")
        t, v = C.c_uint64(), C.c_uint64()
        if self.lib.olc_arena_alloc(self._tab, fp.table, 1, C.byref(t)) != _lib.OLC_OK:
            raise CapacityError("bin-table arena full")
        if self.lib.olc_arena_alloc(self._vox, fp.voxels, 32, C.byref(v)) != _lib.OLC_OK:
            self.lib.olc_arena_release(self._tab, t.value, fp.table)
            raise CapacityError("field arena full")
        slot = min(set(range(self.max_slots)) - set(self.slots))
        self.slots[slot] = (t.value, fp.table, v.value, fp.voxels)
        self.log.append(("admit", req.request_id, slot))
        return slot

    def step(self, collect: bool) -> None:
        self.steps += 1
        self.log.append(("step", collect))

    def fence(self):
        return self._Ev()

    def finish(self, slot, req: SimRequest):
        self.log.append(("finish", req.request_id, slot))
        outer = self

        class P:
            def ready(self) -> bool:
                return True

            def wait(self) -> None:
                pass

            def fill(self, res: SimResult) -> None:
                res.metrics = {"slot": slot, "steps_at_finish": outer.steps}

        return P()

    def retire(self, slot) -> None:
        t, tn, v, vn = self.slots.pop(slot)
        _lib.check(self.lib.olc_arena_release(self._tab, t, tn))
        _lib.check(self.lib.olc_arena_release(self._vox, v, vn))
        self.log.append(("retire", slot))

    def close(self) -> None:
        if self._tab:
            self.lib.olc_arena_destroy(self._tab)
            self.lib.olc_arena_destroy(self._vox)
            self._tab = self._vox = C.c_void_p()
