"""Measured choice of kernel shapes and variants (olc.h OlcTuning).

Every choice computes the same bits, so the tuner only measures: it times each
candidate on the caller's own workload with per-stage CUDA events
(olc_set_profiling) and keeps the fastest.

* ``tune_engine(engine)``: the FP32 stencil tile (rows x planes of the TMA
  substep), whether FP32 fields take two substeps per pass (temporal
  blocking, and the CTA size of that kernel), the share of an FP32 field's
  planes kept in L2 by eviction hints, and the contact walk of a solo
  engine.  The engine's state is saved
  with ``state_dict()`` first and restored after, so tuning leaves the run
  exactly where it was.
* ``tune_batch(make_batch)``: the batched FP32 substep's tile depth for each
  member grid size, measured on a throwaway batch built by ``make_batch()``;
  ``apply_batch(batch, depths)`` sets the result on the real one.

Results are cached per device and workload shape in
``oncolytica_b200/_cache/tuning.json`` (``cache=False`` re-measures).  No
counterpart in the reference, whose dispatches have fixed sizes
(framework/src/oncolytica/gpu/runtime/_gpu_backend.py:134-136).
"""
from __future__ import annotations

import json
import math
import os
import threading

from oncolytica_b200 import _lib

STENCIL_TILES = ((8, 8), (16, 8), (8, 16), (16, 4))
CONTACT_VARIANTS = (_lib.OLC_CONTACT_FLAT, _lib.OLC_CONTACT_NESTED)
CONTACT_NAMES = {_lib.OLC_CONTACT_FLAT: "flat", _lib.OLC_CONTACT_NESTED: "nested"}
BATCH_DEPTHS = (8, 16, 32)
# (threads per CTA, planes per CTA) of the two-substeps-per-pass kernel; (0, 0) = one substep per pass
STENCIL_PAIRS = ((0, 0), (1024, 0), (512, 0), (256, 0), (128, 0))
# share of an FP32 field's planes kept in L2 across one-substep passes (eviction hints)
L2_KEEP = (0, 30, 45, 60)
DEFAULT = {"stencil_tile": (8, 8), "contact_variant": _lib.OLC_CONTACT_FLAT, "batch_tile_depth": 16,
           "stencil_pair": (0, 0), "l2_keep_pct": 0}
VERSION = 3  # cache entries of earlier tuners lack choices; they are measured again


def pair_applies(threads: int, dims) -> bool:
    """Whether the two-substep kernel with ``threads`` per CTA runs on a field
    of ``dims`` (x, y, z): rows of at most 256 voxels, x a multiple of 4, and
    at least three intermediate rows per CTA (olc_field.cu pair_rows)."""
    nx = int(dims[0])
    return threads == 0 or (8 <= nx <= 256 and nx % 4 == 0 and threads // (nx // 4) >= 3)

CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_cache", "tuning.json")
_lock = threading.Lock()


def _device_name() -> str:
    import torch

    return torch.cuda.get_device_name(torch.cuda.current_device())


def _load_cache() -> dict:
    try:
        with open(CACHE) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(key: str, value: dict) -> None:
    """Adds a record to the cache file.  Several processes (one per GPU) may
    tune at once: each writes its own temporary file and renames it over the
    cache, and a failed write only loses the record (it is measured again)."""
    with _lock:
        data = _load_cache()
        data[key] = value
        tmp = f"{CACHE}.{os.getpid()}.tmp"
        try:
            os.makedirs(os.path.dirname(CACHE), exist_ok=True)
            with open(tmp, "w") as fh:
                json.dump(data, fh, indent=1, sort_keys=True)
            os.replace(tmp, CACHE)
        except OSError:
            try:
                os.unlink(tmp)
            except OSError:
                pass


def _bucket(n: int) -> int:
    """Agent counts within a factor of about 1.4 share a cache entry."""
    return 0 if n <= 0 else int(round(2.0 * math.log2(n)))


def engine_key(eng) -> str:
    be = eng._backend_impl
    fields = []
    for name in be.layout.chem_fields:
        st, enc, _ = be.field_codec(name)
        fields.append(f"{name}:{st}:{enc}:{eng.substeps_for(name) if name in eng._diffusion else 0}")
    contact = "mech" if (eng._contact is not None and be.mech_enabled()) else ("on" if eng._contact else "off")
    n = be.counters()["n_agents"]
    return "|".join([f"solo{VERSION}", _device_name(), "x".join(map(str, eng.chemistry_shape)),
                     "x".join(map(str, eng.tissue_shape)), ",".join(fields), contact, f"n{_bucket(n)}"])


def _measure(eng, sd, tuning: dict, stage: str, steps: int) -> float:
    """ms per step of one stage with `tuning`, from the saved state (one
    unmeasured step first: launch set-up and caches)."""
    be = eng._backend_impl
    be.set_tuning(**tuning)
    be.load_state_dict(sd)
    be.run_steps(1)
    be.set_profiling(True)
    be.run_steps(steps)
    prof = be.profile()
    be.set_profiling(False)
    return prof[stage] / max(1, prof["steps"])


def tune_engine(eng, steps: int = 4, cache: bool = True) -> dict:
    """Chooses and sets the stencil tile and the contact walk of a loaded
    solo engine; returns {"tuning": ..., "measured_ms": ..., "cached": bool}."""
    be = eng._backend_impl
    if be is None:
        raise RuntimeError("tune_engine: load_model() first")
    key = engine_key(eng)
    if cache:
        hit = _load_cache().get(key)
        if hit:
            be.set_tuning(**_tuning_args(hit["tuning"]))
            return dict(hit, cached=True)
    sd = be.state_dict()
    engine_step, graphs = eng._step, eng.use_graphs
    eng.set_graphs(False)
    best = dict(DEFAULT)
    measured = {}
    try:
        if be.has_tma_fields():
            times = {}
            for tile in STENCIL_TILES:
                times[tile] = _measure(eng, sd, dict(best, stencil_tile=tile), "ms_substeps", steps)
            best["stencil_tile"] = min(times, key=times.get)
            measured["substeps"] = {f"{a}x{b}": v for (a, b), v in times.items()}
            # two substeps per pass, on the fastest single-pass tile (the odd
            # substep of a field and pinned fields keep single passes)
            times = {}
            for pair in STENCIL_PAIRS:
                if pair_applies(pair[0], eng.chemistry_shape):
                    times[pair] = _measure(eng, sd, dict(best, stencil_pair=pair), "ms_substeps", steps)
            best["stencil_pair"] = min(times, key=times.get)
            measured["substep_pairs"] = {f"{a}/{b}": v for (a, b), v in times.items()}
            # the slab of planes kept in L2 from substep to substep
            if best["stencil_pair"][0] == 0:
                times = {k: _measure(eng, sd, dict(best, l2_keep_pct=k), "ms_substeps", steps) for k in L2_KEEP}
                best["l2_keep_pct"] = min(times, key=times.get)
                measured["substep_l2_keep_pct"] = {str(k): v for k, v in times.items()}
        if eng._contact is not None and not be.mech_enabled():
            times = {}
            for v in CONTACT_VARIANTS:
                times[v] = _measure(eng, sd, dict(best, contact_variant=v), "ms_contact", steps)
            best["contact_variant"] = min(times, key=times.get)
            measured["contact"] = {CONTACT_NAMES[v]: t for v, t in times.items()}
    finally:
        be.set_tuning(**best)
        be.load_state_dict(sd)
        eng._step = engine_step
        eng.set_graphs(graphs)
    rec = {"tuning": {"stencil_tile": list(best["stencil_tile"]), "contact_variant": int(best["contact_variant"]),
                      "batch_tile_depth": int(best["batch_tile_depth"]), "stencil_pair": list(best["stencil_pair"]),
                      "l2_keep_pct": int(best["l2_keep_pct"])},
           "measured_ms": measured, "steps": steps}
    if cache:
        _store(key, rec)
    return dict(rec, cached=False)


def _tuning_args(t: dict) -> dict:
    """set_tuning keyword arguments from a record's "tuning" object."""
    return {"stencil_tile": tuple(t["stencil_tile"]), "contact_variant": int(t["contact_variant"]),
            "batch_tile_depth": int(t["batch_tile_depth"]), "stencil_pair": tuple(t.get("stencil_pair", (0, 0))),
            "l2_keep_pct": int(t.get("l2_keep_pct", 0))}


def apply_engine(eng, rec: dict) -> None:
    """Sets a tuning record's choices on another solo engine of the same
    workload shape."""
    if rec.get("tuning"):
        eng._backend_impl.set_tuning(**_tuning_args(rec["tuning"]))


def batch_key(batch) -> str:
    sizes = sorted({tuple(int(v) for v in e.chemistry_shape) for e in batch.engines})
    storages = ",".join(str(e) for e in batch.field_enc)
    return "|".join(["batch", _device_name(), ";".join("x".join(map(str, s)) for s in sizes), storages])


def apply_batch(batch, depths_by_size: dict) -> list:
    """Sets each member's FP32 substep tile depth from {grid size "GxGxG":
    depth}; returns the per-member list."""
    per = [int(depths_by_size.get("x".join(str(int(v)) for v in e.chemistry_shape), 0)) for e in batch.engines]
    batch.set_tile_depths(per)
    return per


def tune_batch(make_batch, steps: int = 3, cache: bool = True) -> dict:
    """The batched FP32 substep's tile depth for each member grid size, by
    coordinate descent over the sizes (each size's depths timed with the others
    fixed) on a batch from ``make_batch()``, which the tuner steps and closes.
    Returns {"depths": {"GxGxG": depth}, "measured_ms": ..., "cached": bool}."""
    batch = make_batch()
    try:
        key = batch_key(batch)
        if cache:
            hit = _load_cache().get(key)
            if hit:
                return dict(hit, cached=True)
        sizes = sorted({"x".join(str(int(v)) for v in e.chemistry_shape) for e in batch.engines})
        chosen = {s: DEFAULT["batch_tile_depth"] for s in sizes}
        measured = {}
        batch.set_graphs(False)
        batch.run_steps(1)
        for size in sizes:
            times = {}
            for d in BATCH_DEPTHS:
                apply_batch(batch, dict(chosen, **{size: d}))
                batch.run_steps(1)
                batch.set_profiling(True)
                batch.run_steps(steps)
                prof = batch.profile()
                batch.set_profiling(False)
                times[d] = prof["ms_substeps"] / max(1, prof["steps"])
            chosen[size] = min(times, key=times.get)
            measured[size] = times
        rec = {"depths": chosen, "measured_ms": measured, "steps": steps}
        if cache:
            _store(key, rec)
        return dict(rec, cached=False)
    finally:
        batch.close()


def summary(rec: dict) -> dict:
    """The chosen configuration of a tuning record, for a benchmark line."""
    out = dict(rec.get("tuning") or {})
    if "depths" in rec:
        out["batch_tile_depths"] = rec["depths"]
    out["cached"] = bool(rec.get("cached"))
    if rec.get("measured_ms"):
        out["measured_ms"] = rec["measured_ms"]
    return out


__all__ = ["tune_engine", "tune_batch", "apply_engine", "apply_batch", "summary", "pair_applies", "STENCIL_TILES",
           "STENCIL_PAIRS", "L2_KEEP", "CONTACT_VARIANTS", "BATCH_DEPTHS"]
