"""Simulation bundles: the reference's on-disk format (a directory holding
config.json and raw buffer files, GpuBackend.get_config / export_bundle,
framework/src/oncolytica/gpu/runtime/_gpu_backend.py:196-334) written from a
CUDA engine and read back, plus an exact-resume record.

A bundle written here holds, like the reference's:
  config.json   params, layout (grid shapes, max_agents, struct strides and
                field offsets, uniform offsets), execution order, the kernel
                source file and the buffer files;
  cells_in.bin  max_agents agent records (AoS, the struct layout of config.json);
  state.bin     SimState {TotalAgents, NewTotalAgents} (u32 each);
  chem_in.bin   one chemistry record per voxel, grid order of the host Grid;
  tissue_in.bin one tissue record per voxel (when the model has tissue fields);
  uniforms.bin  the uniform block (tissue grid dims, voxel size, params);
  rules.cu      the CUDA C the rule translator emitted (the reference writes
                shader.wgsl);
and in addition resume.npz: the engine's state_dict() (16-bit field bits and
residuals, pending sinks, step counters), from which import_bundle() resumes
bit for bit.  A bundle without resume.npz (one the reference exported) is read
through the struct layout its config.json records.

The struct layout restates the reference's StructSerializer and
optimize_struct_layout (framework/src/oncolytica/gpu/runtime/_memory.py:11-118)
and wgsl_alignment (framework/src/oncolytica/gpu/compiler/_type_system.py:34-42),
so that a reader of the reference's bundles reads these the same way.
"""
from __future__ import annotations

import json
import os
import struct
from typing import Any

import numpy as np

from oncolytica_b200 import _types as T

_SIZE_ALIGN = {"f32": (4, 4), "i32": (4, 4), "u32": (4, 4), "vec3<f32>": (12, 16), "vec3<u32>": (12, 16),
               "vec3<i32>": (12, 16), "vec4<f32>": (16, 16)}


def wgsl_type(t: Any) -> str:
    """The reference's Python -> WGSL type map (bool is stored as i32)."""
    if t is T.vec3:
        return "vec3<f32>"
    if t is T.ivec3:
        return "vec3<i32>"
    if t is T.u32:
        return "u32"
    if t in (T.f32, float):
        return "f32"
    return "i32"


def pack_order(fields: list[tuple[str, str]]) -> list[tuple[str, str]]:
    """Field order that fills vec3 holes: vec4s, each vec3 followed by the next
    scalar, vec2s, the remaining scalars (optimize_struct_layout)."""
    v4 = [f for f in fields if f[1].startswith("vec4")]
    v3 = [f for f in fields if f[1].startswith("vec3")]
    v2 = [f for f in fields if f[1].startswith("vec2")]
    sc = [f for f in fields if not f[1].startswith("vec")]
    out = list(v4)
    for f in v3:
        out.append(f)
        if sc:
            out.append(sc.pop(0))
    return out + v2 + sc


def struct_layout(fields: list[tuple[str, str]]) -> tuple[dict[str, tuple[str, int]], int]:
    """{name: (wgsl type, byte offset)} and the stride (aligned to the largest
    member alignment, at least 16 bytes)."""
    off, max_al, out = 0, 4, {}
    for name, ty in fields:
        sz, al = _SIZE_ALIGN.get(ty, (4, 4))
        max_al = max(max_al, al)
        off += (-off) % al
        out[name] = (ty, off)
        off += sz
    off += (-off) % max_al
    return out, max(off, 16)


def _struct_of(cls: type, with_rng: bool) -> tuple[dict, int]:
    raw = [("_rng_state", "u32")] if with_rng else []
    raw += [(k, wgsl_type(v)) for k, v in T.data_fields(cls).items()]
    return struct_layout(pack_order(raw))


def _pack_records(layout: dict, stride: int, n_records: int, columns: dict[str, np.ndarray], n_used: int) -> bytes:
    buf = np.zeros((n_records, stride), dtype=np.uint8)
    for name, (ty, off) in layout.items():
        if ty.startswith("vec3"):
            for k, a in enumerate("xyz"):
                col = columns.get(f"{name}.{a}")
                if col is not None and n_used:
                    dt = np.float32 if ty == "vec3<f32>" else np.int32
                    buf[:n_used, off + 4 * k:off + 4 * k + 4] = np.ascontiguousarray(col[:n_used], dt) \
                        .view(np.uint8).reshape(n_used, 4)
        else:
            col = columns.get(name)
            if col is not None and n_used:
                dt = {"f32": np.float32, "u32": np.uint32}.get(ty, np.int32)
                buf[:n_used, off:off + 4] = np.ascontiguousarray(np.asarray(col[:n_used]).astype(dt)) \
                    .view(np.uint8).reshape(n_used, 4)
    return buf.tobytes()


def _unpack_records(raw: bytes, fields: dict, stride: int, n: int) -> dict[str, np.ndarray]:
    rec = np.frombuffer(raw, dtype=np.uint8)[: n * stride].reshape(n, stride)
    out = {}
    for name, spec in fields.items():
        ty, off = spec["type"], int(spec["offset"])
        if ty.startswith("vec3"):
            dt = np.float32 if ty == "vec3<f32>" else np.int32
            for k, a in enumerate("xyz"):
                out[f"{name}.{a}"] = np.ascontiguousarray(rec[:, off + 4 * k:off + 4 * k + 4]).view(dt).ravel()
        else:
            base = ty.replace("atomic<", "").rstrip(">")
            dt = {"f32": np.float32, "u32": np.uint32}.get(base, np.int32)
            out[name] = np.ascontiguousarray(rec[:, off:off + 4]).view(dt).ravel()
    return out


def _uniforms(engine: Any) -> tuple[dict, int, bytes]:
    """Uniform block of the reference: tissue_grid_dim (vec3<u32>),
    tissue_voxel_size, then the params sorted by name (get_config)."""
    params = engine._sim._params
    entries = [("tissue_grid_dim", "vec3<u32>"), ("tissue_voxel_size", "f32")]
    hints = T.param_fields(type(params))
    entries += [(k, wgsl_type(hints[k])) for k in sorted(hints)]
    layout, _ = struct_layout(entries)
    size = max((off + _SIZE_ALIGN.get(ty, (4, 4))[0] for ty, off in layout.values()), default=0)
    size += (-size) % 16
    buf = bytearray(size)
    for name, (ty, off) in layout.items():
        if name == "tissue_grid_dim":
            struct.pack_into("3I", buf, off, *(int(v) for v in engine.tissue_shape))
        elif name == "tissue_voxel_size":
            struct.pack_into("f", buf, off, float(engine.tissue_voxel_size))
        else:
            v = getattr(params, name)
            if ty == "vec3<f32>":
                struct.pack_into("3f", buf, off, v.x, v.y, v.z)
            elif ty == "vec3<i32>":
                struct.pack_into("3i", buf, off, int(v.x), int(v.y), int(v.z))
            elif ty == "f32":
                struct.pack_into("f", buf, off, float(v))
            else:
                struct.pack_into("I" if ty == "u32" else "i", buf, off, int(v))
    return {k: {"type": ty, "offset": off} for k, (ty, off) in layout.items()}, size, bytes(buf)


def _json_value(v: Any) -> Any:
    if isinstance(v, (T.vec3, T.ivec3)):
        return [v.x, v.y, v.z]
    if isinstance(v, (np.generic,)):
        return v.item()
    return v


def export_bundle(engine: Any, directory: str, exact: bool = True) -> str:
    """Writes the engine's current state as a bundle into `directory` (created
    if missing); returns the path of config.json."""
    be = engine._backend_impl
    if be is None:
        raise RuntimeError("export_bundle() needs a loaded model (Engine.load_model)")
    os.makedirs(directory, exist_ok=True)
    L = be.layout
    sd = be.state_dict()
    n = len(sd["cols"]["pos.x"])
    cell_layout, cell_stride = _struct_of(L.cell_class, with_rng=True)
    chem_layout, chem_stride = _struct_of(L.chem_class, with_rng=False)
    tissue_layout, tissue_stride = _struct_of(L.tissue_class, with_rng=False)
    uni_fields, uni_size, uni_bytes = _uniforms(engine)
    cap = int(be.caps.max_agents)
    files = {}
    with open(os.path.join(directory, "cells_in.bin"), "wb") as fh:
        fh.write(_pack_records(cell_layout, cell_stride, cap, sd["cols"], n))
    files["Cells_In"] = "cells_in.bin"
    with open(os.path.join(directory, "state.bin"), "wb") as fh:
        fh.write(struct.pack("2I", n, n))
    files["State"] = "state.bin"
    with open(os.path.join(directory, "uniforms.bin"), "wb") as fh:
        fh.write(uni_bytes)
    files["UniformBuffer"] = "uniforms.bin"
    shape = tuple(int(v) for v in engine.chemistry_shape)
    chem_cols = {}
    for i, name in enumerate(L.chem_fields):
        vals = be._field_values(i, be._current()[1])  # x fastest, FP32 (16-bit: value + residual)
        chem_cols[name] = vals.reshape(shape, order="F").ravel(order="C")
    for name in T.data_fields(L.chem_class):
        if name not in chem_cols:
            chem_cols[name] = np.asarray(engine.chemistry.column(name)).ravel(order="C")
    nvox = int(np.prod(shape))
    with open(os.path.join(directory, "chem_in.bin"), "wb") as fh:
        fh.write(_pack_records(chem_layout, chem_stride, nvox, chem_cols, nvox))
    files["Chem_In"] = "chem_in.bin"
    tissue_fields = T.data_fields(L.tissue_class)
    if engine.tissue is not None and tissue_fields and be._tissue_rules:
        be._read_tissue()  # the host grid follows the device's tissue rules
    if engine.tissue is not None and tissue_fields:
        tshape = tuple(int(v) for v in engine.tissue_shape)
        tcols = {k: np.asarray(engine.tissue.column(k)).ravel(order="C") for k in tissue_fields}
        ntv = int(np.prod(tshape))
        with open(os.path.join(directory, "tissue_in.bin"), "wb") as fh:
            fh.write(_pack_records(tissue_layout, tissue_stride, ntv, tcols, ntv))
        files["Tissue_In"] = "tissue_in.bin"
    else:
        files["Tissue_In"] = None
    if be.program is not None:
        with open(os.path.join(directory, "rules.cu"), "w", encoding="utf-8") as fh:
            fh.write(be.program.source)
    if exact:
        flat = {"meta": np.frombuffer(json.dumps({k: sd[k] for k in ("format", "layout", "step_state",
                                                                         "engine_step")}).encode(), np.uint8)}
        for k, v in sd["cols"].items():
            flat[f"col/{k}"] = v
        for group in ("fields", "sinks", "residuals"):
            for k, v in sd[group].items():
                if v is not None:
                    flat[f"{group}/{k}"] = v
        if sd.get("tissue") is not None:
            flat["tissue"] = sd["tissue"]
        np.savez(os.path.join(directory, "resume.npz"), **flat)
        files["resume"] = "resume.npz"

    def struct_json(layout, stride):
        return {"stride": stride, "fields": {k: {"type": ty, "offset": off} for k, (ty, off) in layout.items()}}

    execution_order = []
    if be.program is not None:
        cells = [k for k, kind in be.program.kernels if kind == 0]
        metrics = [k for k, kind in be.program.kernels if kind == 1]
    else:
        cells, metrics = [], []
    for name in L.chem_fields:
        if name in engine._diffusion:
            execution_order.append({"pass": "chem", "kernels": [f"diffusion:{name}"],
                                    "iterations": engine.substeps_for(name)})
    execution_order.append({"pass": "sort", "kernels": ["k_keys", "k_scan_hist", "k_onesweep", "k_bin_ranges",
                                                        "k_permute"], "iterations": 1})
    if cells:
        execution_order.append({"pass": "cell", "kernels": cells, "iterations": 1})
    if engine._contact is not None:
        execution_order.append({"pass": "contact", "kernels": ["k_contact"], "iterations": 1})
    if metrics:
        execution_order.append({"pass": "metric", "kernels": metrics, "iterations": 1})
    params = engine._sim._params
    config = {
        "params": {k: _json_value(getattr(params, k)) for k in params.__dataclass_fields__},
        "layout": {"tissue_shape": list(engine.tissue_shape), "chemistry_shape": list(engine.chemistry_shape),
                   "max_agents": cap,
                   "structs": {"cell": struct_json(cell_layout, cell_stride),
                               "chem": struct_json(chem_layout, chem_stride),
                               "tissue": struct_json(tissue_layout, tissue_stride)},
                   "uniforms": {"size": uni_size, "fields": uni_fields}},
        "execution_order": execution_order,
        "shader_path": "rules.cu" if be.program is not None else None,
        "buffers": files,
    }
    path = os.path.join(directory, "config.json")
    with open(path, "w", encoding="utf-8") as fh:
        json.dump(config, fh, indent=2)
    return path


def import_bundle(engine: Any, directory: str) -> None:
    """Loads a bundle into an engine whose model is loaded (Engine.load_model
    with the same model, geometry and capacity).  With resume.npz the state
    is restored exactly (load_state_dict); otherwise the agents, chemistry and
    tissue records are read through config.json's struct layout and uploaded
    as the host state (sync_to_device)."""
    be = engine._backend_impl
    if be is None:
        raise RuntimeError("import_bundle() needs a loaded model (Engine.load_model)")
    with open(os.path.join(directory, "config.json"), encoding="utf-8") as fh:
        config = json.load(fh)
    lay = config["layout"]
    if tuple(lay["chemistry_shape"]) != tuple(engine.chemistry_shape) or \
            tuple(lay["tissue_shape"]) != tuple(engine.tissue_shape):
        raise ValueError("bundle grid shapes differ from the engine's")
    bufs = config.get("buffers") or {}
    if bufs.get("resume") and os.path.exists(os.path.join(directory, bufs["resume"])):
        z = np.load(os.path.join(directory, bufs["resume"]))
        meta = json.loads(bytes(z["meta"]).decode())
        sd = dict(meta)
        sd["cols"] = {k[4:]: z[k] for k in z.files if k.startswith("col/")}
        for group in ("fields", "sinks", "residuals"):
            sd[group] = {f: (z[f"{group}/{f}"] if f"{group}/{f}" in z.files else None) for f in be.layout.chem_fields}
        sd["tissue"] = z["tissue"] if "tissue" in z.files else None
        sd["params"] = _params_from_json(engine, config.get("params", {}))
        be.load_state_dict(sd)
        return
    # a bundle without the exact record: records through the recorded layout
    with open(os.path.join(directory, bufs["State"]), "rb") as fh:
        n = struct.unpack_from("I", fh.read(8), 0)[0]
    cs = lay["structs"]["cell"]
    with open(os.path.join(directory, bufs["Cells_In"]), "rb") as fh:
        cols = _unpack_records(fh.read(), cs["fields"], int(cs["stride"]), n)
    L = be.layout
    want = {c: dt for c, _, dt in L.cell_cols}
    host = {c: (cols[c].astype(dt) if c in cols else np.zeros(n, dt)) for c, dt in want.items()}
    engine.cells._set_columns(host, L.cell_class)
    shape = tuple(int(v) for v in engine.chemistry_shape)
    if bufs.get("Chem_In"):
        ch = lay["structs"]["chem"]
        nvox = int(np.prod(shape))
        with open(os.path.join(directory, bufs["Chem_In"]), "rb") as fh:
            chem = _unpack_records(fh.read(), ch["fields"], int(ch["stride"]), nvox)
        for name, v in chem.items():
            if name in T.data_fields(L.chem_class):
                engine.chemistry.column(name)[...] = v.reshape(shape)
    if bufs.get("Tissue_In") and engine.tissue is not None:
        ts = lay["structs"]["tissue"]
        tshape = tuple(int(v) for v in engine.tissue_shape)
        with open(os.path.join(directory, bufs["Tissue_In"]), "rb") as fh:
            tis = _unpack_records(fh.read(), ts["fields"], int(ts["stride"]), int(np.prod(tshape)))
        for name, v in tis.items():
            if name in T.data_fields(L.tissue_class):
                engine.tissue.column(name)[...] = v.reshape(tshape)
    params = _params_from_json(engine, config.get("params", {}))
    if params:
        engine.update_params(**params)
    be.sync_to_device()


def _params_from_json(engine: Any, raw: dict) -> dict:
    hints = T.param_fields(type(engine._sim._params))
    out = {}
    for k, v in raw.items():
        t = hints.get(k)
        if t is None:
            continue
        if t is T.vec3:
            out[k] = T.vec3(*v)
        elif t is T.ivec3:
            out[k] = T.ivec3(*v)
        elif t in (T.f32, float):
            out[k] = float(v)
        elif t is bool:
            out[k] = bool(v)
        else:
            out[k] = int(v)
    return out
