"""Rule-DSL interpreter on the CPU (TEST INFRASTRUCTURE — the checker for the
rule translator; the product never imports it).

It runs the model's own Python rule functions, agent by agent, with the
semantics the CUDA kernels implement, restated from the reference:
  * rules read the pre-rule state of neighbours and write a new buffer
    (ping-pong, framework/src/oncolytica/gpu/runtime/_gpu_backend.py:144-149);
  * the per-agent RNG is xorshift32 (template.wgsl:75-82), random_dir two
    draws (:84-98), children get parent_rng ^ 0x12345678
    (engine/assets/shaders/tumor_sim.wgsl:694);
  * die() flags the agent for removal at the next sort
    (_stmt_translator.py:431-440, template.wgsl:152-159);
  * divide() appends one child in parent order (:442-453);
  * neighbors: 27 bins in MooreOffsets order (template.wgsl:11-21), bins
    outside the grid skipped, self skipped (_stmt_translator.py:459-491);
  * chemistry_at / tissue_at: clamped nearest voxel (_types.py:314-346);
  * tissue and chemistry rules (_stmt_translator.py:493-605, with the
    reference's undefined symbols resolved): one call per voxel, reading the
    state before the rule (Tissue_In / Chem_In) and writing a new grid;
    .neighbors are the 26 in-grid Moore voxels in MooreOffsets order,
    tissue .cells the voxel's bin in sorted order, chemistry .cells and
    .tissues its 2 x 2 x 2 tissue voxels in tissue-key order.
Arithmetic is float32 (numpy scalars), matching the kernels' separately
rounded operations except for library functions (cos, sin, log, ...).
Suitable for small cases only (a Python call per agent).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

import oracle  # noqa: E402  (the C oracle: keys, sort, bins, diffusion, contact)

from oncolytica_b200 import _types as T  # noqa: E402
from oncolytica_b200._containers import column_names  # noqa: E402

F = np.float32


def _bin_coord(p, vs, dim) -> int:
    q = F(p) / F(vs)
    if q != q:
        return 0
    c = int(np.trunc(q)) if abs(float(q)) < 2.0e9 else (dim - 1 if q > 0 else 0)
    return min(max(c, 0), dim - 1)


class _Sink:
    def __init__(self, interp, idx):
        object.__setattr__(self, "_i", interp)
        object.__setattr__(self, "_v", idx)

    def __getattr__(self, name):
        return F(0.0)

    def __setattr__(self, name, value):
        self._i.deposits.append((name, self._v, F(value)))


class _MetricAcc:
    def __init__(self, fields):
        object.__setattr__(self, "_f", fields)
        for k, t in fields.items():
            object.__setattr__(self, k, F(0.0) if t in T._FLOAT_TYPES else 0)

    def __setattr__(self, name, value):
        t = self._f[name]
        object.__setattr__(self, name, F(value) if t in T._FLOAT_TYPES else int(value))


class Interpreter(T.RuleHooks):
    """State: columns as in CudaBackend.snapshot() (device order, dead rows
    included), fields as flat x-fastest arrays, tissue columns as (X, Y, Z)."""

    def __init__(self, sim, engine_cfg: dict, snap: dict):
        self.sim = sim
        self.spec = sim._spec
        self.cfg = engine_cfg
        self.fields_spec = T.data_fields(self.spec.cell_class)
        self.cols = column_names({"pos": T.vec3, **{k: v for k, v in self.fields_spec.items() if k != "pos"}})
        self.rows = int(snap["rows"])
        self.data = {c: np.array(snap["cols"][c][: self.rows]) for c, _, _ in self.cols}
        self.data["_rng_state"] = np.array(snap["cols"]["_rng_state"][: self.rows], dtype=np.uint32)
        self.life = np.array(snap["life"][: self.rows], dtype=np.uint8)
        self.fields = {k: np.array(v, dtype=np.float32) for k, v in snap["fields"].items()}
        self.sinks = {k: (np.array(v, dtype=np.float32) if v is not None else None) for k, v in snap["sinks"].items()}
        self.tissue = snap.get("tissue") or engine_cfg.get("tissue_cols")  # the device's, when rules update it
        if self.tissue is not None:
            self.tissue = {k: np.array(v) for k, v in self.tissue.items()}

    # ---- hooks -----------------------------------------------------------
    def random(self) -> np.float32:
        s = self.rng
        s ^= (s << 13) & 0xFFFFFFFF
        s ^= s >> 17
        s ^= (s << 5) & 0xFFFFFFFF
        self.rng = s
        return F(F(s) * F(2.3283064365386963e-10))

    def random_dir(self) -> T.vec3:
        r1, r2 = self.random(), self.random()
        z = r1 * F(2.0) - F(1.0)
        phi = r2 * F(6.283185307179586)
        rxy = np.sqrt(np.fmax(F(0.0), F(1.0) - z * z))
        return T.vec3(rxy * np.cos(phi), rxy * np.sin(phi), z)

    def die(self, cell) -> None:
        self.dead = True

    def divide(self, cell, child) -> None:
        if self.born is not None:
            self.multi = True
            return
        c = child.copy()
        object.__setattr__(c, "_rng_state", (self.rng ^ 0x12345678) & 0xFFFFFFFF)
        self.born = c

    def neighbors(self, cell):
        td, vs = self.cfg["tissue_dims"], self.cfg["tissue_voxel_size"]
        bc = [_bin_coord(getattr(cell.pos, a), vs, td[k]) for k, a in enumerate("xyz")]
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    nx, ny, nz = bc[0] + dx, bc[1] + dy, bc[2] + dz
                    if not (0 <= nx < td[0] and 0 <= ny < td[1] and 0 <= nz < td[2]):
                        continue
                    k = oracle.tissue_key(nx, ny, nz)
                    s, e = int(self.ranges[2 * k]), int(self.ranges[2 * k + 1])
                    for j in range(s, e):
                        if j == self.i:
                            continue
                        yield self._load(self.src, j)

    def _chem_index(self, pos) -> int:
        cd, vs = self.cfg["chem_dims"], self.cfg["chem_voxel_size"]
        cx, cy, cz = (_bin_coord(getattr(pos, a), vs, cd[k]) for k, a in enumerate("xyz"))
        return (cz * cd[1] + cy) * cd[0] + cx

    def chemistry_at(self, pos):
        cd, vs = self.cfg["chem_dims"], self.cfg["chem_voxel_size"]
        return self._chem_voxel(*(_bin_coord(getattr(pos, a), vs, cd[k]) for k, a in enumerate("xyz")))

    def tissue_at(self, pos):
        td, vs = self.cfg["tissue_dims"], self.cfg["tissue_voxel_size"]
        return self._tissue_voxel(*(_bin_coord(getattr(pos, a), vs, td[k]) for k, a in enumerate("xyz")))

    def sink_at(self, pos):
        return _Sink(self, self._chem_index(pos))

    # ---- voxels (tissue / chemistry rules) -------------------------------
    def _tissue_voxel(self, x: int, y: int, z: int):
        t = self.spec.tissue_class()
        if self.tissue is not None:
            for name, arr in self.tissue.items():
                v = arr[x, y, z]
                ft = T.data_fields(self.spec.tissue_class).get(name)
                setattr(t, name, F(v) if ft in T._FLOAT_TYPES else (bool(v) if ft is bool else int(v)))
        object.__setattr__(t, "_vox", (x, y, z))
        return t

    def _chem_voxel(self, x: int, y: int, z: int):
        cd = self.cfg["chem_dims"]
        c = self.spec.chemistry_class()
        v = (z * cd[1] + y) * cd[0] + x
        for name in self.fields:
            setattr(c, name, self.fields[name][v])
        object.__setattr__(c, "_vox", (x, y, z))
        return c

    def _sub_tissue(self, chem):
        x, y, z = chem._vox
        td = self.cfg["tissue_dims"]
        for i in range(8):
            tx, ty, tz = 2 * x + (i & 1), 2 * y + ((i >> 1) & 1), 2 * z + ((i >> 2) & 1)
            if tx < td[0] and ty < td[1] and tz < td[2]:
                yield tx, ty, tz

    def _bin_rows(self, x, y, z):
        k = oracle.tissue_key(x, y, z)
        s, e = int(self.ranges[2 * k]), int(self.ranges[2 * k + 1])
        for j in range(s, e):
            yield self._load(self.data, j)

    def voxel_neighbors(self, voxel):
        tissue = isinstance(voxel, T.Tissue)
        dims = self.cfg["tissue_dims"] if tissue else self.cfg["chem_dims"]
        x, y, z = voxel._vox
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    if dx == 0 and dy == 0 and dz == 0:
                        continue
                    nx, ny, nz = x + dx, y + dy, z + dz
                    if not (0 <= nx < dims[0] and 0 <= ny < dims[1] and 0 <= nz < dims[2]):
                        continue
                    yield self._tissue_voxel(nx, ny, nz) if tissue else self._chem_voxel(nx, ny, nz)

    def voxel_cells(self, voxel):
        if isinstance(voxel, T.Tissue):
            yield from self._bin_rows(*voxel._vox)
            return
        for tx, ty, tz in self._sub_tissue(voxel):
            yield from self._bin_rows(tx, ty, tz)

    def voxel_tissues(self, chem):
        for tx, ty, tz in self._sub_tissue(chem):
            yield self._tissue_voxel(tx, ty, tz)

    def run_tissue_rules(self, rules) -> None:
        td = self.cfg["tissue_dims"]
        names = list(T.data_fields(self.spec.tissue_class))
        for rule in rules:
            out = {k: v.copy() for k, v in self.tissue.items()}
            for z in range(td[2]):
                for y in range(td[1]):
                    for x in range(td[0]):
                        t = self._tissue_voxel(x, y, z)
                        tok = T.install_rule_hooks(self)
                        try:
                            rule(t)
                        finally:
                            T.reset_rule_hooks(tok)
                        for name in names:
                            out[name][x, y, z] = getattr(t, name)
            self.tissue = out

    def run_chemistry_rules(self, rules) -> None:
        cd = self.cfg["chem_dims"]
        for rule in rules:
            for _ in range(int(getattr(rule, "_iterations", 1))):
                out = {k: v.copy() for k, v in self.fields.items()}
                for z in range(cd[2]):
                    for y in range(cd[1]):
                        for x in range(cd[0]):
                            c = self._chem_voxel(x, y, z)
                            tok = T.install_rule_hooks(self)
                            try:
                                rule(c)
                            finally:
                                T.reset_rule_hooks(tok)
                            v = (z * cd[1] + y) * cd[0] + x
                            for name in out:
                                out[name][v] = F(getattr(c, name))
                self.fields = out

    # ---- state -----------------------------------------------------------
    def _load(self, src: dict, i: int):
        kw = {}
        for fname, t in self.fields_spec.items():
            if t in (T.vec3, T.ivec3):
                kw[fname] = t(*(src[f"{fname}.{a}"][i] for a in "xyz"))
            else:
                v = src[fname][i]
                kw[fname] = bool(v) if t is bool else v
        c = self.spec.cell_class(**kw)
        object.__setattr__(c, "_rng_state", int(src["_rng_state"][i]))
        return c

    def _store(self, dst: dict, i: int, c) -> None:
        for fname, t in self.fields_spec.items():
            v = getattr(c, fname)
            if t in (T.vec3, T.ivec3):
                for a in "xyz":
                    dst[f"{fname}.{a}"][i] = getattr(v, a)
            else:
                dst[fname][i] = v
        dst["_rng_state"][i] = c._rng_state

    def sort(self) -> None:
        """Keys, stable sort, compaction, bin table (the grid stage)."""
        td, vs = self.cfg["tissue_dims"], self.cfg["tissue_voxel_size"]
        pos = np.stack([self.data["pos.x"], self.data["pos.y"], self.data["pos.z"]], axis=1)
        keys = oracle.keys(pos, td, vs, self.life)
        ks, perm = oracle.sort_pairs(keys)
        n = int((self.life == 0).sum())
        sentinel = oracle.tissue_key(*td)
        self.ranges = oracle.bin_ranges(ks, sentinel)
        self.data = {k: v[perm[:n]].copy() for k, v in self.data.items()}
        self.rows = n
        self.n_live = n
        self.life = np.zeros(n, np.uint8)

    def run_cell_rules(self, rules) -> dict:
        """Each rule over the live rows, In -> Out; returns counters."""
        births = 0
        multi = False
        for rule in rules:
            src = self.data
            dst = {k: v.copy() for k, v in src.items()}
            self.src = src
            children = []
            for i in range(self.n_live):
                self.i = i
                cell = self._load(src, i)
                self.rng = int(cell._rng_state)
                self.dead = False
                self.born = None
                self.multi = False
                self.deposits = []
                tok = T.install_rule_hooks(self)
                try:
                    rule(cell)
                finally:
                    T.reset_rule_hooks(tok)
                object.__setattr__(cell, "_rng_state", self.rng)
                self._store(dst, i, cell)
                if self.dead:
                    self.life[i] = 1
                for name, v, val in self.deposits:
                    self.sinks[name][v] = self.sinks[name][v] + val
                if self.born is not None:
                    children.append(self.born)
                multi |= self.multi
            cap = self.cfg["capacity"]
            room = max(0, cap - self.rows)
            children = children[:room]
            base = self.rows
            for k in dst:
                dst[k] = np.concatenate([dst[k], np.zeros(len(children), dst[k].dtype)])
            for j, c in enumerate(children):
                self._store(dst, base + j, c)
            self.life = np.concatenate([self.life, np.zeros(len(children), np.uint8)])
            self.rows += len(children)
            births += len(children)
            self.data = dst
        return {"births": births, "multi": multi}

    def run_metric_rules(self, rules, metrics_cls) -> dict:
        acc = _MetricAcc(T.metric_fields(metrics_cls))
        for rule in rules:
            for i in range(self.rows):
                if self.life[i]:
                    continue
                self.i = i
                cell = self._load(self.data, i)
                self.rng = int(cell._rng_state)
                tok = T.install_rule_hooks(self)
                try:
                    rule(cell, acc)
                finally:
                    T.reset_rule_hooks(tok)
        return {k: getattr(acc, k) for k in T.metric_fields(metrics_cls)}

    def diffuse(self, name: str, spec: dict) -> None:
        cd = self.cfg["chem_dims"]
        f = self.fields[name].reshape(cd[::-1])
        s = self.sinks.get(name)
        out = oracle.diffuse(f, s.reshape(cd[::-1]) if s is not None else None, self.cfg["chem_voxel_size"],
                             self.cfg["dt"], spec["diffusion"], spec["decay"], spec["boundary"], spec["substeps"])
        self.fields[name] = out.ravel()
        if s is not None:
            self.sinks[name] = np.zeros_like(s)

    def snapshot(self) -> dict:
        return {"rows": self.rows, "life": self.life.copy(), "cols": {k: v.copy() for k, v in self.data.items()},
                "fields": {k: v.copy() for k, v in self.fields.items()},
                "tissue": {k: v.copy() for k, v in self.tissue.items()} if self.tissue is not None else None,
                "sinks": {k: (v.copy() if v is not None else None) for k, v in self.sinks.items()}}


def engine_cfg(engine) -> dict:
    """What the interpreter needs from a loaded Engine."""
    cfg = {"tissue_dims": tuple(engine.tissue_shape), "tissue_voxel_size": float(engine.tissue_voxel_size),
           "chem_dims": tuple(engine.chemistry_shape), "chem_voxel_size": float(engine.chemistry_voxel_size),
           "capacity": int(engine.max_agents), "dt": float(engine.dt)}
    if engine.tissue is not None:
        cfg["tissue_cols"] = {k: np.asarray(engine.tissue.column(k)) for k in engine.tissue._fields}
    return cfg


def step(interp: Interpreter, engine, collect: bool = False) -> dict:
    """One step with the CUDA backend's stage order (fields, grid, cell rules;
    no contact) and optionally the metric rules."""
    for name, d in engine._diffusion.items():
        interp.diffuse(name, {"diffusion": d.diffusion, "decay": d.decay, "boundary": d.boundary,
                              "substeps": engine.substeps_for(name)})
    interp.sort()
    if engine._tissue_rules:
        interp.run_tissue_rules(engine._tissue_rules)
    if engine._chemistry_rules:
        interp.run_chemistry_rules(engine._chemistry_rules)
    out = interp.run_cell_rules(engine._cell_rules)
    if collect:
        out["metrics"] = interp.run_metric_rules(engine._metric_rules, engine._sim._spec.metrics_class)
    return out
