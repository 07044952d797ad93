"""Translate a model's rules to CUDA C.

Reference behaviour followed (framework/src/oncolytica/gpu/compiler/):
  * rules found by their decorator tag, emitted per kind as separate kernels
    named like the reference's Kernel_CellRule_i / Kernel_MetricRule_i
    (_compiler.py:321-348);
  * per-agent wrapper: load agent, local RNG, body, store RNG, write Out
    (_shader_builder.py:207-221); early returns keep the epilogue
    (translator/_context.py:417-426) — here the body is a function, so a
    ``return`` simply returns to the wrapper;
  * helpers: simulation methods as sim_<name>, data-class methods as
    <kind>_<name> with the receiver and mutated arguments passed by reference
    (_compiler.py:59-201);
  * ``self.params.X`` reads the Params blob (_expr_translator.py:101-107);
    ``ol.random()``/``ol.random_dir()`` use the agent's RNG (:204-216);
    ``tissue_at``/``chemistry_at`` are clamped nearest-voxel lookups (:243-260);
  * ``cell.neighbors`` loops over the 27 bins, skipping out-of-range bins and
    self (_stmt_translator.py:459-491); ``die()``/``divide()`` (:431-453).
Intended (CPU-backend) meaning is kept where the reference translator
diverges: ``for i in range(n)`` loops and loops inside helpers are emitted,
constructor keyword arguments are kept, class defaults initialise new agents.
"""
from __future__ import annotations

import ast
import hashlib
import inspect
import math
import textwrap
import typing
from dataclasses import dataclass, field
from typing import Any

import numpy as np

import oncolytica_b200 as _pkg
from oncolytica_b200 import _math as olmath
from oncolytica_b200 import _types as T
from oncolytica_b200._containers import column_names
from oncolytica_b200._errors import CompilationError

# ------------------------------------------------------------------ types

F32, I32, U32, BOOL, VEC3, IVEC3, VOID = "f32", "i32", "u32", "bool", "vec3", "ivec3", "void"
NUMERIC = (F32, I32, U32, BOOL)
CTYPE = {F32: "float", I32: "int", U32: "olc_u32", BOOL: "bool", VEC3: "olc_vec3", IVEC3: "olc_ivec3",
         VOID: "void"}
ZERO = {F32: "0.0f", I32: "0", U32: "0u", BOOL: "false", VEC3: "olc_v3(0.0f, 0.0f, 0.0f)",
        IVEC3: "olc_iv3(0, 0, 0)"}
KINDS = ("Cell", "Chemistry", "Tissue")
STRUCT_NAME = {"Cell": "Cell_t", "Chemistry": "Chem_t", "Tissue": "Tissue_t"}


def ty_of_py(t: Any) -> str | None:
    """DSL annotation -> translator type."""
    if t in (T.f32, float):
        return F32
    if t in (T.i32, int):
        return I32
    if t is T.u32:
        return U32
    if t is bool:
        return BOOL
    if t is T.vec3:
        return VEC3
    if t is T.ivec3:
        return IVEC3
    if isinstance(t, type):
        for k in KINDS:
            if issubclass(t, getattr(T, k)):
                return ("struct", k)
    origin = typing.get_origin(t)
    if origin in (tuple, typing.Tuple):
        elems = tuple(ty_of_py(a) for a in typing.get_args(t))
        if any(e is None for e in elems):
            return None
        return ("tuple", elems)
    return None


def ctype(t) -> str:
    if isinstance(t, tuple):
        if t[0] == "struct":
            return STRUCT_NAME[t[1]]
        if t[0] == "tuple":
            return tuple_struct_name(t[1])
    return CTYPE[t]


def tuple_struct_name(elems) -> str:
    return "Tup_" + "_".join(e if isinstance(e, str) else ctype(e) for e in elems)


def is_struct(t) -> bool:
    return isinstance(t, tuple) and t[0] == "struct"


def promote(a, b):
    if a == F32 or b == F32:
        return F32
    if a == U32 and b == U32:
        return U32
    return I32


def fmt_float(v: float) -> str:
    v = float(v)
    if math.isnan(v):
        return "__int_as_float(0x7fc00000)"
    if math.isinf(v):
        return "__int_as_float(0x7f800000)" if v > 0 else "__int_as_float(0xff800000)"
    f = np.float32(v)
    r = repr(float(f))
    if "e" not in r and "." not in r:
        r += ".0"
    return r + "f"


def fmt_int(v: int) -> str:
    if -(1 << 31) <= v < (1 << 31):
        return str(int(v))
    if 0 <= v < (1 << 32):
        return f"{int(v)}u"
    raise CompilationError(f"integer constant {v} does not fit 32 bits")


# ------------------------------------------------------------------ layout

@dataclass
class ModelLayout:
    cell_class: type
    chem_class: type
    tissue_class: type
    metrics_class: type
    params_class: type
    cell_fields: dict
    cell_cols: list                 # (column, field, numpy dtype)
    rng_col: int
    chem_fields: list               # names of float fields, field index = position
    tissue_fields: dict
    params: dict                    # name -> (offset, ty)
    params_size: int
    metrics: dict                   # name -> (slot, ty)
    radius_field: str | None = None
    batched: bool = False           # a `_sim` column (simulation index) follows `_rng_state`

    def col_index(self, col: str) -> int:
        for i, (c, _, _) in enumerate(self.cell_cols):
            if c == col:
                return i
        raise KeyError(col)


@dataclass
class Program:
    source: str
    kernels: list                   # (name, kind): 0 cell rule, 1 metric rule, 2 tissue rule, 3 chemistry rule
    layout: ModelLayout
    sink_fields: set = field(default_factory=set)
    digest: str = ""
    iterations: list = field(default_factory=list)  # per kernel (chemistry rules' iterations, else 1)


def make_layout(spec, radius_field: str | None = None, batched: bool = False) -> ModelLayout:
    cell_fields = T.data_fields(spec.cell_class)
    if cell_fields.get("pos") is not T.vec3:
        raise CompilationError(f"Class '{spec.cell_class.__name__}' must have attribute 'pos: ol.vec3'.")
    for name, t in cell_fields.items():
        if ty_of_py(t) is None or is_struct(ty_of_py(t)):
            raise CompilationError(f"unsupported type {t!r} for {spec.cell_class.__name__}.{name}")
    ordered = {"pos": cell_fields["pos"]}
    ordered.update({k: v for k, v in cell_fields.items() if k != "pos"})
    cols = column_names(ordered) + [("_rng_state", "_rng_state", np.uint32)]
    rng_col = len(cols) - 1
    if batched:
        cols.append(("_sim", "_sim", np.uint32))
    # device fields are the float32 chemistry fields; others stay on the host
    chem_fields = {k: v for k, v in T.data_fields(spec.chemistry_class).items() if ty_of_py(v) == F32}
    tissue_fields = {k: v for k, v in T.data_fields(spec.tissue_class).items()}
    for name, t in tissue_fields.items():
        if ty_of_py(t) not in NUMERIC:
            raise CompilationError(f"tissue fields must be scalars: {spec.tissue_class.__name__}.{name}")
    params = {}
    off = 0
    for name, t in sorted(T.param_fields(spec.params_class).items()):
        ty = ty_of_py(t)
        params[name] = (off, ty)
        off += 12 if ty in (VEC3, IVEC3) else 4
    metrics = {}
    for slot, (name, t) in enumerate(T.metric_fields(spec.metrics_class).items()):
        ty = ty_of_py(t)
        if ty not in NUMERIC:
            raise CompilationError(f"metric fields must be scalars: {spec.metrics_class.__name__}.{name}")
        metrics[name] = (slot, ty)
    if radius_field is not None and ty_of_py(cell_fields.get(radius_field)) != F32:
        raise CompilationError(f"contact radius field {radius_field!r} must be an ol.f32 field of the cell class")
    return ModelLayout(spec.cell_class, spec.chemistry_class, spec.tissue_class, spec.metrics_class,
                       spec.params_class, ordered, cols, rng_col, list(chem_fields), tissue_fields, params,
                       max(off, 4), metrics, radius_field, batched)


def pack_params(layout: ModelLayout, params_obj: Any) -> bytes:
    buf = bytearray(layout.params_size)
    for name, (off, ty) in layout.params.items():
        v = getattr(params_obj, name)
        if ty == F32:
            buf[off:off + 4] = np.float32(v).tobytes()
        elif ty in (I32, BOOL):
            buf[off:off + 4] = np.int32(int(v)).tobytes()
        elif ty == U32:
            buf[off:off + 4] = np.uint32(int(v)).tobytes()
        elif ty == VEC3:
            buf[off:off + 12] = np.array([v.x, v.y, v.z], np.float32).tobytes()
        elif ty == IVEC3:
            buf[off:off + 12] = np.array([v.x, v.y, v.z], np.int32).tobytes()
    return bytes(buf)


# ------------------------------------------------------------------ function sources

def resolve_hints(fn, spec) -> dict:
    """Type hints of a rule or helper.  String annotations (PEP 563) are
    evaluated in the function's module plus the model's own classes, so models
    whose classes are defined inside a function still resolve."""
    fn = getattr(fn, "__func__", fn)
    ns = dict(fn.__globals__)
    for cls in (spec.cell_class, spec.tissue_class, spec.chemistry_class, spec.metrics_class, spec.params_class):
        ns.setdefault(cls.__name__, cls)
    out = {}
    for name, ann in inspect.get_annotations(fn).items():
        if isinstance(ann, str):
            try:
                ann = eval(ann, ns)  # noqa: S307 - the user's own annotation text
            except Exception as exc:
                raise CompilationError(f"cannot resolve annotation {ann!r} of {fn.__qualname__}: {exc}")
        out[name] = ann
    return out

def func_ast(fn) -> tuple[ast.FunctionDef, str, str, int]:
    fn = getattr(fn, "__func__", fn)
    src = textwrap.dedent(inspect.getsource(fn))
    tree = ast.parse(src)
    for node in ast.walk(tree):
        if isinstance(node, ast.FunctionDef):
            try:
                line0 = inspect.getsourcelines(fn)[1] - 1
            except (OSError, TypeError):
                line0 = 0
            return node, src, inspect.getsourcefile(fn) or "<rule>", line0
    raise CompilationError(f"no function definition found for {fn!r}")


def strip_docstring(body):
    if body and isinstance(body[0], ast.Expr) and isinstance(body[0].value, ast.Constant) and \
            isinstance(body[0].value.value, str):
        return body[1:]
    return body


# ------------------------------------------------------------------ translator

@dataclass
class FuncInfo:
    cname: str
    pyfunc: Any
    kind: str                       # "rule", "metric", "sim", or a struct kind (method)
    params: list                    # (name, ty, by_ref)
    ret: Any
    node: ast.FunctionDef
    src: str
    filename: str
    line0: int


class Translator:
    def __init__(self, sim: Any, layout: ModelLayout, contact_radius: str | None):
        self.sim = sim
        self.spec = sim._spec
        self.L = layout
        self.contact_radius = contact_radius
        self.funcs: dict[str, FuncInfo] = {}
        self.order: list[str] = []
        self.tuples: set = set()
        self.sink_fields: set = set()
        self.constants: dict[str, str] = {}
        self._pending: list[str] = []

    # ---- helper discovery ------------------------------------------------
    def struct_class(self, kind: str) -> type:
        return {"Cell": self.spec.cell_class, "Chemistry": self.spec.chemistry_class,
                "Tissue": self.spec.tissue_class}[kind]

    def method_info(self, kind: str, name: str, node_for_err: ast.AST | None = None) -> FuncInfo:
        cname = f"{kind.lower()}_{name}"
        if cname in self.funcs:
            return self.funcs[cname]
        cls = self.struct_class(kind)
        fn = getattr(cls, name, None)
        if fn is None or not inspect.isfunction(fn) or any(name in vars(b) for b in T.BASE_CLASSES + [T.BaseData]):
            raise CompilationError(f"{cls.__name__} has no user method {name!r}", node_for_err)
        return self._register(cname, fn, kind)

    def sim_info(self, name: str, node_for_err: ast.AST | None = None) -> FuncInfo:
        cname = f"sim_{name}"
        if cname in self.funcs:
            return self.funcs[cname]
        fn = getattr(type(self.sim), name, None)
        if fn is None or not inspect.isfunction(fn):
            raise CompilationError(f"{type(self.sim).__name__} has no method {name!r}", node_for_err)
        if getattr(fn, "_rule_type", None) is not None:
            raise CompilationError(f"rule {name!r} cannot be called from another rule", node_for_err)
        return self._register(cname, fn, "sim")

    def _register(self, cname: str, fn, kind: str) -> FuncInfo:
        node, src, filename, line0 = func_ast(fn)
        hints = resolve_hints(fn, self.spec)
        params = []
        args = node.args.args
        start = 1  # skip self
        for a in args[start:]:
            t = ty_of_py(hints.get(a.arg))
            if t is None:
                raise CompilationError(f"parameter {a.arg!r} of {fn.__qualname__} needs a DSL type annotation", a,
                                       src, filename, line0)
            params.append([a.arg, t, False])
        ret = ty_of_py(hints["return"]) if "return" in hints and hints["return"] is not None else None
        info = FuncInfo(cname, fn, kind, params, ret, node, src, filename, line0)
        # by-reference: the receiver and any argument the body mutates
        mut = mutated_names(node)
        for p in info.params:
            if (is_struct(p[1]) or p[1] in (VEC3, IVEC3)) and p[0] in mut:
                p[2] = True
        info.self_by_ref = kind in KINDS and ("self" in mut or self._calls_mutating_self(node, kind))
        if isinstance(ret, tuple) and ret[0] == "tuple":
            self.tuples.add(ret[1])
        self.funcs[cname] = info
        self.order.append(cname)
        self._pending.append(cname)
        return info

    def _calls_mutating_self(self, node, kind) -> bool:
        # self.m() where m mutates self (one level; deeper chains are covered
        # because every method's self flag is computed on registration)
        for n in ast.walk(node):
            if isinstance(n, ast.Call) and isinstance(n.func, ast.Attribute) and \
                    isinstance(n.func.value, ast.Name) and n.func.value.id == "self":
                if n.func.attr in ("die", "divide"):
                    continue
                cls = self.struct_class(kind)
                if inspect.isfunction(getattr(cls, n.func.attr, None)):
                    sub, *_ = func_ast(getattr(cls, n.func.attr))
                    if sub is not node and "self" in mutated_names(sub):
                        return True
        return False

    # ---- emission ---------------------------------------------------------
    def build(self) -> Program:
        kernels = []
        bodies = []
        cell_rules = list(self.sim._engine._cell_rules)
        metric_rules = list(self.sim._engine._metric_rules)
        rule_infos = []
        for i, rule in enumerate(cell_rules):
            node, src, filename, line0 = func_ast(rule)
            args = node.args.args
            if len(args) != 2:
                raise CompilationError("a cell rule takes (self, cell)", node, src, filename, line0)
            info = FuncInfo(f"rule_cell_{i}", rule, "rule", [[args[1].arg, ("struct", "Cell"), True]], None, node,
                            src, filename, line0)
            info.self_by_ref = False
            rule_infos.append(info)
        metric_infos = []
        for i, rule in enumerate(metric_rules):
            node, src, filename, line0 = func_ast(rule)
            args = node.args.args
            if len(args) != 3:
                raise CompilationError("a metric rule takes (self, item, metrics)", node, src, filename, line0)
            hints = resolve_hints(rule, self.spec)
            item_t = ty_of_py(hints.get(args[1].arg))
            if item_t != ("struct", "Cell"):
                raise CompilationError("metric rules over tissue/chemistry voxels are not supported by this backend",
                                       node, src, filename, line0)
            info = FuncInfo(f"rule_metric_{i}", rule, "metric", [[args[1].arg, ("struct", "Cell"), False]], None,
                            node, src, filename, line0)
            info.self_by_ref = False
            info.metrics_name = args[2].arg
            metric_infos.append(info)

        voxel_infos = []  # (info, kind, iterations)
        eng = self.sim._engine
        for kind, rules in (("Tissue", list(getattr(eng, "_tissue_rules", []))),
                            ("Chemistry", list(getattr(eng, "_chemistry_rules", [])))):
            for i, rule in enumerate(rules):
                node, src, filename, line0 = func_ast(rule)
                args = node.args.args
                if len(args) != 2:
                    raise CompilationError(f"a {kind.lower()} rule takes (self, voxel)", node, src, filename, line0)
                info = FuncInfo(f"rule_{kind.lower()}_{i}", rule, "rule", [[args[1].arg, ("struct", kind), True]],
                                None, node, src, filename, line0)
                info.self_by_ref = False
                info.voxel_rule = True
                iters = int(getattr(rule, "_iterations", 1)) if kind == "Chemistry" else 1
                voxel_infos.append((info, kind, iters))

        for info in rule_infos + metric_infos + [v[0] for v in voxel_infos]:
            bodies.append(self.emit_function(info))
        # helpers reachable from rules (emission may discover more)
        helper_bodies = []
        done = set()
        while self._pending:
            cname = self._pending.pop(0)
            if cname in done:
                continue
            done.add(cname)
            helper_bodies.append(self.emit_function(self.funcs[cname]))
        protos = [self.prototype(self.funcs[c]) + ";" for c in self.order]

        for i, info in enumerate(rule_infos):
            kname = f"Kernel_CellRule_{i}"
            kernels.append((kname, 0))
            bodies.append(self.cell_kernel(kname, info.cname))
        for i, info in enumerate(metric_infos):
            kname = f"Kernel_MetricRule_{i}"
            kernels.append((kname, 1))
            bodies.append(self.metric_kernel(kname, info.cname))
        iterations = [1] * len(kernels)
        counters = {"Tissue": 0, "Chemistry": 0}
        for info, kind, iters in voxel_infos:
            i = counters[kind]
            counters[kind] += 1
            kname = f"Kernel_{'Tissue' if kind == 'Tissue' else 'Chem'}Rule_{i}"
            kernels.append((kname, 2 if kind == "Tissue" else 3))
            iterations.append(iters)
            bodies.append(self.voxel_kernel(kname, info.cname, kind))

        src = "\n".join([
            "// Generated by oncolytica_b200.compiler from the model's Python rules.",
            # solo metric rules add into per-block shared accumulators
            "" if self.L.batched else f"#define OLC_SOLO_METRIC_WORDS {max(1, len(self.L.metrics))}",
            '#include "olc_rule_rt.cuh"',
            # rule bodies see the whole argument block, or one simulation of a batch
            "typedef OlcSimView OlcP;" if self.L.batched else "typedef OlcRuleParams OlcP;",
            "",
            self.emit_constants(),
            self.emit_structs(),
            self.emit_support(),
            "\n".join(protos),
            "",
            "\n\n".join(helper_bodies),
            "\n\n".join(bodies),
            "",
        ])
        digest = hashlib.sha256(src.encode()).hexdigest()[:16]
        return Program(src, kernels, self.L, set(self.sink_fields), digest, iterations)

    def emit_constants(self) -> str:
        return "\n".join(f"#define {k} {v}" for k, v in sorted(self.constants.items()))

    def emit_structs(self) -> str:
        out = []
        cf = self.L.cell_fields
        out.append("struct Cell_t {\n" + "".join(f"    {ctype(ty_of_py(t))} {n};\n" for n, t in cf.items()) +
                   "    olc_u32 _rng_state;\n" + ("    olc_u32 _sim;\n" if self.L.batched else "") + "};")
        chem = self.L.chem_fields
        # voxels carry their grid coordinates (for .neighbors / .cells / .tissues)
        out.append("struct Chem_t {\n" + ("".join(f"    float {n};\n" for n in chem) or "    int _unused;\n") +
                   "    int _x, _y, _z;\n};")
        tf = self.L.tissue_fields
        out.append("struct Tissue_t {\n" +
                   ("".join(f"    {ctype(ty_of_py(t))} {n};\n" for n, t in tf.items()) or "    int _unused;\n") +
                   "    int _x, _y, _z;\n};")
        for elems in sorted(self.tuples, key=str):
            out.append(f"struct {tuple_struct_name(elems)} {{ " +
                       " ".join(f"{ctype(e)} v{i};" for i, e in enumerate(elems)) + " };")
        out.append("struct OlcCtx {\n    olc_u32 i;\n    bool dead;\n    bool born;\n    bool multi;\n"
                   "    Cell_t child;\n};")
        return "\n\n".join(out)

    def emit_support(self) -> str:
        L = self.L
        lines = []
        # load / store the cell columns
        ld, st, cp = [], [], []
        for idx, (col, fname, dt) in enumerate(L.cell_cols):
            t = "float" if dt == np.float32 else ("olc_u32" if dt == np.uint32 else "int")
            if "." in col:
                a = col.split(".")[1]
                ld.append(f"    c.{fname}.{a} = olc_col_in<{t}>(P, {idx}, i);")
                st.append(f"    olc_col_out<{t}>(P, {idx}, i, c.{fname}.{a});")
            else:
                fty = L.cell_fields.get(fname)
                if fname not in ("_rng_state", "_sim") and ty_of_py(fty) == BOOL:
                    ld.append(f"    c.{fname} = olc_col_in<int>(P, {idx}, i) != 0;")
                    st.append(f"    olc_col_out<int>(P, {idx}, i, c.{fname} ? 1 : 0);")
                else:
                    ld.append(f"    c.{fname} = olc_col_in<{t}>(P, {idx}, i);")
                    st.append(f"    olc_col_out<{t}>(P, {idx}, i, c.{fname});")
            cp.append(f"    olc_col_out<olc_u32>(P, {idx}, i, olc_col_in<olc_u32>(P, {idx}, i));")
        lines.append("__device__ __forceinline__ Cell_t olc_load_cell(const OlcP& P, olc_u32 i) {\n"
                     "    Cell_t c;\n" + "\n".join(ld) + "\n    return c;\n}")
        lines.append("__device__ __forceinline__ void olc_store_cell(const OlcP& P, olc_u32 i, "
                     "const Cell_t& c) {\n" + "\n".join(st) + "\n}")
        lines.append("__device__ __forceinline__ void olc_copy_row(const OlcP& P, olc_u32 i) {\n" +
                     "\n".join(cp) + "\n}")
        # defaults
        for kind in KINDS:
            cls = self.struct_class(kind)
            proto = cls()
            fields = (L.cell_fields if kind == "Cell" else
                      {n: T.f32 for n in L.chem_fields} if kind == "Chemistry" else L.tissue_fields)
            body = [f"    {STRUCT_NAME[kind]} c;"]
            if not fields:
                body.append("    c._unused = 0;")
            for n, t in fields.items():
                body.append(f"    c.{n} = {self.literal_of(getattr(proto, n), ty_of_py(t))};")
            if kind == "Cell":
                body.append("    c._rng_state = 0u;")
                if self.L.batched:
                    body.append("    c._sim = 0u;")
            else:
                body.append("    c._x = 0;\n    c._y = 0;\n    c._z = 0;")
            lines.append(f"__device__ __forceinline__ {STRUCT_NAME[kind]} olc_default_{kind.lower()}() {{\n" +
                         "\n".join(body) + "\n    return c;\n}")
            # copy_from keeps the receiver's private state
            assigns = "\n".join(f"    a.{n} = b.{n};" for n in fields)
            lines.append(f"__device__ __forceinline__ void olc_copy_from(" f"{STRUCT_NAME[kind]}& a, "
                         f"const {STRUCT_NAME[kind]}& b) {{\n{assigns}\n}}")
        # chemistry / tissue lookups
        chem_reads = "\n".join(f"    c.{n} = olc_field_at(P, {i}, v);"
                               for i, n in enumerate(L.chem_fields))
        lines.append("__device__ __forceinline__ Chem_t olc_chem_at(const OlcP& P, olc_vec3 p) {\n"
                     "    Chem_t c = olc_default_chemistry();\n    const olc_u32 v = olc_chem_index(P, p);\n" +
                     chem_reads + "\n    c._x = olc_bin_coord(p.x, P.cvs, P.cdims[0]);\n"
                     "    c._y = olc_bin_coord(p.y, P.cvs, P.cdims[1]);\n"
                     "    c._z = olc_bin_coord(p.z, P.cvs, P.cdims[2]);\n    return c;\n}")
        # chemistry voxel (x, y, z) as rules read it (any storage)
        lines.append("__device__ __forceinline__ Chem_t olc_chem_voxel(const OlcP& P, int x, int y, int z) {\n"
                     "    Chem_t c = olc_default_chemistry();\n"
                     "    const olc_u32 v = ((olc_u32)z * (olc_u32)P.cdims[1] + (olc_u32)y) * (olc_u32)P.cdims[0] + "
                     "(olc_u32)x;\n" + chem_reads + "\n    c._x = x;\n    c._y = y;\n    c._z = z;\n    return c;\n}")
        tis_reads = []
        for i, (n, t) in enumerate(L.tissue_fields.items()):
            ty = ty_of_py(t)
            if ty == F32:
                tis_reads.append(f"    c.{n} = olc_tissue_col<float>(P, {i}, k);")
            elif ty == BOOL:
                tis_reads.append(f"    c.{n} = olc_tissue_col<int>(P, {i}, k) != 0;")
            elif ty == U32:
                tis_reads.append(f"    c.{n} = olc_tissue_col<olc_u32>(P, {i}, k);")
            else:
                tis_reads.append(f"    c.{n} = olc_tissue_col<int>(P, {i}, k);")
        lines.append("__device__ __forceinline__ Tissue_t olc_tissue_voxel(const OlcP& P, int x, int y, int z) {\n"
                     "    Tissue_t c = olc_default_tissue();\n    c._x = x;\n    c._y = y;\n    c._z = z;\n"
                     "    if (!P.tissue) return c;\n"
                     "    const olc_u32 k = olc_tissue_key(x, y, z);\n" + "\n".join(tis_reads) +
                     "\n    return c;\n}")
        lines.append("__device__ __forceinline__ Tissue_t olc_tissue_at(const OlcP& P, olc_vec3 p) {\n"
                     "    const olc_ivec3 t = olc_tissue_coord(P, p);\n"
                     "    return olc_tissue_voxel(P, t.x, t.y, t.z);\n}")
        chem_writes = "\n".join(f"    olc_field_out(P, {i}, v, c.{n});" for i, n in enumerate(L.chem_fields))
        lines.append("__device__ __forceinline__ void olc_store_chem(const OlcP& P, olc_u32 v, "
                     "const Chem_t& c) {\n" + chem_writes + "\n}")
        if not L.batched:
            # voxel-rule stores: the other buffer of the tissue grid / of every field
            tis_writes = []
            for i, (n, t) in enumerate(L.tissue_fields.items()):
                ty = ty_of_py(t)
                if ty == F32:
                    tis_writes.append(f"    olc_tissue_col_out<float>(P, {i}, k, c.{n});")
                elif ty == BOOL:
                    tis_writes.append(f"    olc_tissue_col_out<int>(P, {i}, k, c.{n} ? 1 : 0);")
                elif ty == U32:
                    tis_writes.append(f"    olc_tissue_col_out<olc_u32>(P, {i}, k, c.{n});")
                else:
                    tis_writes.append(f"    olc_tissue_col_out<int>(P, {i}, k, c.{n});")
            lines.append("__device__ __forceinline__ void olc_store_tissue(const OlcP& P, olc_u32 k, "
                         "const Tissue_t& c) {\n" + "\n".join(tis_writes) + "\n}")
        lines.append("__device__ __forceinline__ olc_vec3 olc_rand_dir3(olc_u32& s) {\n"
                     "    float3 d = olc_rand_dir(s);\n    return olc_v3(d.x, d.y, d.z);\n}")
        lines.append("__device__ __forceinline__ void olc_divide(OlcCtx& ctx, olc_u32 rng, const Cell_t& child) {\n"
                     "    if (ctx.born) { ctx.multi = true; return; }\n    ctx.born = true;\n"
                     "    ctx.child = child;\n    ctx.child._rng_state = rng ^ OLC_CHILD_RNG_XOR;\n}")
        return "\n\n".join(lines)

    def literal_of(self, v: Any, ty) -> str:
        if ty == F32:
            return fmt_float(float(v))
        if ty == BOOL:
            return "true" if v else "false"
        if ty in (I32, U32):
            return fmt_int(int(v)) + ("u" if ty == U32 and not str(fmt_int(int(v))).endswith("u") else "")
        if ty == VEC3:
            return f"olc_v3({fmt_float(v.x)}, {fmt_float(v.y)}, {fmt_float(v.z)})"
        if ty == IVEC3:
            return f"olc_iv3({int(v.x)}, {int(v.y)}, {int(v.z)})"
        raise CompilationError(f"no literal for {v!r}")

    def prototype(self, info: FuncInfo) -> str:
        ret = ctype(info.ret) if info.ret is not None else "void"
        ps = ["const OlcP& P", "olc_u32& _rng", "OlcCtx& _ctx"]
        if info.kind in KINDS:
            ps.append(f"{STRUCT_NAME[info.kind]}& self" if info.self_by_ref
                      else f"{STRUCT_NAME[info.kind]} self")
        for name, ty, by_ref in info.params:
            ps.append(f"{ctype(ty)}& {name}" if by_ref else f"{ctype(ty)} {name}")
        return f"__device__ __noinline__ {ret} {info.cname}({', '.join(ps)})" if info.kind not in ("rule", "metric") \
            else f"__device__ __forceinline__ void {info.cname}({', '.join(ps)})"

    def emit_function(self, info: FuncInfo) -> str:
        fe = FuncEmitter(self, info)
        body = fe.run()
        return f"{self.prototype(info)} {{\n{body}\n}}"

    def cell_kernel(self, kname: str, fn: str) -> str:
        L = self.L
        if self.contact_radius is not None:
            radius = f"c.{self.contact_radius}"
        else:
            radius = "P.radius_const"
        return f"""extern "C" __global__ void __launch_bounds__(OLC_RULE_THREADS) {kname}(OlcRuleParams P) {{
    __shared__ olc_u32 s_tile, s_excl;
    __shared__ olc_u32 s_warp[OLC_RULE_THREADS / 32];
    const olc_u32 n_live = P.counters[OLC_CTR_N];
    const olc_u32 rows = olc_rule_rows(P.counters, P.rule_index);
    for (;;) {{
        if (threadIdx.x == 0) s_tile = atomicAdd(P.counters + OLC_CTR_RULE_TILE + P.rule_index, 1u);
        __syncthreads();
        const olc_u32 tile = s_tile;
        __syncthreads();
        if ((olc_u64)tile * OLC_RULE_THREADS >= rows) break;
        const olc_u32 i = tile * OLC_RULE_THREADS + threadIdx.x;
        OlcCtx ctx;
        ctx.i = i;
        ctx.dead = false;
        ctx.born = false;
        ctx.multi = false;
{self.view_decl("i < rows")}
        if (i < n_live) {{
            Cell_t c = olc_load_cell({self.pv}, i);
            olc_u32 rng = c._rng_state;
            {fn}({self.pv}, rng, ctx, c);
            c._rng_state = rng;
            olc_store_cell({self.pv}, i, c);
            const bool dead = ctx.dead || P.life[i] != 0;  // an earlier rule's die() stands
            if (ctx.dead) P.life[i] = 1;
            if (P.posr) P.posr[i] = make_float4(c.pos.x, c.pos.y, c.pos.z, dead ? -1.0f : {radius});{self.child_sim()}
        }} else if (i < rows) {{
            olc_copy_row({self.pv}, i);  // child of an earlier rule this step: carried unchanged
        }}
        const olc_u32 slot = olc_birth_slot(P, ctx.born, tile, rows, s_warp, &s_excl);
        if (ctx.born && slot < P.capacity) {{
            olc_store_cell({self.pv}, slot, ctx.child);
            P.life[slot] = 0;
        }}
        if (ctx.multi) atomicOr(P.counters + OLC_CTR_STATUS, OLC_ST_MULTI_DIVIDE);
    }}
}}"""

    @property
    def pv(self) -> str:
        """What the kernel passes to rule bodies: the argument block, or the view
        of the agent's simulation in batched mode."""
        return "V" if self.L.batched else "P"

    def view_decl(self, has_row: str) -> str:
        if not self.L.batched:
            return ""
        sim_col = len(self.L.cell_cols) - 1
        return (f"        const olc_u32 sim = ({has_row}) ? reinterpret_cast<const olc_u32*>(P.cols_in[{sim_col}])[i] "
                f": 0u;\n        const OlcSimView V = olc_sim_view(P, sim);")

    def child_sim(self) -> str:
        return "\n            ctx.child._sim = c._sim;  // a child belongs to its parent's simulation" \
            if self.L.batched else ""

    def voxel_kernel(self, kname: str, fn: str, kind: str) -> str:
        """One thread per voxel of the tissue (bin) grid or the chemistry grid:
        load the voxel from the current buffer, run the rule, store it to the
        other buffer (the host flips the buffers after the launch)."""
        if self.L.batched:
            if kind == "Tissue":
                raise CompilationError("tissue rules are not compiled in batched mode (members have no tissue grids)")
            return self.batched_chem_kernel(kname, fn)
        dims = "P.tdims" if kind == "Tissue" else "P.cdims"
        load = "olc_tissue_voxel(P, x, y, z)" if kind == "Tissue" else "olc_chem_voxel(P, x, y, z)"
        store = "olc_store_tissue(P, olc_tissue_key(x, y, z), v)" if kind == "Tissue" else "olc_store_chem(P, w, v)"
        return f"""extern "C" __global__ void __launch_bounds__(OLC_RULE_THREADS) {kname}(OlcRuleParams P) {{
    const olc_u32 nx = (olc_u32){dims}[0], ny = (olc_u32){dims}[1], nz = (olc_u32){dims}[2];
    const olc_u32 nv = nx * ny * nz;
    for (olc_u32 w = blockIdx.x * blockDim.x + threadIdx.x; w < nv; w += gridDim.x * blockDim.x) {{
        const int x = (int)(w % nx), y = (int)((w / nx) % ny), z = (int)(w / (nx * ny));
        {STRUCT_NAME[kind]} v = {load};
        olc_u32 rng = 0u;  // voxels have no RNG state
        OlcCtx ctx;
        ctx.i = 0xffffffffu;
        ctx.dead = false;
        ctx.born = false;
        ctx.multi = false;
        {fn}(P, rng, ctx, v);
        {store};
    }}
}}"""

    def batched_chem_kernel(self, kname: str, fn: str) -> str:
        """A chemistry rule over every member of a batch: one CTA per field
        tile of the batch's tile list (P.vtiles: member, tile coordinates), one
        thread per voxel of the tile, each member seen through its own view
        (grid, fields, bin table); stores go to the member's other buffer and
        the host flips every member's parity after the launch."""
        return f"""extern "C" __global__ void __launch_bounds__(OLC_RULE_THREADS) {kname}(OlcRuleParams P) {{
    const int tx = P.vtile[0], ty = P.vtile[1], tz = P.vtile[2];
    const olc_u32 per = (olc_u32)(tx * ty * tz);
    for (olc_u32 ti = blockIdx.x; ti < P.n_vtiles; ti += gridDim.x) {{
        const uint4 t = P.vtiles[ti];
        const OlcSimView V = olc_sim_view(P, t.x);
        for (olc_u32 e = threadIdx.x; e < per; e += blockDim.x) {{
            const int x = (int)t.y * tx + (int)(e % (olc_u32)tx);
            const int y = (int)t.z * ty + (int)((e / (olc_u32)tx) % (olc_u32)ty);
            const int z = (int)t.w * tz + (int)(e / (olc_u32)(tx * ty));
            if (x >= V.cdims[0] || y >= V.cdims[1] || z >= V.cdims[2]) continue;
            const olc_u32 w = ((olc_u32)z * (olc_u32)V.cdims[1] + (olc_u32)y) * (olc_u32)V.cdims[0] + (olc_u32)x;
            Chem_t v = olc_chem_voxel(V, x, y, z);
            olc_u32 rng = 0u;  // voxels have no RNG state
            OlcCtx ctx;
            ctx.i = 0xffffffffu;
            ctx.dead = false;
            ctx.born = false;
            ctx.multi = false;
            {fn}(V, rng, ctx, v);
            olc_store_chem(V, w, v);
        }}
    }}
}}"""

    def metric_kernel(self, kname: str, fn: str) -> str:
        if self.L.batched:
            clear = flush = ""
        else:
            # a solo handle's block adds its shared accumulators (cleared
            # first) to the metric words once, one thread per word
            clear = """    for (int k = threadIdx.x; k < OLC_SOLO_METRIC_WORDS; k += blockDim.x) olc_s_metrics[k] = 0u;
    __syncthreads();
"""
            adds = []
            for slot, ty in sorted(self.L.metrics.values()):
                if ty == F32:
                    add = (f"const float v = __uint_as_float(olc_s_metrics[{slot}]); "
                           f"if (v != 0.0f) atomicAdd(reinterpret_cast<float*>(P.metrics) + {slot}, v);")
                else:
                    add = (f"const olc_u32 v = olc_s_metrics[{slot}]; "
                           f"if (v != 0u) atomicAdd(reinterpret_cast<olc_u32*>(P.metrics) + {slot}, v);")
                adds.append(f"    if (threadIdx.x == {slot} % OLC_RULE_THREADS) {{ {add} }}")
            flush = "    __syncthreads();\n" + "\n".join(adds) + "\n"
        return f"""extern "C" __global__ void __launch_bounds__(OLC_RULE_THREADS) {kname}(OlcRuleParams P) {{
{clear}    const olc_u32 rows = olc_total_rows(P.counters);
    for (olc_u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {{
        if (P.life[i]) continue;
{self.view_decl("true")}
        Cell_t c = olc_load_cell({self.pv}, i);
        olc_u32 rng = c._rng_state;
        OlcCtx ctx;
        ctx.i = i;
        ctx.dead = false;
        ctx.born = false;
        ctx.multi = false;
        {fn}({self.pv}, rng, ctx, c);
    }}
{flush}}}"""


def mutated_names(node: ast.FunctionDef) -> set:
    """Names whose attributes the function assigns (x.a = .., x.a += .., x.a.b = ..)."""
    out = set()

    def root(t):
        while isinstance(t, ast.Attribute):
            t = t.value
        return t.id if isinstance(t, ast.Name) else None

    for n in ast.walk(node):
        targets = []
        if isinstance(n, ast.Assign):
            targets = n.targets
        elif isinstance(n, (ast.AugAssign, ast.AnnAssign)):
            targets = [n.target]
        for t in targets:
            if isinstance(t, ast.Attribute):
                r = root(t)
                if r:
                    out.add(r)
        if isinstance(n, ast.Call) and isinstance(n.func, ast.Attribute) and n.func.attr == "copy_from":
            r = root(n.func.value)
            if r:
                out.add(r)
    return out


# ------------------------------------------------------------------ per-function emitter

class FuncEmitter:
    def __init__(self, tr: Translator, info: FuncInfo):
        self.tr = tr
        self.info = info
        self.locals: dict[str, Any] = {}
        self.params: dict[str, Any] = {p[0]: p[1] for p in info.params}
        self.lines: list[str] = []
        self.indent = 1
        self.tmp = 0
        self.loop_labels: list[str | None] = []
        self.g = dict(getattr(info.pyfunc, "__func__", info.pyfunc).__globals__)
        sp = tr.spec
        for cls in (sp.cell_class, sp.tissue_class, sp.chemistry_class, sp.metrics_class, sp.params_class):
            self.g.setdefault(cls.__name__, cls)
        self.self_kind = info.kind if info.kind in KINDS else "sim"
        self.main = info.params[0][0] if info.kind in ("rule", "metric") else None
        self.metrics_name = getattr(info, "metrics_name", None)

    def err(self, msg: str, node: ast.AST | None) -> CompilationError:
        return CompilationError(msg, node, self.info.src, self.info.filename, self.info.line0)

    def emit(self, s: str) -> None:
        self.lines.append("    " * self.indent + s)

    def fresh(self, p: str = "_t") -> str:
        self.tmp += 1
        return f"{p}{self.tmp}"

    def run(self) -> str:
        body = strip_docstring(self.info.node.body)
        for st in body:
            self.stmt(st)
        decls = [f"    {ctype(t)} {n} = {self.zero(t)};" for n, t in self.locals.items()]
        return "\n".join(decls + self.lines)

    def zero(self, t) -> str:
        if is_struct(t):
            return f"olc_default_{t[1].lower()}()"
        if isinstance(t, tuple) and t[0] == "tuple":
            return "{}"
        return ZERO[t]

    # ---- name typing ------------------------------------------------------
    def var_type(self, name: str):
        if name in self.locals:
            return self.locals[name]
        if name in self.params:
            return self.params[name]
        return None

    def declare(self, name: str, t, node) -> None:
        if name in self.params or name in self.locals:
            return
        if name in ("self", "P", "_rng", "_ctx") or name.startswith("olc_"):
            raise self.err(f"name {name!r} is reserved", node)
        self.locals[name] = t

    def global_value(self, node: ast.AST):
        """Resolves Name/Attribute chains rooted at a module global; returns a
        sentinel when the expression is not static."""
        if isinstance(node, ast.Name):
            if self.var_type(node.id) is not None or node.id == "self":
                return _NOT_STATIC
            if node.id in self.g:
                return self.g[node.id]
            import builtins
            if hasattr(builtins, node.id):
                return getattr(builtins, node.id)
            return _NOT_STATIC
        if isinstance(node, ast.Attribute):
            base = self.global_value(node.value)
            if base is _NOT_STATIC:
                return _NOT_STATIC
            try:
                return getattr(base, node.attr)
            except AttributeError:
                raise self.err(f"{node.attr!r} not found", node)
        return _NOT_STATIC

    def constant_expr(self, v, node) -> tuple[str, Any]:
        if isinstance(v, bool):
            return ("true" if v else "false"), BOOL
        if isinstance(v, (int, np.integer)):
            return fmt_int(int(v)), I32
        if isinstance(v, (float, np.floating)):
            return fmt_float(float(v)), F32
        if isinstance(v, T.vec3):
            return f"olc_v3({fmt_float(v.x)}, {fmt_float(v.y)}, {fmt_float(v.z)})", VEC3
        raise self.err(f"global {v!r} cannot be used in a rule (numbers, bools and vec3 only)", node)

    # ---- statements -------------------------------------------------------
    def stmt(self, n: ast.stmt) -> None:
        m = getattr(self, "st_" + type(n).__name__, None)
        if m is None:
            raise self.err(f"unsupported statement {type(n).__name__}", n)
        m(n)

    def body(self, stmts) -> None:
        self.indent += 1
        for s in stmts:
            self.stmt(s)
        self.indent -= 1

    def st_Pass(self, n):
        pass

    def st_Expr(self, n: ast.Expr):
        v = n.value
        if isinstance(v, ast.Constant):
            return  # docstrings / bare literals
        if isinstance(v, ast.Call) and isinstance(v.func, ast.Attribute):
            fn = v.func
            if fn.attr == "die" and not v.args:
                self.check_main_receiver(fn.value, "die")
                self.emit("_ctx.dead = true;")
                return
            if fn.attr == "divide" and len(v.args) == 1:
                self.check_main_receiver(fn.value, "divide")
                child, ct = self.expr(v.args[0])
                if ct != ("struct", "Cell"):
                    raise self.err("divide() takes a new cell", v)
                self.emit(f"olc_divide(_ctx, _rng, {child});")
                return
            if fn.attr == "copy_from" and len(v.args) == 1:
                dst, dt = self.expr(fn.value)
                src, st_ = self.expr(v.args[0])
                if not is_struct(dt) or dt != st_:
                    raise self.err("copy_from needs two objects of the same class", v)
                self.emit(f"olc_copy_from({dst}, {src});")
                return
        code, _ = self.expr(v)
        self.emit(f"(void)({code});")

    def check_main_receiver(self, recv: ast.AST, what: str) -> None:
        ok = (isinstance(recv, ast.Name) and ((self.main is not None and recv.id == self.main) or
                                              (recv.id == "self" and self.self_kind == "Cell")))
        if not ok:
            raise self.err(f"{what}() can only be called on the rule's own cell", recv)
        if self.info.kind == "metric":
            raise self.err(f"{what}() is not allowed in a metric rule", recv)

    def st_Return(self, n: ast.Return):
        if n.value is None:
            self.emit("return;")
            return
        want = self.info.ret
        if isinstance(n.value, ast.Tuple):
            parts = [self.expr(e) for e in n.value.elts]
            elems = tuple(p[1] for p in parts)
            if want is None:
                want = ("tuple", elems)
                self.info.ret = want
                self.tr.tuples.add(elems)
            if not (isinstance(want, tuple) and want[0] == "tuple") or len(want[1]) != len(parts):
                raise self.err("returned tuple does not match the annotation", n)
            vals = ", ".join(self.cast(c, t, w, n) for (c, t), w in zip(parts, want[1]))
            self.emit(f"return {tuple_struct_name(want[1])}{{{vals}}};")
            return
        code, t = self.expr(n.value)
        if want is None:
            if self.info.kind in ("rule", "metric"):
                raise self.err("rules return nothing", n)
            self.info.ret = want = t
        self.emit(f"return {self.cast(code, t, want, n)};")

    def target_type(self, tgt: ast.AST):
        if isinstance(tgt, ast.Name):
            return self.var_type(tgt.id)
        _, t = self.expr(tgt)
        return t

    def st_Assign(self, n: ast.Assign):
        if len(n.targets) != 1:
            raise self.err("chained assignment is not supported", n)
        tgt = n.targets[0]
        if isinstance(tgt, ast.Tuple):
            code, t = self.expr(n.value)
            if not (isinstance(t, tuple) and t[0] == "tuple") or len(t[1]) != len(tgt.elts):
                raise self.err("tuple unpacking needs a call returning a tuple of the same length", n)
            tmp = self.fresh("_tu")
            self.emit(f"const {tuple_struct_name(t[1])} {tmp} = {code};")
            for i, (e, et) in enumerate(zip(tgt.elts, t[1])):
                if not isinstance(e, ast.Name):
                    raise self.err("tuple targets must be names", e)
                self.declare(e.id, et, e)
                vt = self.var_type(e.id)
                self.emit(f"{e.id} = {self.cast(f'{tmp}.v{i}', et, vt, e)};")
            return
        if isinstance(tgt, ast.Name):
            code, t = self.expr(n.value)
            if self.var_type(tgt.id) is None:
                if t == VOID:
                    raise self.err("cannot assign the result of a function returning nothing", n)
                self.declare(tgt.id, t, tgt)
            vt = self.var_type(tgt.id)
            self.emit(f"{tgt.id} = {self.cast(code, t, vt, n)};")
            return
        if isinstance(tgt, ast.Attribute):
            self.check_not_metrics(tgt)
            lhs, lt = self.expr(tgt)
            code, t = self.expr(n.value)
            self.emit(f"{lhs} = {self.cast(code, t, lt, n)};")
            return
        raise self.err("unsupported assignment target", tgt)

    def check_not_metrics(self, tgt):
        r = tgt
        while isinstance(r, ast.Attribute):
            r = r.value
        if isinstance(r, ast.Name) and self.metrics_name and r.id == self.metrics_name:
            raise self.err("metric fields only support += and -=", tgt)

    def st_AnnAssign(self, n: ast.AnnAssign):
        if not isinstance(n.target, ast.Name):
            raise self.err("annotated assignment needs a plain name", n)
        ann = self.global_value(n.annotation)
        t = ty_of_py(ann) if ann is not _NOT_STATIC else None
        if t is None:
            raise self.err("unknown annotation", n.annotation)
        self.declare(n.target.id, t, n.target)
        vt = self.var_type(n.target.id)
        if n.value is not None:
            code, et = self.expr(n.value)
            self.emit(f"{n.target.id} = {self.cast(code, et, vt, n)};")
        else:
            self.emit(f"{n.target.id} = {self.zero(vt)};")

    def st_AugAssign(self, n: ast.AugAssign):
        tgt = n.target
        op = AUGOPS.get(type(n.op))
        if op is None:
            raise self.err("unsupported augmented operator", n)
        # metrics.f += v
        if isinstance(tgt, ast.Attribute) and isinstance(tgt.value, ast.Name) and self.metrics_name and \
                tgt.value.id == self.metrics_name:
            slot_ty = self.tr.L.metrics.get(tgt.attr)
            if slot_ty is None:
                raise self.err(f"metrics has no field {tgt.attr!r}", tgt)
            slot, mt = slot_ty
            if op not in ("+", "-"):
                raise self.err("metric fields only support += and -=", n)
            code, t = self.expr(n.value)
            code = self.cast(code, t, mt if mt != BOOL else I32, n)
            if op == "-":
                code = f"-({code})"
            fn = {F32: "olc_metric_add_f", U32: "olc_metric_add_u"}.get(mt, "olc_metric_add_i")
            self.emit(f"{fn}(P, {slot}, {code});")
            return
        # self.sink_at(pos).field += rate
        if isinstance(tgt, ast.Attribute) and isinstance(tgt.value, ast.Call) and \
                isinstance(tgt.value.func, ast.Attribute) and tgt.value.func.attr == "sink_at" and \
                isinstance(tgt.value.func.value, ast.Name) and tgt.value.func.value.id == "self":
            if op != "+":
                raise self.err("sink_at(...).field only supports +=", n)
            if tgt.attr not in self.tr.L.chem_fields:
                raise self.err(f"chemistry has no field {tgt.attr!r}", tgt)
            fidx = self.tr.L.chem_fields.index(tgt.attr)
            pos, pt = self.expr(tgt.value.args[0])
            if pt != VEC3:
                raise self.err("sink_at takes a position", tgt.value)
            code, t = self.expr(n.value)
            self.tr.sink_fields.add(tgt.attr)
            self.emit(f"olc_deposit(P, {fidx}, {pos}, {self.cast(code, t, F32, n)});")
            return
        self.check_not_metrics(tgt) if isinstance(tgt, ast.Attribute) else None
        if isinstance(tgt, ast.Name) and self.var_type(tgt.id) is None:
            raise self.err(f"{tgt.id!r} used before assignment", tgt)
        lhs, lt = self.expr(tgt)
        rhs, rt = self.expr(n.value)
        val, vt = self.binop(lhs, lt, op, rhs, rt, n)
        self.emit(f"{lhs} = {self.cast(val, vt, lt, n)};")

    def st_If(self, n: ast.If):
        c = self.cond(n.test)
        self.emit(f"if ({c}) {{")
        self.body(n.body)
        if n.orelse:
            self.emit("} else {")
            self.body(n.orelse)
        self.emit("}")

    def st_While(self, n: ast.While):
        if n.orelse:
            raise self.err("while/else is not supported", n)
        c = self.cond(n.test)
        self.emit(f"while ({c}) {{")
        self.loop_labels.append(None)
        self.body(n.body)
        self.loop_labels.pop()
        self.emit("}")

    def st_Break(self, n):
        if not self.loop_labels:
            raise self.err("break outside a loop", n)
        lab = self.loop_labels[-1]
        self.emit(f"goto {lab};" if lab else "break;")

    def st_Continue(self, n):
        if not self.loop_labels:
            raise self.err("continue outside a loop", n)
        self.emit("continue;")

    def st_For(self, n: ast.For):
        if n.orelse:
            raise self.err("for/else is not supported", n)
        it = n.iter
        if isinstance(it, ast.Call) and isinstance(it.func, ast.Name) and it.func.id == "range":
            if not isinstance(n.target, ast.Name):
                raise self.err("range loop target must be a name", n.target)
            args = [self.expr(a) for a in it.args]
            for c, t in args:
                if t not in (I32, U32):
                    raise self.err("range() takes integers", it)
            if len(args) == 1:
                lo, hi, step = "0", args[0][0], "1"
            elif len(args) == 2:
                lo, hi, step = args[0][0], args[1][0], "1"
            elif len(args) == 3:
                lo, hi, step = args[0][0], args[1][0], args[2][0]
            else:
                raise self.err("range() takes 1 to 3 arguments", it)
            v = n.target.id
            self.declare(v, I32, n.target)
            hv, sv = self.fresh("_hi"), self.fresh("_st")
            self.emit(f"{{ const int {hv} = {hi}; const int {sv} = {step};")
            self.emit(f"for ({v} = {lo}; ({sv} > 0) ? ({v} < {hv}) : ({v} > {hv}); {v} += {sv}) {{")
            self.loop_labels.append(None)
            self.body(n.body)
            self.loop_labels.pop()
            self.emit("} }")
            return
        if isinstance(it, ast.Attribute) and it.attr == "neighbors":
            recv, rt = self.expr(it.value)
            if rt in (("struct", "Tissue"), ("struct", "Chemistry")):
                self.voxel_loop(n, "neighbors", recv, rt[1])
                return
            if rt != ("struct", "Cell"):
                raise self.err(".neighbors belongs to cells, tissue voxels and chemistry voxels", it)
            if not isinstance(n.target, ast.Name):
                raise self.err("loop target must be a name", n.target)
            nb = n.target.id
            if self.var_type(nb) is not None:
                raise self.err(f"loop variable {nb!r} shadows a variable", n.target)
            lab = self.fresh("_nb_done")
            bc, d = self.fresh("_bc"), self.fresh("_d")
            k, j, s, e = self.fresh("_k"), self.fresh("_j"), self.fresh("_s"), self.fresh("_e")
            self.emit("{")
            self.indent += 1
            self.emit(f"const olc_ivec3 {bc} = olc_tissue_coord(P, {recv}.pos);")
            self.emit(f"for (int {d}z = -1; {d}z <= 1; ++{d}z)")
            self.emit(f"for (int {d}y = -1; {d}y <= 1; ++{d}y)")
            self.emit(f"for (int {d}x = -1; {d}x <= 1; ++{d}x) {{")
            self.indent += 1
            self.emit(f"const int {d}nx = {bc}.x + {d}x, {d}ny = {bc}.y + {d}y, {d}nz = {bc}.z + {d}z;")
            self.emit(f"if ({d}nx < 0 || {d}ny < 0 || {d}nz < 0 || {d}nx >= P.tdims[0] || {d}ny >= P.tdims[1] "
                      f"|| {d}nz >= P.tdims[2]) continue;")
            self.emit(f"const olc_u32 {k} = olc_tissue_key({d}nx, {d}ny, {d}nz);")
            self.emit(f"const olc_u32 {s} = P.ranges[2u * {k}], {e} = P.ranges[2u * {k} + 1u];")
            self.emit(f"for (olc_u32 {j} = {s}; {j} < {e}; ++{j}) {{")
            self.indent += 1
            self.emit(f"if ({j} == _ctx.i) continue;")
            self.emit(f"const Cell_t {nb} = olc_load_cell(P, {j});")
            self.params[nb] = ("struct", "Cell")
            self.loop_labels.append(lab)
            for st in n.body:
                self.stmt(st)
            self.loop_labels.pop()
            del self.params[nb]
            self.indent -= 1
            self.emit("}")
            self.indent -= 1
            self.emit("}")
            self.indent -= 1
            self.emit(f"}} {lab}:;")
            return
        if isinstance(it, ast.Attribute) and it.attr in ("neighbors", "cells", "tissues"):
            recv, rt = self.expr(it.value)
            if rt in (("struct", "Tissue"), ("struct", "Chemistry")):
                self.voxel_loop(n, it.attr, recv, rt[1])
                return
            raise self.err(f".{it.attr} loops run over tissue or chemistry voxels (cells: .neighbors only)", it)
        raise self.err("for loops iterate over range(...), .neighbors, .cells or .tissues", n)

    def tied_geometry(self, node) -> None:
        """chem.cells / chem.tissues need the reference's tied grids: one
        chemistry voxel covers 2 x 2 x 2 tissue voxels."""
        eng = self.tr.sim._engine
        ts, cs = tuple(eng.tissue_shape), tuple(eng.chemistry_shape)
        if cs != tuple(t // 2 for t in ts) or abs(eng.chemistry_voxel_size - 2.0 * eng.tissue_voxel_size) > \
                1e-6 * eng.chemistry_voxel_size:
            raise self.err("chemistry .cells / .tissues need the chemistry grid tied to the tissue grid "
                           "(setup_geometry; chemistry voxel = 2 x 2 x 2 tissue voxels)", node)

    def voxel_loop(self, n: ast.For, attr: str, recv: str, kind: str) -> None:
        """Loops over a voxel's 26 Moore neighbours (same grid, in bounds,
        MooreOffsets order), its agents (tissue: the bin's rows in sorted
        order; chemistry: those of its 8 tissue voxels in key order) or, for
        a chemistry voxel, its 8 tissue voxels.  Loop values are copies of
        the state before the rule."""
        if not isinstance(n.target, ast.Name):
            raise self.err("loop target must be a name", n.target)
        nb = n.target.id
        if self.var_type(nb) is not None:
            raise self.err(f"loop variable {nb!r} shadows a variable", n.target)
        if attr == "tissues" and kind != "Chemistry":
            raise self.err(".tissues is a chemistry voxel's loop", n.iter)
        if attr == "tissues" and self.tr.L.batched:
            raise self.err(".tissues needs a tissue grid, which batch members do not have", n.iter)
        if attr in ("cells", "tissues") and kind == "Chemistry":
            self.tied_geometry(n.iter)
        lab = self.fresh("_vx_done")
        b, d = self.fresh("_b"), self.fresh("_d")
        self.emit("{")
        self.indent += 1
        self.emit(f"const int {b}x = {recv}._x, {b}y = {recv}._y, {b}z = {recv}._z;")
        if attr == "neighbors":
            dims = "P.tdims" if kind == "Tissue" else "P.cdims"
            self.emit(f"for (int {d}z = -1; {d}z <= 1; ++{d}z)")
            self.emit(f"for (int {d}y = -1; {d}y <= 1; ++{d}y)")
            self.emit(f"for (int {d}x = -1; {d}x <= 1; ++{d}x) {{")
            self.indent += 1
            self.emit(f"if ({d}x == 0 && {d}y == 0 && {d}z == 0) continue;")
            self.emit(f"const int {d}nx = {b}x + {d}x, {d}ny = {b}y + {d}y, {d}nz = {b}z + {d}z;")
            self.emit(f"if ({d}nx < 0 || {d}ny < 0 || {d}nz < 0 || {d}nx >= {dims}[0] || {d}ny >= {dims}[1] "
                      f"|| {d}nz >= {dims}[2]) continue;")
            load = "olc_tissue_voxel" if kind == "Tissue" else "olc_chem_voxel"
            self.emit(f"const {STRUCT_NAME[kind]} {nb} = {load}(P, {d}nx, {d}ny, {d}nz);")
            self.params[nb] = ("struct", kind)
            closes = 1
        else:
            if kind == "Tissue":
                self.emit(f"for (int {d}i = 0; {d}i < 1; ++{d}i) {{")
                self.indent += 1
                self.emit(f"const int {d}nx = {b}x, {d}ny = {b}y, {d}nz = {b}z;")
            else:
                self.emit(f"for (int {d}i = 0; {d}i < 8; ++{d}i) {{")
                self.indent += 1
                self.emit(f"const int {d}nx = 2 * {b}x + ({d}i & 1), {d}ny = 2 * {b}y + (({d}i >> 1) & 1), "
                          f"{d}nz = 2 * {b}z + (({d}i >> 2) & 1);")
                self.emit(f"if ({d}nx >= P.tdims[0] || {d}ny >= P.tdims[1] || {d}nz >= P.tdims[2]) continue;")
            if attr == "tissues":
                self.emit(f"const Tissue_t {nb} = olc_tissue_voxel(P, {d}nx, {d}ny, {d}nz);")
                self.params[nb] = ("struct", "Tissue")
                closes = 1
            else:
                k, j, s0, e0 = self.fresh("_k"), self.fresh("_j"), self.fresh("_s"), self.fresh("_e")
                self.emit(f"const olc_u32 {k} = olc_tissue_key({d}nx, {d}ny, {d}nz);")
                self.emit(f"const olc_u32 {s0} = P.ranges[2u * {k}], {e0} = P.ranges[2u * {k} + 1u];")
                self.emit(f"for (olc_u32 {j} = {s0}; {j} < {e0}; ++{j}) {{")
                self.indent += 1
                self.emit(f"const Cell_t {nb} = olc_load_cell(P, {j});")
                self.params[nb] = ("struct", "Cell")
                closes = 2
        self.loop_labels.append(lab)
        for st in n.body:
            self.stmt(st)
        self.loop_labels.pop()
        del self.params[nb]
        for _ in range(closes):
            self.indent -= 1
            self.emit("}")
        self.indent -= 1
        self.emit(f"}} {lab}:;")

    # ---- expressions -------------------------------------------------------
    def cond(self, node) -> str:
        code, t = self.expr(node)
        return self.to_bool(code, t, node)

    def to_bool(self, code, t, node) -> str:
        if t == BOOL:
            return code
        if t in (I32, U32):
            return f"(({code}) != 0)"
        if t == F32:
            return f"(({code}) != 0.0f)"
        raise self.err("condition must be a bool or number", node)

    def cast(self, code: str, src, dst, node) -> str:
        if dst is None or src == dst:
            return code
        if dst == F32 and src in (I32, U32, BOOL):
            return f"(float)({code})"
        if dst == I32 and src in (U32, BOOL):
            return f"(int)({code})"
        if dst == U32 and src in (I32, BOOL):
            return f"(olc_u32)({code})"
        if dst == BOOL and src in (I32, U32, F32):
            return self.to_bool(code, src, node)
        if dst in (I32, U32) and src == F32:
            raise self.err("implicit float -> int conversion; use int(...)", node)
        raise self.err(f"type mismatch: {src} cannot be stored as {dst}", node)

    def expr(self, n: ast.AST) -> tuple[str, Any]:
        m = getattr(self, "ex_" + type(n).__name__, None)
        if m is None:
            raise self.err(f"unsupported expression {type(n).__name__}", n)
        return m(n)

    def ex_Constant(self, n: ast.Constant):
        v = n.value
        if isinstance(v, (bool, int, float)):
            return self.constant_expr(v, n)
        raise self.err(f"unsupported constant {v!r}", n)

    def ex_Name(self, n: ast.Name):
        t = self.var_type(n.id)
        if t is not None:
            return n.id, t
        if n.id == "self":
            if self.self_kind in KINDS:
                return "self", ("struct", self.self_kind)
            raise self.err("the simulation object has no value in a rule; use self.params / self.<method>", n)
        v = self.global_value(n)
        if v is _NOT_STATIC:
            raise self.err(f"unknown name {n.id!r}", n)
        return self.constant_expr(v, n)

    def ex_Attribute(self, n: ast.Attribute):
        # self.params.X
        if isinstance(n.value, ast.Attribute) and isinstance(n.value.value, ast.Name) and \
                n.value.value.id == "self" and n.value.attr == "params" and self.self_kind == "sim":
            p = self.tr.L.params.get(n.attr)
            if p is None:
                raise self.err(f"Params has no field {n.attr!r}", n)
            off, t = p
            if t == BOOL:
                return f"(olc_param<int>(P, {off}) != 0)", BOOL
            return f"olc_param<{ctype(t)}>(P, {off})", t
        g = self.global_value(n)
        if g is not _NOT_STATIC:
            return self.constant_expr(g, n)
        base, bt = self.expr(n.value)
        if bt in (VEC3, IVEC3):
            if n.attr not in ("x", "y", "z"):
                raise self.err(f"vectors have x, y, z (not {n.attr!r})", n)
            return f"{base}.{n.attr}", (F32 if bt == VEC3 else I32)
        if is_struct(bt):
            kind = bt[1]
            if self.metrics_name and isinstance(n.value, ast.Name) and n.value.id == self.metrics_name:
                raise self.err("metric fields cannot be read in a rule", n)
            fields = self.struct_fields(kind)
            if n.attr in fields:
                return f"{base}.{n.attr}", fields[n.attr]
            if n.attr in ("coord", "neighbors", "cells", "tissues", "sim"):
                raise self.err(f".{n.attr} is not available on {kind} values in this backend", n)
            raise self.err(f"{kind} has no field {n.attr!r}", n)
        raise self.err(f"cannot read .{n.attr} of a {bt}", n)

    def struct_fields(self, kind: str) -> dict:
        L = self.tr.L
        if kind == "Cell":
            return {k: ty_of_py(v) for k, v in L.cell_fields.items()}
        if kind == "Chemistry":
            return {k: F32 for k in L.chem_fields}
        return {k: ty_of_py(v) for k, v in L.tissue_fields.items()}

    def ex_UnaryOp(self, n: ast.UnaryOp):
        if isinstance(n.op, ast.Not):
            return f"(!{self.cond(n.operand)})", BOOL
        code, t = self.expr(n.operand)
        if isinstance(n.op, ast.USub):
            if t == BOOL:
                return f"(-(int)({code}))", I32
            return f"(-{code})", t
        if isinstance(n.op, ast.UAdd):
            return code, t
        raise self.err("unsupported unary operator", n)

    def binop(self, a, at, op, b, bt, node):
        if at in (VEC3, IVEC3) or bt in (VEC3, IVEC3):
            vt = at if at in (VEC3, IVEC3) else bt
            if op not in ("+", "-", "*", "/"):
                raise self.err(f"operator {op} is not defined on vectors", node)
            if at in NUMERIC and op in ("+", "-", "/"):
                raise self.err(f"scalar {op} vector is not defined", node)
            if vt == VEC3:
                if at in NUMERIC:
                    a = self.cast(a, at, F32, node)
                if bt in NUMERIC:
                    b = self.cast(b, bt, F32, node)
            return f"({a} {op} {b})", vt
        if is_struct(at) or is_struct(bt):
            raise self.err("arithmetic on data objects is not defined", node)
        if at == BOOL:
            a, at = f"(int)({a})", I32
        if bt == BOOL:
            b, bt = f"(int)({b})", I32
        if op == "/":
            return f"({self.cast(a, at, F32, node)} / {self.cast(b, bt, F32, node)})", F32
        t = promote(at, bt)
        if op == "//":
            if t == F32:
                return f"olc_floordiv_f({self.cast(a, at, F32, node)}, {self.cast(b, bt, F32, node)})", F32
            return f"olc_floordiv_i({a}, {b})", I32
        if op == "%":
            if t == F32:
                return f"olc_mod_f({self.cast(a, at, F32, node)}, {self.cast(b, bt, F32, node)})", F32
            return f"olc_mod_i({a}, {b})", I32
        if op == "**":
            return f"powf({self.cast(a, at, F32, node)}, {self.cast(b, bt, F32, node)})", F32
        if op in ("&", "|", "^", "<<", ">>"):
            if t == F32:
                raise self.err(f"operator {op} needs integers", node)
            return f"({a} {op} {b})", t
        return f"({a} {op} {b})", t

    def ex_BinOp(self, n: ast.BinOp):
        op = BINOPS.get(type(n.op))
        if op is None:
            raise self.err("unsupported operator", n)
        a, at = self.expr(n.left)
        b, bt = self.expr(n.right)
        return self.binop(a, at, op, b, bt, n)

    def ex_BoolOp(self, n: ast.BoolOp):
        op = " && " if isinstance(n.op, ast.And) else " || "
        return "(" + op.join(self.cond(v) for v in n.values) + ")", BOOL

    def ex_Compare(self, n: ast.Compare):
        parts = []
        left, lt = self.expr(n.left)
        for op, rnode in zip(n.ops, n.comparators):
            right, rt = self.expr(rnode)
            sym = CMPOPS.get(type(op))
            if sym is None:
                raise self.err("unsupported comparison", n)
            if (lt in (VEC3, IVEC3) or rt in (VEC3, IVEC3)) and sym not in ("==", "!="):
                raise self.err("vectors only compare with == and !=", n)
            parts.append(f"({left} {sym} {right})")
            left, lt = right, rt
        return ("(" + " && ".join(parts) + ")") if len(parts) > 1 else parts[0], BOOL

    def ex_IfExp(self, n: ast.IfExp):
        c = self.cond(n.test)
        a, at = self.expr(n.body)
        b, bt = self.expr(n.orelse)
        if at != bt:
            if at in NUMERIC and bt in NUMERIC:
                t = promote(at, bt)
                a, b = self.cast(a, at, t, n), self.cast(b, bt, t, n)
                at = t
            else:
                raise self.err("both branches of a conditional expression need the same type", n)
        return f"({c} ? {a} : {b})", at

    def ex_Subscript(self, n: ast.Subscript):
        base, bt = self.expr(n.value)
        if isinstance(bt, tuple) and bt[0] == "tuple" and isinstance(n.slice, ast.Constant) and \
                isinstance(n.slice.value, int):
            i = n.slice.value
            if not 0 <= i < len(bt[1]):
                raise self.err("tuple index out of range", n)
            return f"{base}.v{i}", bt[1][i]
        raise self.err("only constant indexing of returned tuples is supported", n)

    def ex_Call(self, n: ast.Call):
        fn = n.func
        # self.<x>(...)
        if isinstance(fn, ast.Attribute) and isinstance(fn.value, ast.Name) and fn.value.id == "self":
            if self.self_kind == "sim":
                if fn.attr == "chemistry_at":
                    p, pt = self.expr(n.args[0])
                    if pt != VEC3:
                        raise self.err("chemistry_at takes a position", n)
                    return f"olc_chem_at(P, {p})", ("struct", "Chemistry")
                if fn.attr == "tissue_at":
                    p, pt = self.expr(n.args[0])
                    if pt != VEC3:
                        raise self.err("tissue_at takes a position", n)
                    return f"olc_tissue_at(P, {p})", ("struct", "Tissue")
                if fn.attr == "sink_at":
                    raise self.err("sink_at(...) is write-only: use self.sink_at(pos).field += rate", n)
                info = self.tr.sim_info(fn.attr, n)
                return self.call_helper(info, None, n)
            info = self.tr.method_info(self.self_kind, fn.attr, n)
            return self.call_helper(info, ("self", ("struct", self.self_kind)), n)
        # obj.method(...) on a data object
        if isinstance(fn, ast.Attribute):
            g = self.global_value(fn)
            if g is _NOT_STATIC:
                recv, rt = self.expr(fn.value)
                if fn.attr == "copy" and not n.args:
                    return recv, rt
                if is_struct(rt):
                    if fn.attr in ("die", "divide", "copy_from"):
                        raise self.err(f"{fn.attr}() is a statement", n)
                    info = self.tr.method_info(rt[1], fn.attr, n)
                    return self.call_helper(info, (recv, rt), n)
                raise self.err(f"cannot call .{fn.attr}() on a {rt}", n)
            return self.call_static(g, n)
        if isinstance(fn, ast.Name):
            g = self.global_value(fn)
            if g is _NOT_STATIC:
                raise self.err(f"unknown function {fn.id!r}", n)
            return self.call_static(g, n)
        raise self.err("unsupported call", n)

    def call_helper(self, info: FuncInfo, recv, n: ast.Call):
        if n.keywords:
            raise self.err("helpers take positional arguments", n)
        if len(n.args) != len(info.params):
            raise self.err(f"{info.pyfunc.__qualname__} takes {len(info.params)} arguments", n)
        args = ["P", "_rng", "_ctx"]
        if recv is not None:
            args.append(recv[0])
        for a, (pname, pt, by_ref) in zip(n.args, info.params):
            code, t = self.expr(a)
            if by_ref:
                if t != pt:
                    raise self.err(f"argument {pname!r} must be a {pt}", a)
                args.append(code)
            else:
                args.append(self.cast(code, t, pt, a))
        if info.ret is None and not self._returns_value(info):
            return f"{info.cname}({', '.join(args)})", VOID
        ret = info.ret if info.ret is not None else self._infer_ret(info)
        return f"{info.cname}({', '.join(args)})", ret

    def _returns_value(self, info: FuncInfo) -> bool:
        return any(isinstance(x, ast.Return) and x.value is not None for x in ast.walk(info.node))

    def _infer_ret(self, info: FuncInfo):
        # emit the helper now to learn its return type
        if info.ret is None:
            FuncEmitter(self.tr, info).run()
        if info.ret is None:
            raise self.err(f"cannot infer the return type of {info.pyfunc.__qualname__}; annotate it", info.node)
        return info.ret

    def call_static(self, g, n: ast.Call):
        args = [self.expr(a) for a in n.args]
        if (g is T.random or g is _pkg.random or g is T.random_dir or g is _pkg.random_dir) and \
                getattr(self.info, "voxel_rule", False):
            raise self.err("tissue and chemistry voxels have no RNG state; random() is for cell rules", n)
        if g is T.random or g is _pkg.random:
            return "olc_next_rand(_rng)", F32
        if g is T.random_dir or g is _pkg.random_dir:
            return "olc_rand_dir3(_rng)", VEC3
        if g is T.vec3:
            if len(args) == 0:
                return "olc_v3(0.0f, 0.0f, 0.0f)", VEC3
            if len(args) == 1:
                c = self.cast(args[0][0], args[0][1], F32, n)
                tmp = c
                return f"olc_v3({tmp}, {tmp}, {tmp})", VEC3
            if len(args) == 3:
                return "olc_v3(" + ", ".join(self.cast(c, t, F32, n) for c, t in args) + ")", VEC3
            raise self.err("vec3() takes 0, 1 or 3 arguments", n)
        if g is T.ivec3:
            if len(args) != 3:
                raise self.err("ivec3() takes 3 arguments", n)
            return "olc_iv3(" + ", ".join(self.cast(c, t, I32, n) for c, t in args) + ")", IVEC3
        if g in (T.f32, float):
            (c, t), = args
            return f"(float)({c})", F32
        if g in (T.i32, int):
            (c, t), = args
            return f"(int)({c})", I32
        if g is T.u32:
            (c, t), = args
            return f"(olc_u32)({c})", U32
        if g is bool:
            (c, t), = args
            return self.to_bool(c, t, n), BOOL
        if isinstance(g, type) and any(issubclass(g, getattr(T, k)) for k in KINDS):
            kind = next(k for k in KINDS if issubclass(g, getattr(T, k)))
            expected = self.tr.struct_class(kind)
            if g is not expected:
                raise self.err(f"{g.__name__} is not the model's {kind} class", n)
            if args:
                raise self.err("data classes take keyword arguments", n)
            fields = self.struct_fields(kind)
            sets = []
            for kw in n.keywords:
                if kw.arg not in fields:
                    raise self.err(f"{g.__name__} has no field {kw.arg!r}", kw)
                c, t = self.expr(kw.value)
                sets.append(f"_c.{kw.arg} = {self.cast(c, t, fields[kw.arg], kw)};")
            if not sets:
                return f"olc_default_{kind.lower()}()", ("struct", kind)
            return (f"[&]() {{ {STRUCT_NAME[kind]} _c = olc_default_{kind.lower()}(); {' '.join(sets)} "
                    f"return _c; }}()"), ("struct", kind)
        name = getattr(g, "__name__", None)
        if getattr(g, "__module__", "") == olmath.__name__ or g in (abs, min, max, round):
            return self.math_call(name, args, n)
        raise self.err(f"function {name or g!r} cannot be called in a rule", n)

    def math_call(self, name, args, n):
        ts = [t for _, t in args]
        cs = [c for c, _ in args]

        def f(i):
            return self.cast(cs[i], ts[i], F32, n)

        def need(k):
            if len(args) != k:
                raise self.err(f"{name}() takes {k} arguments", n)

        if name in UNARY_F:
            need(1)
            return f"{UNARY_F[name]}({f(0)})", F32
        if name == "inverse_sqrt":
            need(1)
            return f"(1.0f / sqrtf({f(0)}))", F32
        if name in ("pow", "atan2"):
            need(2)
            return f"{name}f({f(0)}, {f(1)})", F32
        if name in ("abs", "fabs"):
            need(1)
            if ts[0] in (I32, U32) and name == "abs":
                return f"abs({cs[0]})", ts[0]
            return f"fabsf({f(0)})", F32
        if name in ("min", "max"):
            need(2)
            if ts[0] in (I32, U32) and ts[1] in (I32, U32):
                return f"{name}({cs[0]}, {cs[1]})", promote(ts[0], ts[1])
            return f"f{name}f({f(0)}, {f(1)})", F32
        if name == "clamp":
            need(3)
            if ts[0] == VEC3:
                return f"olc_clampv({cs[0]}, {cs[1]}, {cs[2]})", VEC3
            if all(t in (I32, U32) for t in ts):
                return f"olc_clampi({cs[0]}, {cs[1]}, {cs[2]})", I32
            return f"olc_clampf({f(0)}, {f(1)}, {f(2)})", F32
        if name == "sign":
            need(1)
            if ts[0] in (I32, U32):
                return f"olc_signi({cs[0]})", I32
            return f"olc_sign({f(0)})", F32
        if name == "lerp":
            need(3)
            return f"olc_lerp({f(0)}, {f(1)}, {f(2)})", F32
        if name == "smoothstep":
            need(3)
            return f"olc_smoothstep({f(0)}, {f(1)}, {f(2)})", F32
        if name == "step":
            need(2)
            return f"olc_step_fn({f(0)}, {f(1)})", F32
        if name == "fract":
            need(1)
            return f"olc_fract({f(0)})", F32
        vec_fns = {"length": (1, F32), "length_sq": (1, F32), "normalize": (1, VEC3), "dot": (2, F32),
                   "cross": (2, VEC3), "reflect": (2, VEC3), "distance": (2, F32), "distance_sq": (2, F32)}
        if name in vec_fns:
            k, rt = vec_fns[name]
            need(k)
            if any(t != VEC3 for t in ts):
                raise self.err(f"{name}() takes vec3 arguments", n)
            return f"olc_{name}({', '.join(cs)})", rt
        if name == "lerp_vec":
            need(3)
            return f"olc_lerp_vec({cs[0]}, {cs[1]}, {f(2)})", VEC3
        raise self.err(f"ol.math.{name} is not supported", n)


class _NotStatic:
    pass


_NOT_STATIC = _NotStatic()

UNARY_F = {"sqrt": "sqrtf", "exp": "expf", "exp2": "exp2f", "log": "logf", "log2": "log2f", "sin": "sinf",
           "cos": "cosf", "tan": "tanf", "asin": "asinf", "acos": "acosf", "atan": "atanf", "sinh": "sinhf",
           "cosh": "coshf", "tanh": "tanhf", "floor": "floorf", "ceil": "ceilf", "round": "rintf",
           "trunc": "truncf"}
BINOPS = {ast.Add: "+", ast.Sub: "-", ast.Mult: "*", ast.Div: "/", ast.FloorDiv: "//", ast.Mod: "%", ast.Pow: "**",
          ast.BitAnd: "&", ast.BitOr: "|", ast.BitXor: "^", ast.LShift: "<<", ast.RShift: ">>"}
AUGOPS = {ast.Add: "+", ast.Sub: "-", ast.Mult: "*", ast.Div: "/", ast.FloorDiv: "//", ast.Mod: "%"}
CMPOPS = {ast.Eq: "==", ast.NotEq: "!=", ast.Lt: "<", ast.LtE: "<=", ast.Gt: ">", ast.GtE: ">="}


def translate_model(sim: Any, layout: ModelLayout, contact_radius: str | None) -> Program:
    """Translates every cell and metric rule of ``sim`` (whose engine holds the
    discovered rule lists) into one CUDA C translation unit."""
    tr = Translator(sim, layout, contact_radius)
    return tr.build()
