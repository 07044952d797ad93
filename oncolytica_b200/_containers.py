"""Host containers with the reference API (framework/src/oncolytica/core/utils/_containers.py)
backed by columns (structure of arrays) instead of one Python object per item.

* ``Grid``: voxel grid.  ``grid[i, j, k]`` / ``grid.sample(i, j, k)`` return a
  view whose attributes read and write the column arrays; iteration is in the
  reference's row-major (x, y, z) order.  Columns are numpy arrays of shape
  (X, Y, Z) in Fortran order, so their memory is x-fastest, the layout of the
  device fields.
* ``AgentList``: agents as Python objects (``add``) or as columns
  (``add_arrays``); ``_data`` materialises objects on demand.
"""
from __future__ import annotations

from typing import Any, Iterator

import numpy as np

from oncolytica_b200._types import PRIMITIVE_TYPES, F32, coerce, data_fields, ivec3, vec3

_NP = {"f32": np.float32, "float": np.float32, "i32": np.int32, "int": np.int32, "u32": np.uint32,
       "bool": np.int32}


def np_dtype(t: Any) -> Any:
    name = getattr(t, "__name__", str(t))
    if t is bool or name == "bool":
        return np.int32
    return _NP.get(name, np.float32)


def column_names(fields: dict[str, Any]) -> list[tuple[str, str, Any]]:
    """(column name, field name, component dtype) with vec3/ivec3 split per axis."""
    cols = []
    for name, t in fields.items():
        if t is vec3:
            cols += [(f"{name}.{a}", name, np.float32) for a in "xyz"]
        elif t is ivec3:
            cols += [(f"{name}.{a}", name, np.int32) for a in "xyz"]
        else:
            cols.append((name, name, np_dtype(t)))
    return cols


class VoxelView:
    """One voxel of a Grid; attribute access reads/writes the grid's columns."""

    __slots__ = ("_grid", "_idx")

    def __init__(self, grid: "Grid", idx: tuple[int, int, int]) -> None:
        object.__setattr__(self, "_grid", grid)
        object.__setattr__(self, "_idx", idx)

    @property
    def coord(self) -> ivec3:
        return ivec3(*self._idx)

    def __getattr__(self, name: str) -> Any:
        g = object.__getattribute__(self, "_grid")
        t = g._fields.get(name)
        if t is None:
            raise AttributeError(name)
        i = object.__getattribute__(self, "_idx")
        if t is vec3:
            return vec3(*(g._cols[f"{name}.{a}"][i] for a in "xyz"))
        if t is ivec3:
            return ivec3(*(int(g._cols[f"{name}.{a}"][i]) for a in "xyz"))
        v = g._cols[name][i]
        if v.dtype == np.float32:
            return F32(v)
        if t is bool:
            return bool(v)
        return int(v)

    def __setattr__(self, name: str, value: Any) -> None:
        g = self._grid
        t = g._fields.get(name)
        if t is None:
            raise AttributeError(f"{g._struct_class.__name__} has no field {name!r}")
        i = self._idx
        if t in (vec3, ivec3):
            value = coerce(t, value)
            for a in "xyz":
                g._cols[f"{name}.{a}"][i] = getattr(value, a)
        else:
            g._cols[name][i] = coerce(t, value)

    def __repr__(self) -> str:
        g = self._grid
        body = ", ".join(f"{k}={getattr(self, k)!r}" for k in g._fields)
        return f"{g._struct_class.__name__}@{self._idx}({body})"


class Grid:
    """Voxel grid of a Tissue or Chemistry class (reference _containers.py:17-84)."""

    def __init__(self, struct_class: type, shape: tuple[int, ...], engine: Any) -> None:
        self._struct_class = struct_class
        self._engine = engine
        self._shape = tuple(int(s) for s in shape)
        self._fields = {k: v for k, v in data_fields(struct_class).items() if v in PRIMITIVE_TYPES}
        proto = struct_class()
        self._cols: dict[str, np.ndarray] = {}
        for col, fname, dt in column_names(self._fields):
            default = getattr(proto, fname)
            if isinstance(default, (vec3, ivec3)):
                default = getattr(default, col.split(".")[1])
            self._cols[col] = np.full(self._shape, default, dtype=dt, order="F")

    @property
    def shape(self) -> tuple:
        return self._shape

    def column(self, name: str) -> np.ndarray:
        """The (X, Y, Z) array behind a scalar field or a vector component ("pos.x")."""
        return self._cols[name]

    def field(self, name: str) -> np.ndarray:
        return self._cols[name]

    def __getitem__(self, index) -> VoxelView:
        return VoxelView(self, tuple(int(i) for i in index))

    def sample(self, x: int, y: int, z: int) -> VoxelView:
        return VoxelView(self, (int(x), int(y), int(z)))

    def __iter__(self) -> Iterator[VoxelView]:
        for idx in np.ndindex(*self._shape):
            yield VoxelView(self, idx)

    def __len__(self) -> int:
        return int(np.prod(self._shape))

    def __repr__(self) -> str:
        return f"Field(struct={self._struct_class.__name__!r}, shape={self._shape})"


class AgentList:
    """Agents (reference _containers.py:87-123)."""

    def __init__(self, engine: Any) -> None:
        self._engine = engine
        self._objs: list | None = []
        self._cols: dict[str, np.ndarray] | None = None
        self._cls: type | None = None

    # ---- object view (reference API) ------------------------------------
    @property
    def _data(self) -> list:
        if self._objs is None:
            self._objs = self._materialise()
            self._cols = None
        return self._objs

    @_data.setter
    def _data(self, value: list) -> None:
        self._objs = list(value)
        self._cols = None

    def __iter__(self) -> Iterator[Any]:
        return iter(self._data)

    def __len__(self) -> int:
        if self._objs is None and self._cols is not None:
            return len(next(iter(self._cols.values()))) if self._cols else 0
        return len(self._objs or [])

    def add(self, agent: Any) -> None:
        self._remember_class(type(agent))
        self._data.append(agent)

    def _remove_dead(self) -> int:  # reference API; dead agents are removed on the device
        return 0

    # ---- column view -----------------------------------------------------
    def add_arrays(self, cell_class: type | None = None, **columns: Any) -> None:
        """Appends agents given as columns: ``pos=(N,3)`` array or ``pos.x=...``,
        other fields by name; missing fields take the class defaults."""
        cls = cell_class or self._cls or self._default_class()
        self._remember_class(cls)
        fields = data_fields(cls)
        n = None
        for v in columns.values():
            n = len(v)
            break
        if n is None:
            return
        proto = cls()
        new: dict[str, np.ndarray] = {}
        for col, fname, dt in column_names(fields):
            if col in columns:
                new[col] = np.asarray(columns[col], dtype=dt)
            elif fname in columns and fields[fname] in (vec3, ivec3):
                new[col] = np.asarray(columns[fname], dtype=dt)[:, "xyz".index(col[-1])]
            elif fname in columns:
                new[col] = np.asarray(columns[fname], dtype=dt)
            else:
                d = getattr(proto, fname)
                if isinstance(d, (vec3, ivec3)):
                    d = getattr(d, col[-1])
                new[col] = np.full(n, d, dtype=dt)
        new["_rng_state"] = np.asarray(columns.get("_rng_state", np.zeros(n)), dtype=np.uint32)
        cur = self.columns(cls)
        self._cols = {k: np.concatenate([cur[k], new[k]]) for k in new}
        self._objs = None

    def columns(self, cls: type | None = None) -> dict[str, np.ndarray]:
        """All agents as columns (materialised from objects when needed)."""
        cls = cls or self._cls or self._default_class()
        if self._objs is None and self._cols is not None:
            return self._cols
        fields = data_fields(cls)
        objs = self._objs or []
        out: dict[str, np.ndarray] = {}
        for col, fname, dt in column_names(fields):
            if "." in col:
                a = col[-1]
                out[col] = np.array([getattr(getattr(o, fname), a) for o in objs], dtype=dt)
            else:
                out[col] = np.array([getattr(o, fname) for o in objs], dtype=dt)
        out["_rng_state"] = np.array([getattr(o, "_rng_state", 0) for o in objs], dtype=np.uint32)
        return out

    def _set_columns(self, cols: dict[str, np.ndarray], cls: type) -> None:
        self._remember_class(cls)
        self._cols = cols
        self._objs = None

    def _materialise(self) -> list:
        if not self._cols:
            return []
        cls = self._cls or self._default_class()
        fields = data_fields(cls)
        n = len(next(iter(self._cols.values())))
        out = []
        for i in range(n):
            kw = {}
            for fname, t in fields.items():
                if t in (vec3, ivec3):
                    kw[fname] = t(*(self._cols[f"{fname}.{a}"][i] for a in "xyz"))
                elif fname in self._cols:
                    kw[fname] = self._cols[fname][i].item()
            obj = cls(**kw)
            object.__setattr__(obj, "_rng_state", int(self._cols["_rng_state"][i]))
            out.append(obj)
        return out

    def _remember_class(self, cls: type) -> None:
        if self._cls is None:
            self._cls = cls

    def _default_class(self) -> type:
        eng = self._engine
        sim = getattr(eng, "_sim", None)
        if sim is not None:
            return sim._spec.cell_class
        if self._cls is not None:
            return self._cls
        raise RuntimeError("AgentList: cell class unknown; add an agent object or pass cell_class")
