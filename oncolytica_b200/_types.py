"""DSL value types and model base classes, API-compatible with the reference's
``oncolytica`` package (framework/src/oncolytica/core/utils/_types.py).

Differences from the reference, all deliberate:
  * ``f32`` values are numpy float32 and ``vec3`` holds float32 components, so
    host-side arithmetic rounds like the CUDA rule kernels (the reference uses
    Python doubles on its CPU path and f32 on its GPU path).
  * Rules never run in Python in this package: ``die``/``divide``/``neighbors``
    and ``random`` only work under a rule interpreter that installs a hook
    (the test oracle does); otherwise they raise.
"""
from __future__ import annotations

import builtins as _builtins
import contextvars
import dataclasses
import math as _math
import random as _pyrandom
import sys as _sys
from dataclasses import dataclass
from types import SimpleNamespace
from typing import Annotated, Any, Generic, NewType, TypeVar, get_args, get_origin, get_type_hints

import numpy as np

S = TypeVar("S", bound="Simulation")
T = TypeVar("T", bound="Tissue")
C = TypeVar("C", bound="Chemistry")
A = TypeVar("A", bound="Cell")
M = TypeVar("M", bound="Metrics")
P = TypeVar("P", bound="Params")
U = TypeVar("U")

i32 = NewType("i32", int)
u32 = NewType("u32", int)
f32 = NewType("f32", float)
bool = _builtins.bool  # noqa: A001  (the DSL spells booleans ol.bool)

F32 = np.float32


def _f(v: Any) -> np.float32:
    return np.float32(v)


# ------------------------------------------------------------------ vectors

class vec3:
    """3-component float32 vector (reference _types.py:48-127)."""

    __slots__ = ("x", "y", "z")

    def __init__(self, x: float = 0.0, y: float | None = None, z: float | None = None) -> None:
        if y is None and z is None:
            y = z = x  # vec3(s) broadcasts, as WGSL's vec3<f32>(s)
        object.__setattr__(self, "x", _f(x))
        object.__setattr__(self, "y", _f(y if y is not None else 0.0))
        object.__setattr__(self, "z", _f(z if z is not None else 0.0))

    def __setattr__(self, name: str, value: Any) -> None:
        if name in self.__slots__:
            object.__setattr__(self, name, _f(value))
        else:
            raise AttributeError(f"'vec3' object has no attribute '{name}'")

    def __class_getitem__(cls, _dtype: Any) -> type:
        return cls

    def copy(self) -> "vec3":
        return vec3(self.x, self.y, self.z)

    def __add__(self, o: Any) -> "vec3":
        if not isinstance(o, vec3):
            return NotImplemented
        return vec3(self.x + o.x, self.y + o.y, self.z + o.z)

    __radd__ = __add__

    def __sub__(self, o: Any) -> "vec3":
        if not isinstance(o, vec3):
            return NotImplemented
        return vec3(self.x - o.x, self.y - o.y, self.z - o.z)

    def __mul__(self, o: Any) -> "vec3":
        if isinstance(o, vec3):
            return vec3(self.x * o.x, self.y * o.y, self.z * o.z)
        if isinstance(o, (float, int, np.floating, np.integer)):
            s = _f(o)
            return vec3(self.x * s, self.y * s, self.z * s)
        return NotImplemented

    def __rmul__(self, o: Any) -> "vec3":
        if isinstance(o, (float, int, np.floating, np.integer)):
            s = _f(o)
            return vec3(s * self.x, s * self.y, s * self.z)
        return NotImplemented

    def __truediv__(self, o: Any) -> "vec3":
        if isinstance(o, (float, int, np.floating, np.integer)):
            s = _f(o)
            return vec3(self.x / s, self.y / s, self.z / s)
        return NotImplemented

    def __neg__(self) -> "vec3":
        return vec3(-self.x, -self.y, -self.z)

    def __eq__(self, o: object) -> _builtins.bool:
        return isinstance(o, vec3) and self.x == o.x and self.y == o.y and self.z == o.z

    def __hash__(self) -> int:
        return hash((float(self.x), float(self.y), float(self.z)))

    def __repr__(self) -> str:
        return f"vec3({float(self.x):.4f}f, {float(self.y):.4f}f, {float(self.z):.4f}f)"


class ivec3:
    """3-component int32 vector (reference _types.py:131-202)."""

    __slots__ = ("x", "y", "z")

    def __init__(self, x: int = 0, y: int = 0, z: int = 0) -> None:
        object.__setattr__(self, "x", int(x))
        object.__setattr__(self, "y", int(y))
        object.__setattr__(self, "z", int(z))

    def __setattr__(self, name: str, value: Any) -> None:
        if name in self.__slots__:
            object.__setattr__(self, name, int(value))
        else:
            raise AttributeError(f"'ivec3' object has no attribute '{name}'")

    def __class_getitem__(cls, _dtype: Any) -> type:
        return cls

    def __iter__(self):
        yield self.x
        yield self.y
        yield self.z

    def copy(self) -> "ivec3":
        return ivec3(self.x, self.y, self.z)

    def __add__(self, o: Any) -> "ivec3":
        if not isinstance(o, ivec3):
            return NotImplemented
        return ivec3(self.x + o.x, self.y + o.y, self.z + o.z)

    __radd__ = __add__

    def __sub__(self, o: Any) -> "ivec3":
        if not isinstance(o, ivec3):
            return NotImplemented
        return ivec3(self.x - o.x, self.y - o.y, self.z - o.z)

    def __mul__(self, o: Any):
        if isinstance(o, ivec3):
            return ivec3(self.x * o.x, self.y * o.y, self.z * o.z)
        if isinstance(o, (int, np.integer)):
            return ivec3(self.x * o, self.y * o, self.z * o)
        if isinstance(o, (float, np.floating)):
            return vec3(self.x * _f(o), self.y * _f(o), self.z * _f(o))
        return NotImplemented

    __rmul__ = __mul__

    def __neg__(self) -> "ivec3":
        return ivec3(-self.x, -self.y, -self.z)

    def __eq__(self, o: object) -> _builtins.bool:
        return isinstance(o, ivec3) and self.x == o.x and self.y == o.y and self.z == o.z

    def __hash__(self) -> int:
        return hash((self.x, self.y, self.z))

    def __repr__(self) -> str:
        return f"ivec3({self.x:d}, {self.y:d}, {self.z:d})"


_FLOAT_TYPES = {_builtins.float, f32}
_INT_TYPES = {_builtins.int, i32, u32}
_BOOL_TYPES = {_builtins.bool}
_VEC_TYPES = {vec3, ivec3}
PRIMITIVE_TYPES = _FLOAT_TYPES | _INT_TYPES | _BOOL_TYPES | _VEC_TYPES


def zero_of(t: Any) -> Any:
    if t in _FLOAT_TYPES:
        return F32(0.0)
    if t in _INT_TYPES:
        return 0
    if t in _BOOL_TYPES:
        return False
    if t is vec3:
        return vec3()
    if t is ivec3:
        return ivec3()
    return None


def coerce(t: Any, v: Any) -> Any:
    """Stores a value with its declared DSL type (f32 -> float32, vec3 -> copy)."""
    if t in _FLOAT_TYPES:
        return _f(v)
    if t in _BOOL_TYPES:
        return _builtins.bool(v)
    if t in _INT_TYPES:
        return int(v)
    if t is vec3:
        return v.copy() if isinstance(v, vec3) else vec3(*v)
    if t is ivec3:
        return v.copy() if isinstance(v, ivec3) else ivec3(*v)
    return v


def _resolve_own_hints(cls: type) -> dict:
    own = cls.__dict__.get("__annotations__", {})
    if not own:
        return {}
    module = _sys.modules.get(cls.__module__)
    g = vars(module) if module is not None else {}
    out = {}
    for name, t in own.items():
        if isinstance(t, str):
            try:
                out[name] = eval(t, g)  # noqa: S307 - annotation strings of the user's own module
            except Exception:
                out[name] = t
        else:
            out[name] = t
    return out


def data_fields(cls: type) -> dict[str, Any]:
    """User-visible data fields of a model class (declaration order, no _private)."""
    hints = get_type_hints(cls, include_extras=False)
    return {k: v for k, v in hints.items() if not k.startswith("_")}


# ------------------------------------------------------------------ rule hooks

class RuleHooks:
    """What a rule interpreter provides to code running a rule on the host."""

    def random(self) -> float:  # pragma: no cover - interface
        raise NotImplementedError

    def random_dir(self) -> vec3:  # pragma: no cover - interface
        raise NotImplementedError

    def die(self, cell: Any) -> None:  # pragma: no cover - interface
        raise NotImplementedError

    def divide(self, cell: Any, child: Any) -> None:  # pragma: no cover - interface
        raise NotImplementedError

    def neighbors(self, cell: Any):  # pragma: no cover - interface
        raise NotImplementedError

    def chemistry_at(self, pos: vec3) -> Any:  # pragma: no cover - interface
        raise NotImplementedError

    def tissue_at(self, pos: vec3) -> Any:  # pragma: no cover - interface
        raise NotImplementedError

    def sink_at(self, pos: vec3) -> Any:  # pragma: no cover - interface
        raise NotImplementedError

    def voxel_neighbors(self, voxel: Any):  # pragma: no cover - interface
        raise NotImplementedError

    def voxel_cells(self, voxel: Any):  # pragma: no cover - interface
        raise NotImplementedError

    def voxel_tissues(self, voxel: Any):  # pragma: no cover - interface
        raise NotImplementedError


_hooks: contextvars.ContextVar[RuleHooks | None] = contextvars.ContextVar("oncolytica_b200_rule_hooks",
                                                                         default=None)


def install_rule_hooks(h: RuleHooks | None):
    return _hooks.set(h)


def reset_rule_hooks(token) -> None:
    _hooks.reset(token)


def _need_hooks(what: str) -> RuleHooks:
    h = _hooks.get()
    if h is None:
        raise RuntimeError(f"{what} is only meaningful inside a rule; rules run on the GPU in oncolytica_b200")
    return h


def random() -> float:
    """ol.random(): on the GPU the agent's xorshift32 stream (template.wgsl:75-82).
    Outside a rule it is Python's random() (reference _types.py:703-704)."""
    h = _hooks.get()
    if h is None:
        return _pyrandom.random()
    return h.random()


def random_dir() -> vec3:
    h = _hooks.get()
    if h is None:
        phi = _pyrandom.random() * _math.tau
        z = _pyrandom.random() * 2.0 - 1.0
        r = _math.sqrt(max(0.0, 1.0 - z * z))
        return vec3(r * _math.cos(phi), r * _math.sin(phi), z)
    return h.random_dir()


# ------------------------------------------------------------------ model classes

class Simulation(Generic[T, C, A, M, P]):
    """Base class of a user model (reference _types.py:240-363).

    ``class MySim(ol.Simulation[MyTissue, MyChem, MyCell, MyMetrics, MyParams])``
    """

    _engine: Any = None

    def __init__(self) -> None:
        self._params = self._spec.params_class()
        self._metrics = self._spec.metrics_class(self)
        self._params._validate()

    def __init_subclass__(cls, **kwargs: Any) -> None:
        super().__init_subclass__(**kwargs)
        generic = None
        for base in getattr(cls, "__orig_bases__", []):
            if get_origin(base) is Simulation:
                generic = base
                break
        if generic is None:
            raise RuntimeError(
                "Explicit type specialization is required for Simulation class.\n"
                "Usage: class MySimulation(ol.Simulation[MyTissue, MyChem, MyCell, MyMetrics, MyParams]):")
        args = get_args(generic)
        cls._spec = SimpleNamespace(tissue_class=args[0], chemistry_class=args[1], cell_class=args[2],
                                    metrics_class=args[3], params_class=args[4])
        for i, actual in enumerate(args):
            base = BASE_CLASSES[i]
            if isinstance(actual, str) or not isinstance(actual, type):
                raise TypeError(f"Parameter {i + 1} of ol.Simulation is a forward reference ({actual!r}); define "
                                f"the data classes before the Simulation class.")
            if not issubclass(actual, base):
                raise TypeError(f"Validation failed for parameter {i + 1} in ol.Simulation.\n"
                                f"The type '{actual.__name__}' must be a subclass of 'ol.{base.__name__}'.")
            if len([b for b in BASE_CLASSES if issubclass(actual, b)]) > 1:
                raise TypeError(f"The type '{actual.__name__}' must subclass exactly one of the ol base classes.")
            if base is Cell:
                hints = get_type_hints(actual)
                if hints.get("pos") is not vec3:
                    raise TypeError(f"Class '{actual.__name__}' must have attribute 'pos: ol.vec3'.")

    @property
    def params(self) -> Any:
        return self._params

    @property
    def engine(self) -> Any:
        return self._engine

    def tissue_at(self, pos: vec3) -> Any:
        """Tissue voxel at floor(pos / tissue_voxel_size), clamped (reference _types.py:314-329)."""
        return _need_hooks("tissue_at").tissue_at(pos)

    def chemistry_at(self, pos: vec3) -> Any:
        """Chemistry voxel at floor(pos / chemistry_voxel_size), clamped (reference _types.py:331-346)."""
        return _need_hooks("chemistry_at").chemistry_at(pos)

    def sink_at(self, pos: vec3) -> Any:
        """Write-only accumulator of first-order uptake rates at the chemistry voxel
        of ``pos``: ``self.sink_at(p).o2 += k`` adds k to the sink of field o2.
        The field step then applies f <- f / (1 + K dt) (engine
        tumor_sim.wgsl:387-412).  No counterpart in the reference DSL."""
        return _need_hooks("sink_at").sink_at(pos)

    def __setattr__(self, name: str, value: object) -> None:
        super().__setattr__(name, value)
        if name == "params":
            if not isinstance(value, self._spec.params_class):
                raise TypeError(f"Invalid type for 'params': expected '{self._spec.params_class.__name__}', "
                                f"got '{type(value).__name__}'.")
            value._validate()

    def __repr__(self) -> str:
        return f"{self.__class__.__name__}()"


class BaseData(Generic[U]):
    """Common base of Tissue / Chemistry / Cell (reference _types.py:368-421)."""

    _rng_state: u32

    def __init_subclass__(cls, **kwargs: Any) -> None:
        super().__init_subclass__(**kwargs)
        hints = get_type_hints(cls)
        defaults = {n: getattr(cls, n) for n in hints if n in _class_dicts(cls)}
        fields = {k: v for k, v in hints.items() if not k.startswith("_")}
        cls._ol_fields = fields

        def __init__(self, **kw: Any) -> None:
            for name in kw:
                if name not in hints:
                    raise TypeError(f"{cls.__name__} has no field {name!r}")
            for name, t in fields.items():
                if name in kw:
                    v = kw[name]
                elif name in defaults:
                    v = defaults[name]
                else:
                    v = zero_of(t)
                object.__setattr__(self, name, coerce(t, v) if t in PRIMITIVE_TYPES else v)
            object.__setattr__(self, "_rng_state", int(kw.get("_rng_state", 0)))

        cls.__init__ = __init__

    def __setattr__(self, name: str, value: Any) -> None:
        t = type(self).__dict__.get("_ol_fields", None) or getattr(type(self), "_ol_fields", {})
        if name in t and t[name] in PRIMITIVE_TYPES:
            value = coerce(t[name], value)
        object.__setattr__(self, name, value)

    def copy(self) -> Any:
        new = object.__new__(type(self))
        for k, v in self.__dict__.items():
            object.__setattr__(new, k, v.copy() if isinstance(v, (vec3, ivec3)) else v)
        return new

    def copy_from(self, other: Any) -> None:
        for name in getattr(type(self), "_ol_fields", {}):
            v = getattr(other, name)
            setattr(self, name, v.copy() if isinstance(v, (vec3, ivec3)) else v)

    def __repr__(self) -> str:
        f = getattr(type(self), "_ol_fields", {})
        body = ", ".join(f"{k}={getattr(self, k, None)!r}" for k in f)
        return f"{type(self).__name__}({body})"


def _class_dicts(cls: type) -> set[str]:
    names: set[str] = set()
    for k in cls.__mro__:
        if k in (object, Generic):
            continue
        names.update(k.__dict__.keys())
    return names


class Tissue(BaseData, Generic[S, T, C, A, M, P]):
    """Tissue voxel (reference _types.py:456-483)."""

    @property
    def neighbors(self):
        """The 26 Moore-neighbour tissue voxels inside the grid."""
        return _need_hooks("neighbors").voxel_neighbors(self)

    @property
    def cells(self):
        """The agents in this voxel (its bin of the spatial sort)."""
        return _need_hooks("cells").voxel_cells(self)


class Chemistry(BaseData, Generic[S, T, C, A, M, P]):
    """Chemistry voxel (reference _types.py:486-530)."""

    @property
    def neighbors(self):
        """The 26 Moore-neighbour chemistry voxels inside the grid."""
        return _need_hooks("neighbors").voxel_neighbors(self)

    @property
    def tissues(self):
        """The 2 x 2 x 2 tissue voxels this chemistry voxel covers."""
        return _need_hooks("tissues").voxel_tissues(self)

    @property
    def cells(self):
        """The agents of those tissue voxels."""
        return _need_hooks("cells").voxel_cells(self)


class Cell(BaseData, Generic[S, T, C, A, M, P]):
    """Agent (reference _types.py:533-579)."""

    @property
    def neighbors(self):
        """Agents in the 27 bins around this agent's bin, self excluded."""
        return _need_hooks("neighbors").neighbors(self)

    def divide(self, cell: Any) -> None:
        """Appends ``cell`` as a child of this agent at the end of the step."""
        _need_hooks("divide").divide(self, cell)

    def die(self) -> None:
        """Removes this agent at the next sort."""
        _need_hooks("die").die(self)


class Metrics(Generic[S, T, C, A, M, P]):
    """Per-step accumulators written by @metric_rule (reference _types.py:583-633)."""

    total_alive: int

    def __init__(self, sim: Any = None) -> None:
        object.__setattr__(self, "_sim", sim)
        for name, t in metric_fields(type(self)).items():
            object.__setattr__(self, name, zero_of(t))

    def __init_subclass__(cls, **kwargs: Any) -> None:
        super().__init_subclass__(**kwargs)
        for name, t in _resolve_own_hints(cls).items():
            if name.startswith("_") or name in cls.__dict__:
                continue
            setattr(cls, name, zero_of(t))

    @property
    def sim(self) -> Any:
        return self._sim

    def _clear(self) -> None:
        for name, t in metric_fields(type(self)).items():
            object.__setattr__(self, name, zero_of(t))

    def __repr__(self) -> str:
        body = ", ".join(f"{k}={getattr(self, k)!r}" for k in metric_fields(type(self)))
        return f"{type(self).__name__}({body})"


def metric_fields(cls: type) -> dict[str, Any]:
    """Accumulator fields of a Metrics class (declaration order, inherited first)."""
    return {k: v for k, v in get_type_hints(cls).items() if not k.startswith("_")}


_PARAM_HINTS: dict = {}


def _param_hints(cls: type) -> dict:
    """get_type_hints of a Params class, resolved once per class (resolving
    string annotations costs tens of microseconds, and update_params
    validates every field on every call)."""
    h = _PARAM_HINTS.get(cls)
    if h is None:
        h = _PARAM_HINTS[cls] = get_type_hints(cls)
    return h


@dataclass(frozen=True, init=False)
class Params:
    """Frozen typed parameters (reference _types.py:638-698)."""

    def __init__(self, **kwargs: Any) -> None:
        hints = _param_hints(type(self))
        for k in kwargs:
            if k not in hints:
                raise TypeError(f"Missing field '{k}' in {type(self).__name__}")
        for name, ann in hints.items():
            if name in kwargs:
                v = kwargs[name]
            elif hasattr(type(self), name):
                v = getattr(type(self), name)
            elif ann in PRIMITIVE_TYPES:
                v = zero_of(ann)
            else:
                raise TypeError(f"Missing value for field '{name}' in {type(self).__name__}")
            object.__setattr__(self, name, v)
        self._validate()

    def __init_subclass__(cls, **kwargs: Any) -> None:
        super().__init_subclass__(**kwargs)
        dataclass(frozen=True, init=False)(cls)
        loose = {k for k, v in cls.__dict__.items()
                 if not k.startswith("_") and not callable(v) and k not in getattr(cls, "__annotations__", {})}
        if loose:
            raise TypeError(f"All fields in {cls.__name__} must be annotated\nUnannotated: {', '.join(sorted(loose))}")
        cls()._validate()

    def _validate_field(self, name: str, val: Any) -> None:
        hints = _param_hints(type(self))
        if name not in hints:
            raise TypeError(f"Missing field '{name}' in {type(self).__name__}")
        t = hints[name]
        bad = (t in _FLOAT_TYPES and not isinstance(val, (float, np.floating))
               or t in _INT_TYPES and (not isinstance(val, (int, np.integer)) or isinstance(val, _builtins.bool))
               or t in _BOOL_TYPES and not isinstance(val, _builtins.bool)
               or t in _VEC_TYPES and not isinstance(val, t))
        if bad:
            raise TypeError(f"Type mismatch for '{name}' in {type(self).__name__}: expected {t.__name__}, "
                            f"got {type(val).__name__} ({val!r})")

    def _validate(self) -> None:
        hints = _param_hints(type(self))
        for name, t in hints.items():
            if t not in PRIMITIVE_TYPES:
                raise TypeError(f"Unsupported type '{t}' for '{name}' in {type(self).__name__}")
            if hasattr(self, name):
                self._validate_field(name, getattr(self, name))


def param_fields(cls: type) -> dict[str, Any]:
    return dict(_param_hints(cls))


BASE_CLASSES = [Tissue, Chemistry, Cell, Metrics, Params]
ANNOTATION_NAMES = {"i32": i32, "u32": u32, "f32": f32, "bool": bool, "vec3": vec3, "ivec3": ivec3,
                    "int": int, "float": float}

__all__ = ["i32", "u32", "f32", "bool", "vec3", "ivec3", "Simulation", "BaseData", "Tissue", "Chemistry", "Cell",
           "Metrics", "Params", "random", "random_dir", "dataclasses", "Annotated"]
