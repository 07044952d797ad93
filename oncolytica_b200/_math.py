"""ol.math — the math namespace of the DSL (reference framework/src/oncolytica/core/utils/_math.py).

Every function evaluates in float32 with one rounding per operation, matching
the CUDA helpers in csrc/olc_rule_rt.cuh.  The translator maps each name to a
CUDA function (``compiler.emit_cuda.MATH``).
"""
from __future__ import annotations

import builtins as _builtins
import math as _pymath

import numpy as np

from oncolytica_b200._types import F32, f32, i32, ivec3, u32, vec3
from oncolytica_b200._types import bool as ol_bool


def _f(v) -> np.float32:
    return np.float32(v)


def dot(a: vec3, b: vec3) -> np.float32:
    return (a.x * b.x + a.y * b.y) + a.z * b.z


def length_sq(v: vec3) -> np.float32:
    return dot(v, v)


def length(v: vec3) -> np.float32:
    return np.sqrt(dot(v, v))


def distance_sq(a: vec3, b: vec3) -> np.float32:
    return length_sq(a - b)


def distance(a: vec3, b: vec3) -> np.float32:
    return length(a - b)


def normalize(v: vec3) -> vec3:
    n = length(v)
    if n == 0.0:
        return vec3(0.0, 0.0, 0.0)
    inv = F32(1.0) / n
    return v * inv


def cross(a: vec3, b: vec3) -> vec3:
    return vec3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x)


def reflect(v: vec3, normal: vec3) -> vec3:
    d = F32(2.0) * dot(v, normal)
    return v - normal * d


def lerp_vec(a: vec3, b: vec3, t) -> vec3:
    t = _f(t)
    it = F32(1.0) - t
    return vec3(a.x * it + b.x * t, a.y * it + b.y * t, a.z * it + b.z * t)


def clamp(value, min_val, max_val):
    if isinstance(value, vec3):
        return vec3(max(min_val.x, min(max_val.x, value.x)), max(min_val.y, min(max_val.y, value.y)),
                    max(min_val.z, min(max_val.z, value.z)))
    if isinstance(value, (int, np.integer)) and isinstance(min_val, (int, np.integer)) and \
            isinstance(max_val, (int, np.integer)):
        return _builtins.max(min_val, _builtins.min(max_val, value))
    v, lo, hi = _f(value), _f(min_val), _f(max_val)
    return np.fmax(lo, np.fmin(hi, v))


def lerp(a, b, t) -> np.float32:
    a, b, t = _f(a), _f(b), _f(t)
    return a + (b - a) * t


def sign(x):
    if isinstance(x, (int, np.integer)) and not isinstance(x, bool):
        return 1 if x > 0 else (-1 if x < 0 else 0)
    x = _f(x)
    return F32(1.0) if x > 0 else (F32(-1.0) if x < 0 else F32(0.0))


def smoothstep(edge0, edge1, x) -> np.float32:
    t = clamp((_f(x) - _f(edge0)) / (_f(edge1) - _f(edge0)), F32(0.0), F32(1.0))
    return t * t * (F32(3.0) - F32(2.0) * t)


def step(edge, x) -> np.float32:
    return F32(0.0) if _f(x) < _f(edge) else F32(1.0)


def fract(x) -> np.float32:
    x = _f(x)
    return x - np.floor(x)


def _u(fn):
    def g(x):
        return fn(_f(x))

    g.__name__ = fn.__name__
    return g


sqrt = _u(np.sqrt)
exp = _u(np.exp)
exp2 = _u(np.exp2)
log = _u(np.log)
log2 = _u(np.log2)
sin = _u(np.sin)
cos = _u(np.cos)
tan = _u(np.tan)
asin = _u(np.arcsin)
acos = _u(np.arccos)
atan = _u(np.arctan)
sinh = _u(np.sinh)
cosh = _u(np.cosh)
tanh = _u(np.tanh)
floor = _u(np.floor)
ceil = _u(np.ceil)
fabs = _u(np.fabs)
trunc = _u(np.trunc)
round = _u(np.rint)  # noqa: A001


def inverse_sqrt(x) -> np.float32:
    return F32(1.0) / np.sqrt(_f(x))


def pow(a, b) -> np.float32:  # noqa: A001
    return np.power(_f(a), _f(b))


def atan2(y, x) -> np.float32:
    return np.arctan2(_f(y), _f(x))


def abs(x):  # noqa: A001
    if isinstance(x, (int, np.integer)) and not isinstance(x, bool):
        return _builtins.abs(x)
    return np.fabs(_f(x))


def min(a, b):  # noqa: A001
    if all(isinstance(v, (int, np.integer)) for v in (a, b)):
        return _builtins.min(a, b)
    return np.fmin(_f(a), _f(b))


def max(a, b):  # noqa: A001
    if all(isinstance(v, (int, np.integer)) for v in (a, b)):
        return _builtins.max(a, b)
    return np.fmax(_f(a), _f(b))


pi = _pymath.pi
tau = _pymath.tau
inf = _pymath.inf

# Return types for the translator's type inference (reference _math.py:150-208).
INTRINSIC_RETURNS = {
    "length": f32, "length_sq": f32, "distance": f32, "distance_sq": f32, "dot": f32,
    "normalize": vec3, "cross": vec3, "reflect": vec3, "lerp_vec": vec3, "random_dir": vec3,
    "sin": f32, "cos": f32, "tan": f32, "asin": f32, "acos": f32, "atan": f32, "atan2": f32, "sinh": f32,
    "cosh": f32, "tanh": f32, "pow": f32, "exp": f32, "exp2": f32, "log": f32, "log2": f32, "sqrt": f32,
    "inverse_sqrt": f32, "fabs": f32, "floor": f32, "ceil": f32, "round": f32, "trunc": f32, "fract": f32,
    "lerp": f32, "step": f32, "smoothstep": f32, "random": f32,
    "i32": i32, "u32": u32, "f32": f32, "bool": ol_bool, "vec3": vec3, "ivec3": ivec3, "int": i32, "float": f32,
}
