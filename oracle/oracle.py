"""numpy front end of the C oracle (TEST INFRASTRUCTURE).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker.  The product package oncolytica_b200 never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

from build import build  # noqa: E402

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = build()
        L = C.CDLL(path)
        P = C.c_void_p
        L.orc_next_rand.restype = C.c_float
        L.orc_next_rand.argtypes = [C.POINTER(C.c_uint32)]
        L.orc_seed_rng.restype = C.c_uint32
        L.orc_seed_rng.argtypes = [C.c_uint32, C.c_uint32]
        L.orc_rng_batch.argtypes = [P, C.c_uint32, C.c_int, P, P]
        L.orc_tissue_key.restype = C.c_uint32
        L.orc_tissue_key.argtypes = [C.c_int, C.c_int, C.c_int]
        L.orc_chem_key.restype = C.c_uint32
        L.orc_chem_key.argtypes = [C.c_int, C.c_int, C.c_int]
        L.orc_keys.argtypes = [P, P, P, P, C.c_uint32, P, C.c_float, P]
        L.orc_sort_pairs.argtypes = [P, P, P, P, C.c_uint32]
        L.orc_bin_ranges.argtypes = [P, C.c_uint32, C.c_uint32, P]
        L.orc_diffuse.restype = C.c_int
        L.orc_diffuse.argtypes = [P, P, P, P, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int,
                                  C.c_int]
        L.orc_diffuse_pinned.restype = C.c_int
        L.orc_diffuse_pinned.argtypes = [P, P, P, P, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int,
                                         P, C.c_uint32, C.c_float, C.c_int]
        L.orc_contact.argtypes = [P, P, C.c_uint32, P, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                                  P, P, P, P, P, C.c_int]
        L.orc_contact_mech.argtypes = [P, P, C.c_uint32, P, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                                       P, P, P, C.c_float, C.c_float, C.c_float, P, P, P, C.c_float, C.c_float,
                                       P, P, P, C.c_int]
        L.orc_contact_motion.argtypes = [P, P, C.c_uint32, P, C.c_float, C.c_float, C.c_float, C.c_float,
                                         C.c_float, P, P, P, C.c_float, C.c_float, C.c_float, P, P, P, C.c_float,
                                         C.c_float, P, P, P, P, P, C.c_float, C.c_float, C.c_float, C.c_int, P, P,
                                         P, P, P, P, C.c_int]
        L.orc_tumour_step.restype = C.c_int
        L.orc_tumour_step.argtypes = [P, C.c_int]
        L.orc_tumour_fields.restype = C.c_int
        L.orc_tumour_fields.argtypes = [P, C.c_int]
        L.orc_tumour_agents.restype = C.c_int
        L.orc_tumour_agents.argtypes = [P, C.c_int]
        L.orc_tumour_sizeof.restype = C.c_size_t
        L.orc_round16.argtypes = [P, P, C.c_size_t, C.c_int, P]
        L.orc_diffuse16e.restype = C.c_int
        L.orc_diffuse16e.argtypes = [P, P, P, P, P, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int,
                                     C.c_int, C.c_int, C.c_uint32, C.c_int, C.c_int]
        L.orc_encode16.argtypes = [P, P, C.c_size_t, C.c_int, C.c_int, C.c_float]
        L.orc_decode16.argtypes = [P, P, P, C.c_size_t, C.c_int, C.c_int, C.c_float]
        _lib = L
    return _lib


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ------------------------------------------------------------------ stages

def seed_rng(seed: int, n: int) -> np.ndarray:
    L = lib()
    return np.array([L.orc_seed_rng(seed & 0xFFFFFFFF, i) for i in range(n)], dtype=np.uint32)


def rng_batch(states: np.ndarray, draws: int, dirs: bool = False):
    s = np.ascontiguousarray(states, dtype=np.uint32).copy()
    out = np.zeros((len(s), max(draws, 0)), dtype=np.float32)
    d = np.zeros((len(s), 3), dtype=np.float32) if dirs else None
    lib().orc_rng_batch(_p(s), len(s), draws, _p(out), _p(d))
    return s, out, d


def tissue_key(cx: int, cy: int, cz: int) -> int:
    return int(lib().orc_tissue_key(cx, cy, cz))


def chem_key(cx: int, cy: int, cz: int) -> int:
    return int(lib().orc_chem_key(cx, cy, cz))


def keys(pos: np.ndarray, dims, vs: float, dead: np.ndarray | None = None) -> np.ndarray:
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    x, y, z = (np.ascontiguousarray(pos[:, k]) for k in range(3))
    out = np.zeros(len(pos), dtype=np.uint32)
    d = None if dead is None else np.ascontiguousarray(dead, dtype=np.uint8)
    dims_a = np.array(dims, dtype=np.int32)
    lib().orc_keys(_p(x), _p(y), _p(z), _p(d), len(pos), _p(dims_a), C.c_float(vs), _p(out))
    return out


def sort_pairs(k: np.ndarray, v: np.ndarray | None = None):
    k = np.ascontiguousarray(k, dtype=np.uint32)
    vv = None if v is None else np.ascontiguousarray(v, dtype=np.uint32)
    ko = np.zeros_like(k)
    vo = np.zeros(len(k), dtype=np.uint32)
    lib().orc_sort_pairs(_p(k), _p(vv), _p(ko), _p(vo), len(k))
    return ko, vo


def bin_ranges(sorted_keys: np.ndarray, n_bins: int) -> np.ndarray:
    k = np.ascontiguousarray(sorted_keys, dtype=np.uint32)
    out = np.zeros(2 * n_bins, dtype=np.uint32)
    lib().orc_bin_ranges(_p(k), len(k), n_bins, _p(out))
    return out


def diffuse(f: np.ndarray, sink: np.ndarray | None, dx: float, dt: float, D: float, decay: float,
            boundary: float, substeps: int, nthreads: int = 0) -> np.ndarray:
    """f is indexed [z, y, x]; returns the field after sink + substeps."""
    f = np.ascontiguousarray(f, dtype=np.float32).copy()
    tmp = np.zeros_like(f)
    s = None if sink is None else np.ascontiguousarray(sink, dtype=np.float32).copy()
    dims = np.array([f.shape[2], f.shape[1], f.shape[0]], dtype=np.int32)
    rc = lib().orc_diffuse(_p(f), _p(tmp), _p(s), _p(dims), C.c_float(dx), C.c_float(dt), C.c_float(D),
                           C.c_float(decay), C.c_float(boundary), substeps, nthreads)
    if rc != 0:
        raise ValueError("oracle diffuse: unstable or bad arguments")
    return f


def diffuse_pinned(f: np.ndarray, sink, dx, dt, D, decay, boundary, substeps, pins, pin_value,
                   nthreads: int = 0) -> np.ndarray:
    """orc_diffuse_pinned on a (nz, ny, nx) float32 grid; returns the new grid."""
    f = np.ascontiguousarray(f, dtype=np.float32).copy()
    tmp = np.zeros_like(f)
    s = None if sink is None else np.ascontiguousarray(sink, dtype=np.float32).copy()
    dims = np.array(f.shape[::-1], dtype=np.int32)
    pv = np.ascontiguousarray(pins, dtype=np.uint32)
    rc = lib().orc_diffuse_pinned(_p(f), _p(tmp), _p(s), _p(dims), C.c_float(dx), C.c_float(dt), C.c_float(D),
                                  C.c_float(decay), C.c_float(boundary), substeps, _p(pv), len(pv),
                                  C.c_float(pin_value), nthreads)
    if rc != 0:
        raise ValueError("orc_diffuse_pinned: unstable or bad arguments")
    return f


def to_bits16(f: np.ndarray, storage: int, encoding: int = 0, boundary: float = 0.0) -> np.ndarray:
    """float32 values -> BF16 (storage 1 and 3) or FP16 (storage 2 and 4) bit
    patterns, rounded to nearest even (finite values); with an encoding (1
    deficit, 2 three offsets) the encoded elements of a field whose boundary
    value is ``boundary`` (``orc_encode16``)."""
    f = np.ascontiguousarray(f, dtype=np.float32)
    if encoding:
        out = np.zeros(f.shape, np.uint16)
        lib().orc_encode16(_p(f), _p(out), f.size, storage, encoding, C.c_float(boundary))
        return out
    if storage in (2, 4):
        return f.astype(np.float16).view(np.uint16)
    u = f.view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def round16(f: np.ndarray, storage: int, rnd: np.ndarray | None = None) -> np.ndarray:
    """The 16-bit storage roundings element-wise (``orc_round16``): 1/2 to
    nearest even, 3/4 stochastic with ``rnd`` (uint32 per element), 5 FP16
    toward zero."""
    f = np.ascontiguousarray(f, dtype=np.float32)
    out = np.zeros(f.shape, np.uint16)
    r = None if rnd is None else np.ascontiguousarray(rnd, dtype=np.uint32)
    lib().orc_round16(_p(f), _p(out), f.size, storage, _p(r))
    return out


def from_bits16(h: np.ndarray, storage: int, encoding: int = 0, boundary: float = 0.0,
                comp: np.ndarray | None = None) -> np.ndarray:
    """Field values of 16-bit elements (``orc_decode16`` for an encoding, or
    when the residuals ``comp`` are to be added in the encoded domain)."""
    h = np.ascontiguousarray(h, dtype=np.uint16)
    if encoding or comp is not None:
        out = np.zeros(h.shape, np.float32)
        c = None if comp is None else np.ascontiguousarray(comp, dtype=np.float32).reshape(h.shape)
        lib().orc_decode16(_p(h), _p(c), _p(out), h.size, storage, encoding, C.c_float(boundary))
        return out
    if storage in (2, 4):
        return h.view(np.float16).astype(np.float32)
    return (h.astype(np.uint32) << 16).view(np.float32)


def diffuse16(bits: np.ndarray, sink: np.ndarray | None, comp: np.ndarray, dx: float, dt: float, D: float,
              decay: float, boundary: float, substeps: int, storage: int, step: int = 0, field: int = 0,
              nthreads: int = 0, encoding: int = 0):
    """One step of a 16-bit field (indexed [z, y, x]): returns (bits, comp).
    ``step`` and ``field`` salt the stochastic rounding of storages 3 and 4;
    ``encoding`` is the elements' (0 value, 1 deficit, 2 three offsets)."""
    f = np.ascontiguousarray(bits, dtype=np.uint16).copy()
    tmp = np.zeros_like(f)
    c = np.ascontiguousarray(comp, dtype=np.float32).copy()
    s = None if sink is None else np.ascontiguousarray(sink, dtype=np.float32).copy()
    dims = np.array([f.shape[2], f.shape[1], f.shape[0]], dtype=np.int32)
    rc = lib().orc_diffuse16e(_p(f), _p(tmp), _p(s), _p(c), _p(dims), C.c_float(dx), C.c_float(dt), C.c_float(D),
                              C.c_float(decay), C.c_float(boundary), substeps, storage, encoding, C.c_uint32(step),
                              field, nthreads)
    if rc != 0:
        raise ValueError("oracle diffuse16: unstable or bad arguments")
    return f, c


def diffuse_f64(f: np.ndarray, sink: np.ndarray | None, dx: float, dt: float, D: float, decay: float,
                boundary: float, substeps: int, split: bool = False, nthreads: int = 0,
                tmp: np.ndarray | None = None) -> np.ndarray:
    """A field scheme evaluated in FP64: the FP32 scheme (decay in every
    substep) or, with ``split``, the 16-bit scheme's (decay once per step).
    With ``tmp`` (a float64 array of f's shape) a C-contiguous float64 ``f``
    is advanced in place and returned (long runs at full size)."""
    if tmp is not None and f.dtype == np.float64 and f.flags.c_contiguous:
        assert tmp.shape == f.shape and tmp.dtype == np.float64
    else:
        f = np.ascontiguousarray(f, dtype=np.float64).copy()
        tmp = np.zeros_like(f)
    s = None if sink is None else np.ascontiguousarray(sink, dtype=np.float32)
    dims = np.array([f.shape[2], f.shape[1], f.shape[0]], dtype=np.int32)
    rc = lib().orc_diffuse_f64(_p(f), _p(tmp), _p(s), _p(dims), C.c_double(dx), C.c_double(dt), C.c_double(D),
                               C.c_double(decay), C.c_double(boundary), substeps, int(bool(split)), nthreads)
    if rc != 0:
        raise ValueError("oracle diffuse_f64: bad arguments")
    return f


def contact(posr: np.ndarray, ranges: np.ndarray, tdims, tvs: float, stiffness: float, mobility: float,
            max_disp: float, dt: float, lo, hi, nthreads: int = 0):
    posr = np.ascontiguousarray(posr, dtype=np.float32)
    n = len(posr)
    x = posr[:, 0].copy()
    y = posr[:, 1].copy()
    z = posr[:, 2].copy()
    td = np.array(tdims, dtype=np.int32)
    lo_a = np.array(lo, dtype=np.float32)
    hi_a = np.array(hi, dtype=np.float32)
    r = np.ascontiguousarray(ranges, dtype=np.uint32)
    lib().orc_contact(_p(posr), _p(r), n, _p(td), C.c_float(tvs), C.c_float(stiffness), C.c_float(mobility),
                      C.c_float(max_disp), C.c_float(dt), _p(lo_a), _p(hi_a), _p(x), _p(y), _p(z), nthreads)
    return np.stack([x, y, z], axis=1)


def contact_mech(posr: np.ndarray, ranges: np.ndarray, tdims, tvs: float, stiffness: float, mobility: float,
                 max_disp: float, dt: float, lo, hi, state=None, necrotic_factor: float = 1.0, adh_k: float = 0.0,
                 adh_range: float = 0.0, vel: np.ndarray | None = None, damping: float = 0.0,
                 max_speed: float = 0.0, nthreads: int = 0):
    """orc_contact_mech; returns positions (n, 3) and, with `vel`, the new velocities."""
    posr = np.ascontiguousarray(posr, dtype=np.float32)
    n = len(posr)
    x, y, z = (posr[:, k].copy() for k in range(3))
    td = np.array(tdims, dtype=np.int32)
    lo_a = np.array(lo, dtype=np.float32)
    hi_a = np.array(hi, dtype=np.float32)
    r = np.ascontiguousarray(ranges, dtype=np.uint32)
    st = None if state is None else np.ascontiguousarray(state, dtype=np.int32)
    v = None if vel is None else [np.ascontiguousarray(vel[:, k], dtype=np.float32).copy() for k in range(3)]
    lib().orc_contact_mech(_p(posr), _p(r), n, _p(td), C.c_float(tvs), C.c_float(stiffness), C.c_float(mobility),
                           C.c_float(max_disp), C.c_float(dt), _p(lo_a), _p(hi_a), _p(st), C.c_float(necrotic_factor),
                           C.c_float(adh_k), C.c_float(adh_range), _p(v[0]) if v else None,
                           _p(v[1]) if v else None, _p(v[2]) if v else None, C.c_float(damping),
                           C.c_float(max_speed), _p(x), _p(y), _p(z), nthreads)
    pos = np.stack([x, y, z], axis=1)
    return (pos, np.stack(v, axis=1)) if v else (pos, None)


def contact_motion(posr, ranges, tdims, tvs, stiffness, mobility, max_disp, dt, lo, hi, state=None,
                   necrotic_factor=1.0, adh_k=0.0, adh_range=0.0, vel=None, damping=0.0, max_speed=0.0,
                   species=None, rng=None, o2=None, glu=None, cdims=(1, 1, 1), cvs=1.0, chemo_force=2.0,
                   impulse=0.4, table=((0.0, 0.0, 0.0),), nthreads: int = 0):
    """orc_contact_motion; `table` rows are (chemotaxis_o2, chemotaxis_glucose,
    move_prob).  Returns positions, velocities (or None) and the advanced RNG
    states (or None)."""
    posr = np.ascontiguousarray(posr, dtype=np.float32)
    n = len(posr)
    x, y, z = (posr[:, k].copy() for k in range(3))
    td = np.array(tdims, dtype=np.int32)
    cd = np.array(cdims, dtype=np.int32)
    lo_a = np.array(lo, dtype=np.float32)
    hi_a = np.array(hi, dtype=np.float32)
    r = np.ascontiguousarray(ranges, dtype=np.uint32)
    st = None if state is None else np.ascontiguousarray(state, dtype=np.int32)
    v = None if vel is None else [np.ascontiguousarray(vel[:, k], dtype=np.float32).copy() for k in range(3)]
    spc = None if species is None else np.ascontiguousarray(species, dtype=np.int32)
    rg = None if rng is None else np.ascontiguousarray(rng, dtype=np.uint32).copy()
    f0 = None if o2 is None else np.ascontiguousarray(o2, dtype=np.float32)
    f1 = None if glu is None else np.ascontiguousarray(glu, dtype=np.float32)
    tab = np.zeros((8, 3), np.float32)
    if len(table):
        tab[: len(table)] = np.asarray(table, np.float32).reshape(len(table), 3)
    so2, sglu, smv = (np.ascontiguousarray(tab[:, k]) for k in range(3))
    lib().orc_contact_motion(_p(posr), _p(r), n, _p(td), C.c_float(tvs), C.c_float(stiffness),
                             C.c_float(mobility), C.c_float(max_disp), C.c_float(dt), _p(lo_a), _p(hi_a), _p(st),
                             C.c_float(necrotic_factor), C.c_float(adh_k), C.c_float(adh_range),
                             _p(v[0]) if v else None, _p(v[1]) if v else None, _p(v[2]) if v else None,
                             C.c_float(damping), C.c_float(max_speed), _p(spc), _p(rg), _p(f0), _p(f1), _p(cd),
                             C.c_float(cvs), C.c_float(chemo_force), C.c_float(impulse), len(table), _p(so2),
                             _p(sglu), _p(smv), _p(x), _p(y), _p(z), nthreads)
    return np.stack([x, y, z], axis=1), (np.stack(v, axis=1) if v else None), rg


# ------------------------------------------------------------------ tumour workload

class OrcTumour(C.Structure):
    _fields_ = [
        ("cap", C.c_uint32), ("n", C.c_uint32),
        ("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p), ("radius", C.c_void_p), ("volume", C.c_void_p),
        ("state", C.c_void_p), ("rng", C.c_void_p),
        ("x2", C.c_void_p), ("y2", C.c_void_p), ("z2", C.c_void_p), ("radius2", C.c_void_p),
        ("volume2", C.c_void_p), ("state2", C.c_void_p), ("rng2", C.c_void_p),
        ("dead", C.c_void_p),
        ("tdims", C.c_int32 * 3), ("tvs", C.c_float),
        ("cdims", C.c_int32 * 3), ("cvs", C.c_float),
        ("lo", C.c_float * 3), ("hi", C.c_float * 3),
        ("o2", C.c_void_p), ("o2_tmp", C.c_void_p), ("o2_sink", C.c_void_p),
        ("drug", C.c_void_p), ("drug_tmp", C.c_void_p),
        ("has_drug", C.c_int),
        ("dt", C.c_float), ("growth", C.c_float), ("v_div", C.c_float), ("o2_necrotic", C.c_float),
        ("o2_quiescent", C.c_float), ("uptake", C.c_float), ("death_k", C.c_float),
        ("D_o2", C.c_float), ("D_drug", C.c_float), ("decay_drug", C.c_float), ("bnd_o2", C.c_float),
        ("bnd_drug", C.c_float),
        ("S_o2", C.c_int), ("S_drug", C.c_int),
        ("stiffness", C.c_float), ("mobility", C.c_float), ("max_disp", C.c_float), ("margin", C.c_float),
        ("births", C.c_uint32), ("deaths", C.c_uint32),
    ]


AGENT_COLS = ("x", "y", "z", "radius", "volume", "state", "rng")
_DT = {"x": np.float32, "y": np.float32, "z": np.float32, "radius": np.float32, "volume": np.float32,
       "state": np.int32, "rng": np.uint32}


class TumourOracle:
    """Owns numpy buffers for the C tumour step.  `spec` is a workloads.TumourSpec."""

    def __init__(self, spec, agents: dict, o2: np.ndarray, drug: np.ndarray | None, capacity: int):
        assert lib().orc_tumour_sizeof() == C.sizeof(OrcTumour)
        self.spec = spec
        self.cap = capacity
        self.bufs = {}
        for k in AGENT_COLS:
            a = np.zeros(capacity, dtype=_DT[k])
            b = np.zeros(capacity, dtype=_DT[k])
            a[: len(agents[k])] = agents[k]
            self.bufs[k] = a
            self.bufs[k + "2"] = b
        self.dead = np.zeros(capacity, dtype=np.uint8)
        self.o2 = np.ascontiguousarray(o2, dtype=np.float32).copy()
        self.o2_tmp = np.zeros_like(self.o2)
        self.o2_sink = np.zeros_like(self.o2)
        self.has_drug = drug is not None
        self.drug = np.ascontiguousarray(drug, dtype=np.float32).copy() if drug is not None else np.zeros(1, np.float32)
        self.drug_tmp = np.zeros_like(self.drug)
        t = OrcTumour()
        t.cap = capacity
        t.n = len(agents["x"])
        t.tdims[:] = spec.tissue_dims
        t.tvs = spec.bin_size
        t.cdims[:] = spec.field_dims
        t.cvs = spec.dx
        t.lo[:] = (0.0, 0.0, 0.0)
        t.hi[:] = (spec.domain,) * 3
        t.has_drug = int(self.has_drug)
        for name in ("dt", "growth", "v_div", "o2_necrotic", "o2_quiescent", "uptake", "death_k", "D_o2",
                     "D_drug", "decay_drug", "bnd_o2", "bnd_drug", "stiffness", "mobility", "max_disp",
                     "margin"):
            setattr(t, name, float(getattr(spec, name)))
        t.S_o2 = int(spec.S_o2)
        t.S_drug = int(spec.S_drug)
        self.t = t
        self._bind()

    @classmethod
    def from_snapshot(cls, spec, snap: dict, capacity: int) -> "TumourOracle":
        """Oracle state equal to a device snapshot (CudaBackend.snapshot())."""
        c = snap["cols"]
        agents = {"x": c["pos.x"], "y": c["pos.y"], "z": c["pos.z"], "radius": c["radius"], "volume": c["volume"],
                  "state": c["state"], "rng": c["_rng_state"]}
        shp = tuple(spec.field_dims[::-1])
        o2 = snap["fields"]["o2"].reshape(shp)
        drug = snap["fields"]["drug"].reshape(shp) if spec.has_drug else None
        o = cls(spec, agents, o2, drug, capacity)
        o.dead[: snap["rows"]] = snap["life"]
        if snap["sinks"].get("o2") is not None:
            o.o2_sink[...] = snap["sinks"]["o2"].reshape(shp)
        return o

    def _bind(self):
        t = self.t
        for k in AGENT_COLS:
            setattr(t, k, self.bufs[k].ctypes.data)
            setattr(t, k + "2", self.bufs[k + "2"].ctypes.data)
        t.dead = self.dead.ctypes.data
        t.o2 = self.o2.ctypes.data
        t.o2_tmp = self.o2_tmp.ctypes.data
        t.o2_sink = self.o2_sink.ctypes.data
        t.drug = self.drug.ctypes.data
        t.drug_tmp = self.drug_tmp.ctypes.data

    def _sync_after(self):
        # the C side swaps its agent buffer pointers; mirror that here
        t = self.t
        for k in AGENT_COLS:
            if getattr(t, k) != self.bufs[k].ctypes.data:
                self.bufs[k], self.bufs[k + "2"] = self.bufs[k + "2"], self.bufs[k]
        self._bind()

    def step(self, nthreads: int = 0):
        rc = lib().orc_tumour_step(C.byref(self.t), nthreads)
        self._sync_after()
        if rc != 0:
            raise RuntimeError("oracle tumour step failed")

    def fields(self, nthreads: int = 0):
        if lib().orc_tumour_fields(C.byref(self.t), nthreads) != 0:
            raise RuntimeError("oracle fields failed")

    def fields_sample(self, substeps: int, nthreads: int = 0) -> None:
        """`substeps` substeps of every field in place, at the same diffusion
        number as the full step (dt scaled by substeps / S) — a bounded sample
        of the field phase for timing."""
        sp = self.spec
        dims = np.array(sp.field_dims, dtype=np.int32)
        L = lib()
        for f, tmp, D, decay, bnd, S in ((self.o2, self.o2_tmp, sp.D_o2, 0.0, sp.bnd_o2, sp.S_o2),
                                         (self.drug, self.drug_tmp, sp.D_drug, sp.decay_drug, sp.bnd_drug,
                                          sp.S_drug)):
            if S == 0 or f.size < 8:
                continue
            rc = L.orc_diffuse(_p(f), _p(tmp), None, _p(dims), C.c_float(sp.dx), C.c_float(sp.dt * substeps / S),
                               C.c_float(D), C.c_float(decay), C.c_float(bnd), substeps, nthreads)
            if rc != 0:
                raise RuntimeError("oracle fields sample failed")

    def agents_part(self, nthreads: int = 0):
        rc = lib().orc_tumour_agents(C.byref(self.t), nthreads)
        self._sync_after()
        if rc != 0:
            raise RuntimeError("oracle agents failed")

    @property
    def rows(self) -> int:
        return int(self.t.n)

    def live_agents(self) -> dict:
        n = self.rows
        keep = self.dead[:n] == 0
        return {k: self.bufs[k][:n][keep].copy() for k in AGENT_COLS}


# ------------------------------------------------------------------ engine metrics

ENGINE_METRIC_NAMES = (
    "total_live", "n_prolif", "n_quiesc", "n_necr", "frac_prolif", "frac_quiesc", "frac_necr", "frac_hypoxic",
    "csc_count", "csc_frac", "centroid_x", "centroid_y", "centroid_z", "r_gyration", "r_invasive", "r_necrotic",
    "rim_thickness", "mean_energy", "mean_o2", "mean_glu", "mean_speed", "crowd_frac", "step",
)


def _bin(p: np.ndarray, vs: float, dim: int) -> np.ndarray:
    """trunc(p / vs) with an IEEE float32 divide, clamped to [0, dim - 1]."""
    q = (np.asarray(p, dtype=np.float32) / np.float32(vs)).astype(np.float32)
    c = np.trunc(q)
    c = np.where(np.isnan(c), 0.0, c)
    return np.clip(c, 0, dim - 1).astype(np.int64)


def engine_metrics(x, y, z, life, state, center, step: int, o2=None, glu=None, cdims=None, cvs=None,
                   bin_counts=None, tdims=None, tvs=None, energy=None, speed=None, csc=None,
                   hypoxia: float = 0.1, crowd: int = 12) -> dict:
    """Restates Kernel_CollectMetrics / Kernel_FinalizeMetrics
    (engine/assets/shaders/tumor_sim.wgsl:255-361) in FP64 with exact counts.

    x, y, z, life, state: the rows in use (life 0 = alive); o2 / glu: flat
    float32 fields (x fastest) sampled at the agent's nearest voxel; bin_counts:
    agents per bin key of the last sort (crowding: more than `crowd`).  Necrotic
    agents (state 3) only count; state 0 (deleted) is skipped; state 1 is
    proliferating and any other state quiescent."""
    x = np.asarray(x, np.float32)
    y = np.asarray(y, np.float32)
    z = np.asarray(z, np.float32)
    st = np.ones(len(x), np.int32) if state is None else np.asarray(state, np.int32)
    alive = (np.asarray(life) == 0) & (st != 0)
    necr = alive & (st == 3)
    live = alive & (st != 3)
    prolif = live & (st == 1)
    n_prolif, n_live, n_necr = int(prolif.sum()), int(live.sum()), int(necr.sum())
    n_quiesc = n_live - n_prolif
    dx = x[live].astype(np.float64) - np.float64(np.float32(center[0]))
    dy = y[live].astype(np.float64) - np.float64(np.float32(center[1]))
    dz = z[live].astype(np.float64) - np.float64(np.float32(center[2]))
    r2 = dx * dx + dy * dy + dz * dz
    f_live = max(float(n_live), 1.0)
    f_total = max(float(n_live + n_necr), 1.0)
    n_csc = int((np.asarray(csc)[live] != 0).sum()) if csc is not None else 0
    n_hyp, s_o2, s_glu = 0, 0.0, 0.0
    if o2 is not None or glu is not None:
        cx, cy, cz = (_bin(c[live], cvs, cdims[k]) for k, c in enumerate((x, y, z)))
        v = (cz * cdims[1] + cy) * cdims[0] + cx
        if o2 is not None:
            s = np.asarray(o2, np.float32)[v]
            s_o2 = float(s.astype(np.float64).sum())
            n_hyp = int((s < np.float32(hypoxia)).sum())
        if glu is not None:
            s_glu = float(np.asarray(glu, np.float32)[v].astype(np.float64).sum())
    n_crowd = 0
    if bin_counts is not None:
        tx, ty, tz = (_bin(c[live], tvs, tdims[k]) for k, c in enumerate((x, y, z)))
        keys = np.array([tissue_key(int(a), int(b), int(c)) for a, b, c in zip(tx, ty, tz)], dtype=np.int64)
        n_crowd = int((np.asarray(bin_counts)[keys] > crowd).sum())
    s_energy = float(np.asarray(energy, np.float32)[live].astype(np.float64).sum()) if energy is not None else 0.0
    s_speed = 0.0
    if speed is not None:
        sv = [np.asarray(c, np.float32)[live].astype(np.float64) for c in speed]
        s_speed = float(np.sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]).sum())
    r_inv = float(np.sqrt(r2).max()) if n_live else 0.0
    r_necr = 0.5 * (n_necr / 0.65) ** 0.333333 if n_necr > 0 else 0.0
    out = [n_live, n_prolif, n_quiesc, n_necr, n_prolif / f_live, n_quiesc / f_live, n_necr / f_total,
           n_hyp / f_live, n_csc, n_csc / f_live,
           float(np.float32(center[0])) + float(dx.sum()) / f_live,
           float(np.float32(center[1])) + float(dy.sum()) / f_live,
           float(np.float32(center[2])) + float(dz.sum()) / f_live,
           float(np.sqrt(r2.sum() / f_live)), r_inv, r_necr, max(r_inv - r_necr, 0.0),
           s_energy / f_live, s_o2 / f_live, s_glu / f_live, s_speed / f_live, n_crowd / f_live, float(step)]
    return dict(zip(ENGINE_METRIC_NAMES, [float(v) for v in out]))


def bin_counts_of(x, y, z, life, tdims, tvs, n_table: int) -> np.ndarray:
    """Agents per bin key among rows with life 0 (the bin table's range
    lengths after a sort of those rows)."""
    keep = np.asarray(life) == 0
    tx, ty, tz = (_bin(np.asarray(c)[keep], tvs, tdims[k]) for k, c in enumerate((x, y, z)))
    keys = np.array([tissue_key(int(a), int(b), int(c)) for a, b, c in zip(tx, ty, tz)], dtype=np.int64)
    return np.bincount(keys, minlength=n_table)
