"""Host-side conversions of 16-bit field elements (numpy, FP32 arithmetic).

The device stores BF16 or FP16 elements with an encoding (olc.h OLC_ENC_*):
``value`` holds the field value, ``deficit`` holds boundary - value, and
``offset3`` holds the value minus the offset o in {0, b/2, b} nearest it, o
and the sign named by bits 15 and 14.  These functions convert field values to
elements (rounded to nearest even, as the device's reaction pass rounds) for
uploads, and elements (plus their FP32 residuals, kept in the encoded domain)
back to field values for readback.  Every operation is one FP32 operation in
the order the kernels use (oncolytica_b200/csrc/olc_store16.cuh: Codec), so
uploads and readbacks agree with the device bit for bit.
"""
from __future__ import annotations

import numpy as np

ENCODINGS = {"value": 0, "deficit": 1, "offset3": 2}
BF16_STORAGES = (1, 3)  # OLC_FIELD_BF16, OLC_FIELD_BF16_SR (2 and 4 are FP16)

_F = np.float32


def _round16(f: np.ndarray, storage: int) -> np.ndarray:
    """FP32 -> BF16 / FP16 bit patterns, to nearest even (finite values)."""
    f = np.ascontiguousarray(f, dtype=np.float32)
    if storage not in BF16_STORAGES:
        return f.astype(np.float16).view(np.uint16)
    u = f.view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def _widen16(h: np.ndarray, storage: int) -> np.ndarray:
    h = np.ascontiguousarray(h, dtype=np.uint16)
    if storage not in BF16_STORAGES:
        return h.view(np.float16).astype(np.float32)
    return (h.astype(np.uint32) << 16).view(np.float32)


def _consts(boundary: float):
    b = _F(boundary)
    hb = _F(_F(0.5) * b)
    qb = _F(_F(0.25) * b)
    return b, hb, qb, _F(b - qb)


def encode(values: np.ndarray, storage: int, encoding: int, boundary: float) -> np.ndarray:
    """Field values -> 16-bit elements (uint16), rounded to nearest even."""
    f = np.ascontiguousarray(values, dtype=np.float32)
    if encoding == 0:
        return _round16(f, storage)
    b, hb, qb, uq = _consts(boundary)
    if encoding == 1:
        return _round16(b - f, storage)
    f = np.minimum(np.maximum(f, _F(0.0)), b)
    lo, hi = f < qb, f > uq
    d = f - hb
    mag = np.where(lo, np.abs(f), np.where(hi, b - f, np.abs(d))).astype(np.float32)
    code = np.where(lo, 0, np.where(hi, 0xC000, np.where(d < 0, 0x8000, 0x4000))).astype(np.uint16)
    return _round16(mag, storage) | code


def work(h: np.ndarray, storage: int, encoding: int, boundary: float) -> np.ndarray:
    """The encoded-domain value of each element (the deficit for ``deficit``,
    the field value otherwise)."""
    h = np.ascontiguousarray(h, dtype=np.uint16)
    if encoding != 2:
        return _widen16(h, storage)
    _, hb, _, _ = _consts(boundary)
    m = _widen16(h & np.uint16(0xBFFF), storage)
    units = ((h >> 15) + ((h >> 14) & 1)).astype(np.float32)
    return (m + (units * hb).astype(np.float32)).astype(np.float32)


def decode(h: np.ndarray, storage: int, encoding: int, boundary: float,
           residual: np.ndarray | None = None) -> np.ndarray:
    """16-bit elements (plus their residuals, when given) -> field values."""
    w = work(h, storage, encoding, boundary)
    if residual is not None:
        w = (w + np.ascontiguousarray(residual, dtype=np.float32).reshape(w.shape)).astype(np.float32)
    if encoding == 1:
        return (_F(boundary) - w).astype(np.float32)
    return w


def resolve(encoding: str, storage: int, decay: float, boundary: float, initial_mean: float | None) -> int:
    """The encoding code of a field: explicit names map directly; "auto"
    picks ``offset3`` for BF16 storage with a boundary value in (0, 4]: it
    resolves values near 0, b/2 and b finely wherever the field goes (an O2
    field stays near b only until a large population depletes it; ``deficit``
    then loses precision near 0: 1.4e-3 relative L2 against FP64 after 1,000
    steps of the 1 M-agent workload, against 7e-4 for ``offset3``); FP16 and
    FP32 fields, and BF16 fields outside that range, keep ``value``.
    ``decay`` and ``initial_mean`` are accepted for callers that choose by
    them."""
    if encoding != "auto":
        if encoding not in ENCODINGS:
            raise ValueError(f"encoding must be 'auto' or one of {sorted(ENCODINGS)}, got {encoding!r}")
        code = ENCODINGS[encoding]
        if code and storage == 0:
            raise ValueError("encodings apply to 16-bit field storage only")
        if code == 1 and not boundary > 0.0:
            raise ValueError("encoding 'deficit' needs a boundary value > 0")
        if code == 2 and not 0.0 < boundary <= 4.0:
            raise ValueError("encoding 'offset3' needs 0 < boundary <= 4")
        return code
    if storage not in BF16_STORAGES or not 0.0 < boundary <= 4.0:
        return 0
    return 2
