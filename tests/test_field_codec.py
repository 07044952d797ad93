"""16-bit field encodings on the CPU: the product's host codec
(oncolytica_b200._fieldcodec, used for uploads and readbacks) against the
oracle's restatement of the kernels' codec (orc_encode16 / orc_decode16), bit
for bit, on random values and on the edges between the offsets; round trips
stay within half a unit in the last place of the stored magnitude; and the
oracle's 16-bit step keeps an encoded field in [0, b]."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from oncolytica_b200 import _fieldcodec as fc


def _values(b: float, n: int = 20_000, seed: int = 3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    q = np.float32(0.25) * np.float32(b)
    edges = np.array([0.0, -0.0, q, np.float32(b) - q, 0.5 * b, b, 1e-30, 1e-6, b * (1 - 1e-7)], np.float32)
    near = np.concatenate([np.nextafter(edges, np.float32(-1)), np.nextafter(edges, np.float32(9))])
    vals = np.concatenate([edges, near, rng.uniform(0.0, b, n).astype(np.float32),
                           (b * rng.uniform(0.0, 1.0, n) ** 8).astype(np.float32),
                           (b - b * rng.uniform(0.0, 1.0, n) ** 8).astype(np.float32)])
    return np.clip(vals, 0.0, b).astype(np.float32)


@pytest.mark.parametrize("storage", [1, 2, 3, 4])
@pytest.mark.parametrize("encoding", [0, 1, 2])
@pytest.mark.parametrize("b", [1.0, 0.7, 3.5])
def test_host_codec_matches_the_oracle(storage, encoding, b):
    v = _values(b)
    bits = fc.encode(v, storage, encoding, b)
    np.testing.assert_array_equal(bits, oracle.to_bits16(v, storage, encoding, b))
    rng = np.random.default_rng(7)
    comp = (rng.standard_normal(v.size) * 1e-4).astype(np.float32)
    np.testing.assert_array_equal(fc.decode(bits, storage, encoding, b), oracle.from_bits16(bits, storage, encoding, b))
    np.testing.assert_array_equal(fc.decode(bits, storage, encoding, b, comp),
                                  oracle.from_bits16(bits, storage, encoding, b, comp=comp))


@pytest.mark.parametrize("storage", [1, 2])
def test_encodings_resolve_values_finely_near_their_offsets(storage):
    b = 1.0
    v = _values(b, seed=11)
    back = {e: fc.decode(fc.encode(v, storage, e, b), storage, e, b) for e in (0, 1, 2)}
    mant = 8 if storage == 1 else 11  # significand bits of BF16 / FP16
    # value: half an ulp of the value; deficit: of b - value; offset3: of the
    # distance to the nearest of 0, b/2, b (FP32 rounding of the reconstruction on top)
    dist = {0: np.abs(v), 1: np.abs(b - v), 2: np.minimum(np.minimum(v, np.abs(v - 0.5 * b)), b - v)}
    for e, d in dist.items():
        bound = d * 2.0 ** -mant + 1e-7 + 2.0 ** -(24 if storage == 2 else 24) * 4
        if storage == 2:
            bound = np.maximum(bound, 2.0 ** -25)  # FP16 subnormal spacing
        assert np.all(np.abs(back[e] - v) <= bound + 1e-30), e
    # near b the deficit and the offsets beat plain values by orders of magnitude
    top = v > 0.99
    assert np.abs(back[1] - v)[top].max() < np.abs(back[0] - v)[top].max() / 16


def test_offset3_codes_use_the_two_top_bits():
    b = 1.0
    v = np.array([0.1, 0.3, 0.6, 0.9, 1.0, 0.5, 0.0], np.float32)
    h = fc.encode(v, 1, 2, b)
    np.testing.assert_array_equal(h >> 14, [0, 2, 1, 3, 3, 1, 0])
    np.testing.assert_array_equal(fc.decode(h, 1, 2, b)[[4, 5, 6]], [1.0, 0.5, 0.0])


@pytest.mark.parametrize("storage,encoding", [(3, 1), (3, 2), (4, 1), (4, 2), (1, 1), (1, 2)])
def test_oracle_step_keeps_encoded_fields_in_range(storage, encoding):
    n = 24
    f = np.full((n, n, n), 1.0 if encoding == 1 else 0.0, np.float32)
    f[0], f[-1], f[:, 0], f[:, -1], f[:, :, 0], f[:, :, -1] = 1, 1, 1, 1, 1, 1
    bits = oracle.to_bits16(f, storage, encoding, 1.0)
    comp = np.zeros(f.shape, np.float32)
    sink = np.zeros(f.shape, np.float32)
    sink[8:16, 8:16, 8:16] = 0.5
    for step in range(5):
        bits, comp = oracle.diffuse16(bits, sink, comp, 4.0, 0.1, 2000.0, 0.1 * (encoding == 2), 1.0, 76, storage,
                                      step=step, encoding=encoding)
        vals = oracle.from_bits16(bits, storage, encoding, 1.0, comp=comp)
        assert vals.min() >= -1e-6 and vals.max() <= 1.0 + 1e-6
        assert np.all(vals[0] == 1.0) and np.all(vals[:, :, -1] == 1.0)


def test_auto_resolution():
    assert fc.resolve("auto", 3, 0.0, 1.0, 1.0) == 2     # O2-like BF16: three offsets (it may be depleted)
    assert fc.resolve("auto", 3, 0.1, 1.0, 0.0) == 2     # decaying drug: three offsets
    assert fc.resolve("auto", 1, 0.0, 1.0, 0.0) == 2     # BF16, nearest: three offsets
    assert fc.resolve("deficit", 3, 0.0, 1.0, 1.0) == 1  # the deficit on request
    assert fc.resolve("auto", 4, 0.0, 1.0, 1.0) == 0     # FP16 keeps values
    assert fc.resolve("auto", 3, 0.0, 0.0, 1.0) == 0     # no positive boundary value
    assert fc.resolve("value", 3, 0.0, 1.0, 1.0) == 0
    with pytest.raises(ValueError):
        fc.resolve("offset3", 3, 0.0, 8.0, 1.0)
    with pytest.raises(ValueError):
        fc.resolve("deficit", 0, 0.0, 1.0, 1.0)
