"""The oracle's 16-bit storage roundings (CPU): round-to-nearest matches
numpy's casts, FP16 toward zero brackets every value by adjacent FP16
numbers, and the stochastic roundings of BF16 and FP16 pick one of the two
neighbours with the probability of the discarded fraction (unbiased)."""
from __future__ import annotations

import numpy as np

import oracle


def _values(n=200_000, seed=3):
    rng = np.random.default_rng(seed)
    v = np.concatenate([rng.uniform(0.0, 1.0, n), 10.0 ** rng.uniform(-9, 4, n), -rng.uniform(0, 2, n // 4),
                        np.array([0.0, 1.0, 0.5, 65504.0, 6.103515625e-05, 5.960464477539063e-08], np.float64)])
    return v.astype(np.float32)


def test_fp16_nearest_matches_numpy_cast():
    v = _values()
    np.testing.assert_array_equal(oracle.round16(v, 2), v.astype(np.float16).view(np.uint16))


def test_fp16_toward_zero_brackets_each_value():
    v = _values()
    h = oracle.round16(v, 5).view(np.float16)
    a = np.abs(v.astype(np.float64))
    lo = np.abs(h.astype(np.float64))
    assert (lo <= a).all()
    up = np.nextafter(np.abs(h), np.float16(np.inf)).astype(np.float64)
    big = a >= 65504.0
    assert (up[~big] > a[~big]).all()
    assert (np.signbit(h) == np.signbit(v)).all()


def test_stochastic_roundings_are_unbiased():
    rng = np.random.default_rng(11)
    for storage, bits, to_f in ((3, 16, lambda h: (h.astype(np.uint32) << 16).view(np.float32)),
                                (4, 13, lambda h: h.view(np.float16).astype(np.float32))):
        x = rng.uniform(0.01, 1.0, 64).astype(np.float32)
        reps = 4000
        xs = np.repeat(x, reps)
        r = rng.integers(0, 2 ** 32, xs.size, dtype=np.uint64).astype(np.uint32)
        got = to_f(oracle.round16(xs, storage, r)).astype(np.float64).reshape(len(x), reps)
        down = to_f(oracle.round16(x, 5) if storage == 4 else
                    ((x.view(np.uint32) >> 16).astype(np.uint16))).astype(np.float64)
        # every result is the value rounded down or the next representable number up
        assert ((got == down[:, None]) | (got > down[:, None])).all()
        ulp = np.abs(got.max(axis=1) - down)
        mean_err = got.mean(axis=1) - x
        # unbiased within 5 standard errors of a two-point draw
        assert (np.abs(mean_err) <= 5 * 0.5 * np.maximum(ulp, 1e-12) / np.sqrt(reps) + 1e-12).all(), storage
        # exact values are kept
        exact = to_f(oracle.round16(x, 2 if storage == 4 else 1))
        kept = oracle.round16(exact, storage, np.full(exact.size, 0xFFFFFFFF, np.uint32))
        np.testing.assert_array_equal(to_f(kept), exact)


def test_stochastic_roundings_match_the_b200_conversions():
    """The oracle's BF16 / FP16 stochastic rounding equals the B200's
    cvt.rs.bf16x2.f32 / cvt.rs.f16x2.f32 on the recorded cases (single random
    bits, random values, every subnormal FP16 result of 2^20 random draws);
    tests/golden/make_rounding_fixture.cu made the file on a B200."""
    import os

    from conftest import GOLDEN

    raw = open(os.path.join(GOLDEN, "rounding_sr.bin"), "rb").read()
    n = int(np.frombuffer(raw[:4], np.int32)[0])
    a, b, r, f16, bf16 = np.frombuffer(raw[4:], np.uint32).reshape(5, n)
    a, b = a.view(np.float32), b.view(np.float32)
    assert n > 16384 and (np.minimum(a, b) < 2.0 ** -14).sum() > 30
    for storage, hw in ((4, f16), (3, bf16)):
        lo = oracle.round16(b, storage, r & 0xFFFF).astype(np.uint32)
        hi = oracle.round16(a, storage, r >> 16).astype(np.uint32)
        np.testing.assert_array_equal((hi << 16) | lo, hw, err_msg=f"storage {storage}")
