"""The allocation-free sort entry point (olc_stage_sort_pairs_noalloc).

It serves callers that cannot allocate device memory — a process whose HBM
belongs to an allocator it does not expose, or a caller that must not pay
cudaMalloc's implicit synchronisation — by taking the sort's temporary memory
from a static device array inside libolc.so.  These tests call it through the
C ABI and compare it, on calls in a row, with olc_stage_sort_pairs (which
takes caller scratch) and with the oracle's stable sort.  The sort is integer
work, so the outputs must be identical, and each call's status word (read back
by olc_sort_noalloc_status) must be clean.  This file is collected last so that a run stopping at the first
failure has already run every other test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle
from oncolytica_b200 import _lib

pytestmark = pytest.mark.gpu

MAX_KEYS = 1 << 20


def _dev(a, cuda):
    import torch

    return torch.from_numpy(a.view(np.int32).copy()).to(cuda)


def _host(t):
    import torch

    torch.cuda.synchronize()
    return t.cpu().numpy().view(np.uint32)


def _sort_with_scratch(olc, cuda, k, v, bits):
    import torch

    n = len(k)
    kin, vin = _dev(k, cuda), (_dev(v, cuda) if v is not None else None)
    kout = torch.empty(n, dtype=torch.int32, device=cuda)
    vout = torch.empty(n, dtype=torch.int32, device=cuda)
    nbytes = olc.olc_sort_scratch_bytes(n, bits)
    scratch = torch.empty(nbytes, dtype=torch.uint8, device=cuda)
    _lib.check(olc.olc_stage_sort_pairs(C.c_void_p(kin.data_ptr()),
                                        C.c_void_p(vin.data_ptr()) if vin is not None else None,
                                        C.c_void_p(kout.data_ptr()), C.c_void_p(vout.data_ptr()), n, bits,
                                        C.c_void_p(scratch.data_ptr()), nbytes, None))
    return _host(kout), _host(vout)


def _sort_noalloc(olc, cuda, k, v, bits):
    import torch

    n = len(k)
    kin, vin = _dev(k, cuda), (_dev(v, cuda) if v is not None else None)
    kout = torch.empty(n, dtype=torch.int32, device=cuda)
    vout = torch.empty(n, dtype=torch.int32, device=cuda)
    _lib.check(olc.olc_stage_sort_pairs_noalloc(C.c_void_p(kin.data_ptr()),
                                                C.c_void_p(vin.data_ptr()) if vin is not None else None,
                                                C.c_void_p(kout.data_ptr()), C.c_void_p(vout.data_ptr()), n, bits,
                                                None))
    return _host(kout), _host(vout)


def _noalloc_status(olc) -> int:
    w = C.c_uint32(0xFFFFFFFF)
    _lib.check(olc.olc_sort_noalloc_status(C.byref(w), None))
    return int(w.value)


def test_noalloc_sort_matches_the_scratch_sort_on_two_calls(cuda, olc):
    rng = np.random.default_rng(2024)
    # full-width keys at the maximum size (four passes: the layout the static
    # array is sized for), then calls that reuse a dirty array
    cases = [(MAX_KEYS, 32, True), (MAX_KEYS, 21, True), (300_001, 13, False)]
    for n, bits, with_vals in cases:
        hi = 1 << bits
        k = rng.integers(0, hi, size=n, dtype=np.uint64).astype(np.uint32)
        v = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32) if with_vals else None
        ref_k, ref_v = _sort_with_scratch(olc, cuda, k, v, bits)
        got_k, got_v = _sort_noalloc(olc, cuda, k, v, bits)
        assert _noalloc_status(olc) == 0
        np.testing.assert_array_equal(got_k, ref_k)
        np.testing.assert_array_equal(got_v, ref_v)
        # the oracle's stable sort: same keys, and the permutation it applies
        ork, perm = oracle.sort_pairs(k)
        np.testing.assert_array_equal(got_k, ork)
        np.testing.assert_array_equal(got_v, v[perm] if v is not None else perm.astype(np.uint32))


def test_noalloc_sort_rejects_bad_key_widths(cuda, olc):
    for bits in (0, 33):
        rc = olc.olc_stage_sort_pairs_noalloc(C.c_void_p(256), None, C.c_void_p(256), C.c_void_p(256), 16, bits,
                                              None)
        assert rc == _lib.OLC_ERR_ARG, bits
        assert "key_bits" in _lib.last_error()


def test_noalloc_sort_rejects_more_keys_than_its_scratch_holds(cuda, olc):
    rc = olc.olc_stage_sort_pairs_noalloc(C.c_void_p(256), None, C.c_void_p(256), C.c_void_p(256), MAX_KEYS + 1,
                                          21, None)
    assert rc == _lib.OLC_ERR_CAPACITY
    assert "1048576" in _lib.last_error()
