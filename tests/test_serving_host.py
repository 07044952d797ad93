"""Serving pool, host side (no GPU): the arena allocator behind admission by
free device memory, and the continuous-batching scheduler run against a fake
pool device — admission order, backfill, out-of-order completion,
cancellation, malformed and oversized requests, and injected faults (fake
out-of-memory, a failing admission)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from oncolytica_b200 import _lib
from oncolytica_b200.serving import (FakePoolDevice, FaultInjector, Footprint, ServingPool, SimRequest,
                                     plan_arenas)


# ---------------------------------------------------------------- arena allocator
class _Arena:
    def __init__(self, olc, cap):
        self.olc = olc
        self.h = C.c_void_p()
        _lib.check(olc.olc_arena_create(cap, C.byref(self.h)))

    def alloc(self, n, align=1):
        off = C.c_uint64()
        rc = self.olc.olc_arena_alloc(self.h, n, align, C.byref(off))
        return off.value if rc == _lib.OLC_OK else None

    def release(self, off, n):
        return self.olc.olc_arena_release(self.h, off, n)

    def stats(self):
        u, lf, fr = C.c_uint64(), C.c_uint64(), C.c_uint64()
        _lib.check(self.olc.olc_arena_stats(self.h, C.byref(u), C.byref(lf), C.byref(fr)))
        return u.value, lf.value, fr.value

    def close(self):
        self.olc.olc_arena_destroy(self.h)


def test_arena_random_alloc_release_never_overlaps(olc):
    cap = 1 << 20
    a = _Arena(olc, cap)
    rng = np.random.default_rng(7)
    live = {}
    owner = np.zeros(cap, np.int32)  # 0 free, else the allocation's id
    next_id = 1
    for it in range(3000):
        if live and (rng.random() < 0.45 or len(live) > 60):
            key = list(live)[rng.integers(len(live))]
            off, n = live.pop(key)
            assert a.release(off, n) == _lib.OLC_OK
            assert (owner[off:off + n] == key).all()
            owner[off:off + n] = 0
        else:
            n = int(rng.integers(1, 40000))
            align = int(1 << rng.integers(0, 8))
            off = a.alloc(n, align)
            if off is None:
                # refused only when no aligned free run of n exists
                free = owner == 0
                runs = np.flatnonzero(np.diff(np.concatenate(([0], free.astype(np.int8), [0]))))
                fits = any(((s + align - 1) // align * align) + n <= e for s, e in zip(runs[::2], runs[1::2]))
                assert not fits
                continue
            assert off % align == 0 and off + n <= cap
            assert (owner[off:off + n] == 0).all()
            owner[off:off + n] = next_id
            live[next_id] = (off, n)
            next_id += 1
        used, _, _ = a.stats()
        assert used == int((owner != 0).sum())
    for key, (off, n) in list(live.items()):
        assert a.release(off, n) == _lib.OLC_OK
    assert a.stats() == (0, cap, 1)  # every free range merged back
    a.close()


def test_arena_rejects_double_free_and_bad_ranges(olc):
    a = _Arena(olc, 1000)
    off = a.alloc(100)
    assert a.release(off, 100) == _lib.OLC_OK
    assert a.release(off, 100) == _lib.OLC_ERR_ARG
    assert a.release(990, 20) == _lib.OLC_ERR_ARG
    assert a.alloc(1001) is None
    assert olc.olc_arena_alloc(a.h, 10, 3, C.byref(C.c_uint64())) == _lib.OLC_ERR_ARG  # align not a power of 2
    x = a.alloc(400)
    y = a.alloc(400)
    assert a.release(x + 1, 10) == _lib.OLC_ERR_ARG  # inside an allocation, not a whole range
    assert a.release(x, 400) == _lib.OLC_OK and a.release(y, 400) == _lib.OLC_OK
    assert a.stats() == (0, 1000, 1)
    a.close()


def test_arena_best_fit_keeps_large_runs_whole(olc):
    a = _Arena(olc, 1000)
    r = [a.alloc(100) for _ in range(10)]
    a.release(r[1], 100)              # hole of 100 at 100
    a.release(r[5], 100)
    a.release(r[6], 100)              # hole of 200 at 500
    assert a.alloc(100) == r[1]       # the small hole, not the large one
    assert a.alloc(200) == r[5]
    a.close()


# ---------------------------------------------------------------- scheduler
class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 0.001
        return self.t


def _req(rid, steps, rows=100, table=64, voxels=1000, **kw):
    return SimRequest(engine={"footprint": Footprint(rows, table, voxels), **kw}, sim=None, steps=steps,
                      request_id=rid)


def _pool(slots=8, rows=1000, table=1024, voxels=10_000, **kw):
    dev = FakePoolDevice(slots, rows, table, voxels)
    return ServingPool(dev, clock=Clock(), **kw), dev


def test_requests_finish_out_of_order_after_exactly_their_steps():
    pool, dev = _pool()
    steps = {0: 9, 1: 3, 2: 6, 3: 1}
    for rid, n in steps.items():
        pool.submit(_req(rid, n))
    res = pool.drain()
    assert [r.request_id for r in res] == [3, 1, 2, 0]
    for r in res:
        assert r.status == "done" and r.steps == steps[r.request_id]
        # all four were admitted before the first step, so each finished at its own step count
        assert r.metrics["steps_at_finish"] == steps[r.request_id]
    assert dev.steps == 9
    assert not dev.slots  # every slot and arena range returned
    # a step collects reductions only when a member finishes in it
    assert [c for kind, *c in dev.log if kind == "step"] == [[s in (1, 3, 6, 9)] for s in range(1, 10)]


def test_admission_waits_for_free_memory_then_backfills():
    pool, dev = _pool(voxels=10_000)
    pool.submit(_req(0, 5, voxels=6000))
    pool.submit(_req(1, 2, voxels=6000))   # does not fit beside request 0
    pool.submit(_req(2, 2, voxels=3000))   # fits: admitted ahead of 1 (backfill)
    pool.step()
    assert set(pool.residents) == {0, 2}
    assert [r.request_id for r in pool.queue] == [1]
    res = pool.drain()
    admitted = [rid for kind, rid, *_ in (e for e in dev.log if e[0] == "admit")]
    assert admitted == [0, 2, 1]
    assert {r.request_id: r.status for r in res} == {0: "done", 1: "done", 2: "done"}
    # request 1 joined after request 0 retired (5 steps), then ran its 2
    assert pool.results[1].metrics["steps_at_finish"] == 7


def test_without_backfill_the_queue_is_strict_fifo():
    pool, dev = _pool(voxels=10_000, backfill=False)
    pool.submit(_req(0, 5, voxels=6000))
    pool.submit(_req(1, 2, voxels=6000))
    pool.submit(_req(2, 2, voxels=3000))
    pool.step()
    assert set(pool.residents) == {0}
    pool.drain()
    admitted = [e[1] for e in dev.log if e[0] == "admit"]
    assert admitted == [0, 1, 2]


def test_rows_are_reserved_by_max_agents():
    pool, dev = _pool(rows=1000)
    pool.submit(_req(0, 3, rows=700))
    pool.submit(_req(1, 3, rows=400))
    pool.step()
    assert set(pool.residents) == {0} and pool.rows_reserved == 700
    pool.drain()
    assert pool.rows_reserved == 0
    assert pool.results[1].status == "done"


def test_malformed_and_oversized_requests_are_rejected_at_submission():
    pool, dev = _pool(voxels=10_000)
    pool.submit(_req(0, 0))
    pool.submit(_req(1, 3, malformed=True))
    pool.submit(_req(2, 3, voxels=20_000))
    pool.submit(_req(3, 3))
    res = pool.drain()
    assert pool.results[0].status == "rejected" and "steps" in pool.results[0].error
    assert pool.results[1].status == "rejected" and "malformed" in pool.results[1].error
    assert pool.results[2].status == "rejected" and "pool holds" in pool.results[2].error
    assert [r.request_id for r in res] == [3] and res[0].status == "done"


def test_injected_out_of_memory_delays_admission():
    faults = FaultInjector(oom={1: 3})
    pool, dev = _pool(faults=faults)
    pool.submit(_req(0, 10))
    pool.submit(_req(1, 2))
    for _ in range(3):
        pool.step()
        assert 1 not in pool.residents
    pool.step()
    assert 1 in pool.residents
    pool.drain()
    assert faults.events == [("oom", 1)] * 3
    assert pool.results[1].status == "done"
    assert pool.results[1].metrics["steps_at_finish"] == 5  # admitted before step 4, ran 2 steps


def test_injected_admission_failure_fails_only_that_request():
    faults = FaultInjector(fail={1})
    pool, dev = _pool(faults=faults)
    for rid in range(3):
        pool.submit(_req(rid, 2))
    pool.drain()
    assert pool.results[1].status == "failed" and "injected" in pool.results[1].error
    assert pool.results[0].status == "done" and pool.results[2].status == "done"
    assert not dev.slots


def test_an_empty_pool_that_keeps_refusing_rejects_the_request():
    faults = FaultInjector(oom={0: 10 ** 6})
    pool, dev = _pool(faults=faults)
    pool.submit(_req(0, 2))
    pool.submit(_req(1, 2))
    pool.drain()
    assert pool.results[0].status == "rejected"
    assert pool.results[1].status == "done"


def test_cancel_queued_and_resident_requests():
    pool, dev = _pool(slots=1)
    pool.submit(_req(0, 10))
    pool.submit(_req(1, 10))
    pool.step()
    assert set(pool.residents) == {0}
    assert pool.cancel(1)                  # queued
    assert pool.results[1].status == "cancelled"
    pool.step()
    assert pool.cancel(0)                  # resident: its slot is retired between steps
    assert pool.results[0].status == "cancelled" and pool.results[0].steps == 2
    assert not dev.slots and pool.rows_reserved == 0
    assert not pool.cancel(0)
    pool.submit(_req(2, 1))
    pool.drain()
    assert pool.results[2].status == "done"


def test_serve_replays_arrivals_and_measures_time_to_completion():
    pool, dev = _pool(slots=2)
    arrivals = [(0.0, lambda: _req(-1, 3)), (0.002, lambda: _req(-1, 1)), (0.004, lambda: _req(-1, 2)),
                (0.02, lambda: _req(-1, 1))]
    res = pool.serve(arrivals)
    assert sorted(r.request_id for r in res) == [0, 1, 2, 3]
    for r in res:
        assert r.status == "done"
        assert r.ttc is not None and r.ttc > 0
        assert r.admitted >= r.arrival
    assert pool.max_resident <= 2


def test_plan_arenas_follows_the_mix():
    mix = [Footprint(1000, 4096, 32 ** 3), Footprint(30_000, 262_144, 128 ** 3)]
    plan = plan_arenas(8 << 30, mix, n_cols=8, storages=[0, 0], sinks=[True, False])
    rows, vox, tab = plan["max_rows"], plan["field_voxels"], plan["table_entries"]
    assert rows / vox == pytest.approx(31_000 / (32 ** 3 + 128 ** 3), rel=1e-3)
    assert tab / vox == pytest.approx((4096 + 262_144) / (32 ** 3 + 128 ** 3), rel=1e-3)
    from oncolytica_b200.serving import row_bytes, voxel_bytes
    used = rows * row_bytes(8) + vox * voxel_bytes([0, 0], [True, False]) + tab * 8
    assert used == pytest.approx(8 << 30, rel=1e-3)


def test_serve_with_prefetching_workers():
    pool, dev = _pool(slots=3)
    built = []

    def make(rid, steps):
        def f():
            built.append(rid)
            return _req(rid, steps)
        return f

    arrivals = [(0.001 * k, make(k, 1 + k % 4)) for k in range(12)]
    res = pool.serve(arrivals, prefetch=0.05, workers=2)
    assert sorted(r.request_id for r in res) == list(range(12))
    assert all(r.status == "done" for r in res)
    assert sorted(built) == list(range(12))
