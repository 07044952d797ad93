"""Host side of the device-status checks (no GPU): the StatusWatch cadence
and policies against a fake status word, and the serving pool failing its
residents when the device status gains bits (FakePoolDevice)."""
from __future__ import annotations

import warnings

import pytest

from oncolytica_b200 import _lib
from oncolytica_b200.serving import FakePoolDevice, Footprint, ServingPool, SimRequest


class FakeWord:
    def __init__(self) -> None:
        self.bits = 0
        self.reads = 0

    def __call__(self) -> int:
        self.reads += 1
        return self.bits


def test_watch_reads_every_k_steps_and_after_synced_steps():
    w = FakeWord()
    sw = _lib.StatusWatch(w, "test", every=4)
    assert list(sw.chunks(10)) == [4, 4, 2]
    for k in sw.chunks(10):
        sw.after(k)
    assert w.reads == 2 and sw.since == 2
    assert list(sw.chunks(3)) == [2, 1]  # the next check point comes after two more steps
    sw.after(1, synced=True)
    assert w.reads == 3 and sw.since == 0


def test_watch_raises_each_new_bit_once():
    w = FakeWord()
    sw = _lib.StatusWatch(w, "test", every=1)
    sw.after(1)
    w.bits = _lib.OLC_STATUS_CAPACITY
    with pytest.raises(_lib.DeviceStatusError) as ei:
        sw.after(1)
    assert ei.value.code == _lib.OLC_ERR_CAPACITY and "capacity" in str(ei.value)
    sw.after(1)  # already reported
    w.bits |= _lib.OLC_STATUS_TIMEOUT
    with pytest.raises(_lib.DeviceStatusError) as ei:
        sw.after(1)
    assert ei.value.code == _lib.OLC_ERR_TIMEOUT and ei.value.new_bits == _lib.OLC_STATUS_TIMEOUT


def test_watch_policies():
    w = FakeWord()
    w.bits = _lib.OLC_STATUS_MULTI_DIVIDE
    sw = _lib.StatusWatch(w, "test", every=1, policy="warn")
    with warnings.catch_warnings(record=True) as rec:
        warnings.simplefilter("always")
        sw.after(1)
    assert len(rec) == 1 and "divide" in str(rec[0].message)
    ig = _lib.StatusWatch(w, "test", every=1, policy="ignore")
    ig.after(5)
    assert list(ig.chunks(7)) == [7]
    assert _lib.status_names(0) == "clean"
    assert "unknown" in _lib.status_names(0x100)


def _req(rows, steps):
    return SimRequest({"footprint": Footprint(rows, 10, 100)}, None, steps)


def test_pool_fails_residents_when_the_device_status_gains_bits():
    dev = FakePoolDevice(max_slots=4, max_rows=1000, table_entries=100, field_voxels=1000)
    pool = ServingPool(dev, depth=1)
    pool.status_every = 2
    a, b = pool.submit(_req(100, 10)), pool.submit(_req(100, 3))
    pool.step()
    dev.status_bits = _lib.OLC_STATUS_TIMEOUT  # a bounded wait gave up during these steps
    pool.step()
    # both residents were on the device when the bit appeared: both fail
    assert pool.results[a].status == "failed" and "timeout" in pool.results[a].error
    assert pool.results[b].status == "failed"
    assert not pool.residents and not dev.slots
    # later requests run (the bit is reported once)
    c = pool.submit(_req(100, 2))
    pool.drain()
    assert pool.results[c].status == "done"


# ---------------------------------------------------------------- queued readbacks (no GPU)

class _FakeReadbackLib:
    """olc_step / olc_queue_readback of a handle whose step k (1-based) leaves
    metric word k and status bits `status_at[k]`."""

    def __init__(self):
        self.steps = 0
        self.queued = {}
        self.status_at = {}

    def olc_step(self, handle, n, collect, stream):
        self.steps += n
        return _lib.OLC_OK

    def olc_queue_readback(self, handle, stream, ticket_ref):
        t = len(self.queued) + 1
        self.queued[t] = self.steps
        ticket_ref._obj.value = t
        return _lib.OLC_OK


def _fake_backend(every=64):
    import numpy as np
    from types import SimpleNamespace

    from oncolytica_b200.backend import CudaBackend

    be = CudaBackend.__new__(CudaBackend)
    lib = _FakeReadbackLib()
    be.lib, be.handle, be._stream = lib, None, lambda: None
    be.layout = SimpleNamespace(metrics={"live": (0, "i32")})
    be.engine = SimpleNamespace(_metrics=SimpleNamespace(live=0), status_check_every=every, on_device_status="raise")
    be._pending, be._applied_ticket, be._last_reductions = [], 0, None
    be.status = _lib.StatusWatch(lambda: 0, "test", every=every)

    def take(ticket):
        step = lib.queued[ticket]
        c = _lib.OlcCounters()
        c.status = lib.status_at.get(step, 0)
        c.steps = step
        return np.array([step], dtype=np.uint32), c

    be._take_readback = take
    be._check = lambda rc: None
    return be, lib


def test_queued_readbacks_keep_the_newest_metrics():
    be, lib = _fake_backend()
    h1 = be.run_steps(1, collect_metrics=True, wait=False)
    h2 = be.run_steps(1, collect_metrics=True, wait=False)
    assert len(be._pending) == 2
    assert h2.result() == {"live": 2} and be.engine._metrics.live == 2
    # an older step's result is still its own, and does not replace the newer one
    assert h1.result() == {"live": 1} and be.engine._metrics.live == 2
    assert h1.counters["steps"] == 1 and not be._pending
    assert be.run_steps(1, collect_metrics=True) is None and be.engine._metrics.live == 3


def test_queued_readbacks_never_outrun_the_slots():
    be, lib = _fake_backend()
    handles = [be.run_steps(1, collect_metrics=True, wait=False) for _ in range(6)]
    # every queue beyond the slots takes the oldest first, so no ticket is overwritten
    assert len(be._pending) <= _lib.READBACK_SLOTS - 1
    assert [h._values for h in handles[:3]] == [{"live": 1}, {"live": 2}, {"live": 3}]
    be.resolve_pending()
    assert [h.result()["live"] for h in handles] == [1, 2, 3, 4, 5, 6] and be.engine._metrics.live == 6


def test_queued_readback_reports_status_bits():
    be, lib = _fake_backend()
    lib.status_at[2] = _lib.OLC_STATUS_CAPACITY
    be.run_steps(1, collect_metrics=True)
    h = be.run_steps(1, collect_metrics=True, wait=False)
    with pytest.raises(_lib.DeviceStatusError):
        h.result()
    assert be.engine._metrics.live == 2  # the values still arrived
    be.run_steps(1, collect_metrics=True)  # the bit was reported once
