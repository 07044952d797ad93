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
