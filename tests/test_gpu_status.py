"""Device status: the bounded waits give up and report, and the host raises.

Every device wait in the library is bounded: the decoupled look-back of the
sort and of the births (olc_lookback) and the TMA tile wait of the stencil
kernels (olc_mbar_wait_bounded).  olc_selftest_bounded_waits runs both against
words that are never published, with a short poll limit; the kernels must
return, record OLC_STATUS_TIMEOUT and leave the context usable.  The engine
reads the sticky status word every ``status_check_every`` steps and after
collected steps, and raises DeviceStatusError for bits it has not reported
(the reference drops overflowing children silently,
framework/src/oncolytica/gpu/compiler/translator/_stmt_translator.py:448).
"""
from __future__ import annotations

import ctypes as C
import warnings

import numpy as np
import pytest

import oncolytica_b200 as ol
from oncolytica_b200 import _lib

pytestmark = pytest.mark.gpu


def test_bounded_waits_give_up_and_report(cuda, olc):
    import torch

    out = (C.c_uint32 * 3)()
    _lib.check(olc.olc_selftest_bounded_waits(1000, C.byref(out), None))
    assert out[0] == _lib.OLC_STATUS_TIMEOUT, hex(out[0])  # look-back walk gave up
    assert out[1] == _lib.OLC_STATUS_TIMEOUT, hex(out[1])  # mbarrier wait gave up (and never completed)
    assert out[2] == 0  # the unpublished tile counted as an empty prefix
    # the context is intact: a sort through the same library still runs clean
    k = np.random.default_rng(1).integers(0, 1 << 16, size=50_000, dtype=np.uint64).astype(np.uint32)
    kin = torch.from_numpy(k.view(np.int32)).to(cuda)
    ko = torch.empty_like(kin)
    vo = torch.empty_like(kin)
    nbytes = olc.olc_sort_scratch_bytes(len(k), 16)
    scratch = torch.zeros(nbytes, dtype=torch.uint8, device=cuda)
    _lib.check(olc.olc_stage_sort_pairs(C.c_void_p(kin.data_ptr()), None, C.c_void_p(ko.data_ptr()),
                                        C.c_void_p(vo.data_ptr()), len(k), 16, C.c_void_p(scratch.data_ptr()),
                                        nbytes, None))
    torch.cuda.synchronize()
    off = olc.olc_sort_status_offset()
    assert int(scratch[off:off + 4].cpu().numpy().view(np.uint32)[0]) == 0
    np.testing.assert_array_equal(ko.cpu().numpy().view(np.uint32), np.sort(k, kind="stable"))


def test_selftest_rejects_bad_limits(cuda, olc):
    out = (C.c_uint32 * 3)()
    assert olc.olc_selftest_bounded_waits(0, C.byref(out), None) == _lib.OLC_ERR_ARG
    assert olc.olc_selftest_bounded_waits(1 << 20, C.byref(out), None) == _lib.OLC_ERR_ARG


class SCell(ol.Cell):
    pos: ol.vec3
    age: ol.i32 = 0


class SMetrics(ol.Metrics):
    n: ol.i32 = 0


class SParams(ol.Params):
    pass


class STissue(ol.Tissue):
    pass


class SChem(ol.Chemistry):
    c: ol.f32 = 0.0


class SplitSim(ol.Simulation[STissue, SChem, SCell, SMetrics, SParams]):
    @ol.cell_rule
    def split(self, cell: SCell):
        child: SCell = SCell(pos=cell.pos, age=0)
        cell.divide(child)

    @ol.metric_rule
    def count(self, cell: SCell, m: SMetrics):
        m.n += 1


def _overflowing_engine(policy: str):
    eng = ol.Engine(backend="cuda", max_agents=150)
    eng.setup_geometry((8, 8, 8), 1.0)
    eng.on_device_status = policy
    eng.cells.add_arrays(SCell, pos=np.full((100, 3), 4.0), age=np.zeros(100, np.int32))
    eng.load_model(SplitSim())
    return eng


def test_capacity_overflow_raises_on_the_collected_step(cuda):
    eng = _overflowing_engine("raise")
    with pytest.raises(_lib.DeviceStatusError) as ei:
        eng.run_step(collect_metrics=True)  # 100 children, room for 50
    assert ei.value.code == _lib.OLC_ERR_CAPACITY
    assert ei.value.new_bits == _lib.OLC_STATUS_CAPACITY
    assert eng._backend_impl.counters()["n_agents"] == 150
    # reported once: the next step (still overflowing) does not raise again
    eng.run_step(collect_metrics=True)


def test_capacity_overflow_is_found_within_the_check_interval(cuda):
    eng = _overflowing_engine("raise")
    eng.status_check_every = 4
    with pytest.raises(_lib.DeviceStatusError):
        eng.run_steps(4)  # no metrics: the fourth step's check finds the bit


def test_status_policies_warn_and_ignore(cuda):
    eng = _overflowing_engine("warn")
    with warnings.catch_warnings(record=True) as rec:
        warnings.simplefilter("always")
        eng.run_step(collect_metrics=True)
    assert any("capacity" in str(w.message) for w in rec)
    eng = _overflowing_engine("ignore")
    eng.run_step(collect_metrics=True)
    assert eng._backend_impl.counters()["status"] & _lib.OLC_STATUS_CAPACITY
