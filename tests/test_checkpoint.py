"""Checkpoints: the bundle record layout against the reference's own
serializer (a fixture it generated, CPU), and resuming from state_dict() or a
bundle bit for bit (GPU)."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

from oncolytica_b200 import bundle


def test_record_layout_matches_the_reference_serializer():
    with open(os.path.join(GOLDEN, "struct_layouts.json")) as fh:
        cases = json.load(fh)["cases"]
    for c in cases:
        fields = [tuple(f) for f in c["fields"]]
        order = bundle.pack_order(fields)
        assert [list(f) for f in order] == c["order"]
        layout, stride = bundle.struct_layout(order)
        assert {k: off for k, (_, off) in layout.items()} == c["offsets"]
        assert stride == c["stride"]


def test_records_round_trip():
    layout, stride = bundle.struct_layout(bundle.pack_order([("_rng_state", "u32"), ("pos", "vec3<f32>"),
                                                             ("state", "i32"), ("r", "f32")]))
    rng = np.random.default_rng(0)
    n, cap = 37, 50
    cols = {"pos.x": rng.random(n, np.float32), "pos.y": rng.random(n, np.float32),
            "pos.z": rng.random(n, np.float32), "state": rng.integers(0, 4, n).astype(np.int32),
            "r": rng.random(n, np.float32), "_rng_state": rng.integers(1, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)}
    raw = bundle._pack_records(layout, stride, cap, cols, n)
    assert len(raw) == cap * stride
    back = bundle._unpack_records(raw, {k: {"type": t, "offset": o} for k, (t, o) in layout.items()}, stride, n)
    for k, v in cols.items():
        np.testing.assert_array_equal(back[k], v)


def _spec(storage):
    from oncolytica_b200 import workloads as W

    return W.scaled(W.SCALE, n_agents=3000, domain=120.0, ball_radius=35.0, field_dims=(32, 32, 32),
                    capacity=20_000, seed=9, uptake=2.0, death_k=0.3, init_drug=0.2, v_lo=1.9, v_hi=2.0,
                    storage=storage)


def _same_state(a: dict, b: dict):
    assert a["rows"] == b["rows"]
    np.testing.assert_array_equal(a["life"], b["life"])
    for k in a["cols"]:
        np.testing.assert_array_equal(a["cols"][k], b["cols"][k], err_msg=k)
    for group in ("fields", "sinks", "residuals"):
        for k, v in (a.get(group) or {}).items():
            if v is not None:
                np.testing.assert_array_equal(v, b[group][k], err_msg=f"{group}/{k}")


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["f32", "f16_sr"])
@pytest.mark.parametrize("route", ["state_dict", "bundle"])
def test_resume_continues_bit_for_bit(cuda, storage, route, tmp_path):
    from oncolytica_b200 import workloads as W

    spec = _spec(storage)
    a = W.build_engine(spec)
    a.run_steps(3)
    if route == "state_dict":
        sd = a.state_dict()
    else:
        a.export_bundle(str(tmp_path / "bundle"))
    a.run_steps(4)
    want = a._backend_impl.snapshot()
    steps_a = a._backend_impl.counters()
    m_a = a.get_engine_metrics()

    b = W.build_engine(spec)
    if route == "state_dict":
        b.load_state_dict(sd)
    else:
        b.import_bundle(str(tmp_path / "bundle"))
    b.run_steps(4)
    _same_state(want, b._backend_impl.snapshot())
    steps_b = b._backend_impl.counters()
    assert steps_b["steps"] == steps_a["steps"] and steps_b["agent_steps"] == steps_a["agent_steps"]
    assert b.get_engine_metrics() == m_a


@pytest.mark.gpu
def test_bundle_records_read_back_like_the_reference(cuda, tmp_path):
    """Without the resume record, import_bundle reads the AoS records through
    config.json's layout (the path a bundle the reference exported takes): the
    live agents and the O2 field come back as sync_to_host sees them."""
    from oncolytica_b200 import workloads as W

    spec = _spec("f32")
    a = W.build_engine(spec)
    a.run_steps(2)
    d = str(tmp_path / "plain")
    a.export_bundle(d, exact=False)
    assert not os.path.exists(os.path.join(d, "resume.npz"))
    with open(os.path.join(d, "config.json")) as fh:
        cfg = json.load(fh)
    assert cfg["layout"]["structs"]["cell"]["fields"]["pos"]["offset"] == 0
    a.sync_to_host()
    host = a.cells.columns()
    o2 = np.array(a.chemistry.column("o2"))

    b = W.build_engine(spec)
    b.import_bundle(d)
    b.sync_to_host()
    got = b.cells.columns()
    for k in ("pos.x", "pos.y", "pos.z", "radius", "volume", "state", "_rng_state"):
        np.testing.assert_array_equal(got[k], host[k], err_msg=k)
    np.testing.assert_array_equal(np.array(b.chemistry.column("o2")), o2)
