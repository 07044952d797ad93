"""The autotuner (oncolytica_b200.autotune) and the choices it makes.

Every kernel shape and variant it chooses between must give the same bits:
each stencil tile and contact walk of a solo engine, and each batched FP32
tile depth, are run from one initial state and compared with the defaults.
Tuning itself restores the engine's state (the run continues bit for bit as
if it had not been tuned), and a second tuning of the same shape comes from
the cache."""
from __future__ import annotations

import numpy as np
import pytest

from oncolytica_b200 import _lib, autotune
from oncolytica_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _spec(dense: bool = False):
    # dense: ~100 agents per 10 um bin
    return W.scaled(W.SCALE, n_agents=30_000, domain=320.0, ball_radius=40.0 if dense else 90.0,
                    field_dims=(64, 64, 64), capacity=150_000, seed=4, uptake=2.0, death_k=0.2, init_drug=0.1,
                    v_lo=1.85, v_hi=2.0)


def _same(a: dict, b: dict, what: str) -> None:
    assert a["rows"] == b["rows"], what
    np.testing.assert_array_equal(a["life"], b["life"], err_msg=what)
    for k in a["cols"]:
        np.testing.assert_array_equal(a["cols"][k], b["cols"][k], err_msg=f"{what} {k}")
    for k in a["fields"]:
        np.testing.assert_array_equal(a["fields"][k], b["fields"][k], err_msg=f"{what} {k}")


@pytest.mark.parametrize("tile", autotune.STENCIL_TILES)
@pytest.mark.parametrize("contact", autotune.CONTACT_VARIANTS)
def test_every_choice_gives_the_same_bits(cuda, tile, contact):
    spec = _spec()
    state = W.initial_state(spec)
    ref = W.build_engine(spec, state)
    ref.run_steps(3)
    eng = W.build_engine(spec, state)
    eng._backend_impl.set_tuning(stencil_tile=tile, contact_variant=contact)
    assert eng._backend_impl.get_tuning()["stencil_tile"] == tuple(tile)
    eng.run_steps(3)
    _same(eng._backend_impl.snapshot(), ref._backend_impl.snapshot(), f"tile {tile} contact {contact}")


@pytest.mark.parametrize("pair", [p for p in autotune.STENCIL_PAIRS if p[0]] + [(256, 7)])
def test_two_substeps_per_pass_give_the_same_bits(cuda, pair):
    spec = _spec()
    state = W.initial_state(spec)
    ref = W.build_engine(spec, state)
    ref.run_steps(3)
    eng = W.build_engine(spec, state)
    eng._backend_impl.set_tuning(stencil_pair=pair)
    assert eng._backend_impl.get_tuning()["stencil_pair"] == tuple(pair)
    eng.run_steps(3)
    _same(eng._backend_impl.snapshot(), ref._backend_impl.snapshot(), f"pair {pair}")


@pytest.mark.parametrize("keep", [k for k in autotune.L2_KEEP if k] + [100])
def test_l2_resident_slab_gives_the_same_bits(cuda, keep):
    spec = _spec()
    state = W.initial_state(spec)
    ref = W.build_engine(spec, state)
    ref.run_steps(3)
    eng = W.build_engine(spec, state)
    eng._backend_impl.set_tuning(l2_keep_pct=keep)
    assert eng._backend_impl.get_tuning()["l2_keep_pct"] == keep
    eng.run_steps(3)
    _same(eng._backend_impl.snapshot(), ref._backend_impl.snapshot(), f"l2 keep {keep}")


@pytest.mark.parametrize("contact", autotune.CONTACT_VARIANTS)
def test_contact_variants_agree_on_a_dense_population(cuda, contact):
    spec = _spec(dense=True)
    state = W.initial_state(spec)
    ref = W.build_engine(spec, state)
    ref.run_steps(2)
    eng = W.build_engine(spec, state)
    eng._backend_impl.set_tuning(contact_variant=contact)
    eng.run_steps(2)
    _same(eng._backend_impl.snapshot(), ref._backend_impl.snapshot(), f"dense, contact {contact}")


def test_tuning_restores_the_run_and_caches(cuda, tmp_path, monkeypatch):
    monkeypatch.setattr(autotune, "CACHE", str(tmp_path / "tuning.json"))
    spec = _spec()
    state = W.initial_state(spec)
    ref = W.build_engine(spec, state)
    ref.run_steps(2)
    eng = W.build_engine(spec, state)
    eng.run_steps(1)
    rec = autotune.tune_engine(eng, steps=2)
    assert not rec["cached"]
    assert tuple(rec["tuning"]["stencil_tile"]) in autotune.STENCIL_TILES
    assert rec["tuning"]["contact_variant"] in autotune.CONTACT_VARIANTS
    assert {"substeps", "substep_pairs", "contact"} <= set(rec["measured_ms"])
    assert tuple(rec["tuning"]["stencil_pair"]) in autotune.STENCIL_PAIRS
    assert eng._backend_impl.get_tuning()["stencil_tile"] == tuple(rec["tuning"]["stencil_tile"])
    assert eng._step == 1 and eng._backend_impl.counters()["steps"] == 1
    eng.run_steps(1)
    _same(eng._backend_impl.snapshot(), ref._backend_impl.snapshot(), "after tuning")
    other = W.build_engine(spec, state)
    assert autotune.tune_engine(other, steps=2)["cached"]
    assert other._backend_impl.get_tuning() == eng._backend_impl.get_tuning()


def test_tuning_rejects_unknown_shapes(cuda):
    eng = W.build_engine(_spec())
    with pytest.raises(_lib.OlcError):
        eng._backend_impl.set_tuning(stencil_tile=(4, 4))
    with pytest.raises(_lib.OlcError):
        eng._backend_impl.set_tuning(batch_tile_depth=12)
    with pytest.raises(_lib.OlcError):
        eng._backend_impl.set_tuning(stencil_pair=(384, 0))
    with pytest.raises(_lib.OlcError):
        eng._backend_impl.set_tuning(l2_keep_pct=120)


def test_batch_tile_depths_give_the_same_bits(cuda, tmp_path, monkeypatch):
    monkeypatch.setattr(autotune, "CACHE", str(tmp_path / "tuning.json"))
    specs = W.batched_specs(6, seed=3)
    states = [W.initial_state(sp) for sp in specs]
    ref = W.build_batch(specs, states)
    ref.run_steps(3)
    b = W.build_batch(specs, states)
    b.set_tile_depths([8, 32, 16, 32, 8, 0])
    b.run_steps(3)
    for k in range(len(specs)):
        _same(b.snapshot(k), ref.snapshot(k), f"member {k}")
    rec = autotune.tune_batch(lambda: W.build_batch(specs, states), steps=1)
    sizes = {"x".join(str(v) for v in sp.field_dims) for sp in specs}
    assert set(rec["depths"]) == sizes and all(d in autotune.BATCH_DEPTHS for d in rec["depths"].values())
    per = autotune.apply_batch(b, rec["depths"])
    assert len(per) == len(specs)
    assert autotune.tune_batch(lambda: W.build_batch(specs, states), steps=1)["cached"]
