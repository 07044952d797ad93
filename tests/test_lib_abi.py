"""libolc.so loads, exports every entry point include/olc.h declares, and its
argument checks reject bad input before touching a GPU (CPU-only tests)."""
from __future__ import annotations

import ctypes as C
import os
import re

import pytest

from conftest import REPO

from oncolytica_b200 import _lib


def _declared_symbols() -> set[str]:
    text = open(os.path.join(REPO, "include", "olc.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(olc_[a-z_0-9]+)\s*\(", text))


def test_header_and_binding_agree():
    assert _declared_symbols() == set(_lib.EXPORTS)


def test_library_exports_every_declared_symbol(olc):
    for name in _declared_symbols():
        assert hasattr(olc, name), name


def test_struct_sizes_match_header_layout():
    assert C.sizeof(_lib.OlcGeom) == 4 * (3 + 1 + 3 + 1 + 3 + 3)
    assert C.sizeof(_lib.OlcCaps) == 4 * 9
    assert C.sizeof(_lib.OlcDiffusion) == 28
    assert C.sizeof(_lib.OlcContact) == 28
    assert C.sizeof(_lib.OlcTuning) == 4 * 7
    assert C.sizeof(_lib.OlcCounters) == 40
    assert C.sizeof(_lib.OlcProfile) == 16 + 6 * 8
    assert C.sizeof(_lib.OlcPoolConfig) == 4 + 12 + 8 + 8
    assert C.sizeof(_lib.OlcPoolUsage) == 8 + 6 * 8


def test_create_pool_rejects_bad_configs_without_a_gpu(olc):
    caps = _lib.OlcCaps(max_agents=1024, n_agent_fields=4, n_fields=1, state_field=-1)
    h = C.c_void_p()
    cfg = _lib.OlcPoolConfig(max_slots=0, table_entries=4096, field_voxels=4096)
    cfg.max_tissue_dims[:] = (16, 16, 16)
    assert olc.olc_create_pool(C.byref(cfg), C.byref(caps), C.byref(h)) == _lib.OLC_ERR_ARG
    cfg.max_slots = 1 << 20                     # 20 slot bits + 12 bin-key bits of 16^3 overflow 32
    cfg.max_tissue_dims[:] = (32, 32, 32)
    assert olc.olc_create_pool(C.byref(cfg), C.byref(caps), C.byref(h)) == _lib.OLC_ERR_ARG
    assert "32 key bits" in _lib.last_error()
    cfg.max_slots, cfg.field_voxels = 64, 0
    assert olc.olc_create_pool(C.byref(cfg), C.byref(caps), C.byref(h)) == _lib.OLC_ERR_ARG
    assert olc.olc_pool_admit(None, None, None, None, 0, None, None, None) == _lib.OLC_ERR_ARG


def test_version_string(olc):
    assert b"sm_100a" in olc.olc_version()


def test_sort_scratch_size_is_host_only(olc):
    small = olc.olc_sort_scratch_bytes(1000, 21)
    big = olc.olc_sort_scratch_bytes(1_000_000, 21)
    assert 0 < small < big
    assert olc.olc_sort_scratch_bytes(10, 0) == 0
    assert olc.olc_sort_scratch_bytes(10, 33) == 0


def test_bad_arguments_are_rejected_without_a_gpu(olc):
    g = _lib.OlcGeom()
    g.tissue_dims[:] = (3, 4, 4)  # odd: rejected (reference limit)
    g.tissue_voxel_size = 1.0
    rc = olc.olc_stage_keys(None, None, None, None, 0, C.byref(g), None, None)
    assert rc == _lib.OLC_ERR_ARG
    assert "even" in _lib.last_error()
    rc = olc.olc_stage_sort_pairs(None, None, None, None, 10, 0, None, 0, None)
    assert rc == _lib.OLC_ERR_ARG
    rc = olc.olc_stage_sort_pairs(None, None, None, None, 10, 21, None, 0, None)
    assert rc == _lib.OLC_ERR_ARG
    d = _lib.OlcDiffusion(diffusion=1.0, decay=0.0, boundary=0.0, substeps=1, has_sink=0)
    dims = (C.c_int32 * 3)(8, 8, 8)
    rc = olc.olc_stage_diffuse(C.c_void_p(16), C.c_void_p(16), None, C.byref(dims), 1.0, 1.0, C.byref(d), None)
    assert rc == _lib.OLC_ERR_ARG
    assert "unstable" in _lib.last_error()


def test_create_rejects_bad_geometry(olc):
    g = _lib.OlcGeom()
    g.tissue_dims[:] = (250, 10, 10)
    g.tissue_voxel_size = 1.0
    caps = _lib.OlcCaps(max_agents=16, n_agent_fields=3, n_fields=0, state_field=-1)
    h = C.c_void_p()
    assert olc.olc_create(C.byref(g), C.byref(caps), C.byref(h)) == _lib.OLC_ERR_ARG
    assert "240" in _lib.last_error()
