"""Stage parity on the GPU: each libolc stage entry point against the CPU
oracle on identical inputs.  Integer stages (RNG states, keys, sort, bin
table) must match bit for bit; floating-point stages that use only separately
rounded + - * / sqrt (diffusion, sink, contact) must match bit for bit too;
the random direction (cos/sin) within 2 ulp."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from conftest import GOLDEN

import oracle
from oncolytica_b200 import _lib

pytestmark = pytest.mark.gpu


def dptr(t):
    return C.c_void_p(t.data_ptr())


def to_dev(a: np.ndarray, cuda):
    import torch

    if a.dtype == np.uint32:
        return torch.from_numpy(a.view(np.int32).copy()).to(cuda)
    if a.dtype == np.uint8:
        return torch.from_numpy(a.copy()).to(cuda)
    return torch.from_numpy(np.ascontiguousarray(a).copy()).to(cuda)


def to_host(t, dtype=None) -> np.ndarray:
    import torch

    torch.cuda.synchronize()
    a = t.cpu().numpy()
    return a.view(dtype) if dtype is not None else a


def geom(dims, vs, lo=(0, 0, 0), hi=None) -> _lib.OlcGeom:
    g = _lib.OlcGeom()
    g.tissue_dims[:] = dims
    g.tissue_voxel_size = vs
    g.chem_dims[:] = (0, 0, 0)
    g.chem_voxel_size = 1.0
    g.domain_lo[:] = lo
    g.domain_hi[:] = hi if hi is not None else tuple(d * vs for d in dims)
    return g


# ------------------------------------------------------------------ RNG

def test_rng_bit_exact(cuda, olc):
    import torch

    n, draws = 5000, 7
    states = oracle.seed_rng(11, n)
    s_ref, d_ref, dir_ref = oracle.rng_batch(states, draws, dirs=True)
    st = to_dev(states, cuda)
    out = torch.empty(n * draws, dtype=torch.float32, device=cuda)
    dirs = torch.empty(n * 3, dtype=torch.float32, device=cuda)
    _lib.check(olc.olc_stage_rng(dptr(st), n, draws, dptr(out), dptr(dirs), None))
    np.testing.assert_array_equal(to_host(st, np.uint32), s_ref)
    np.testing.assert_array_equal(to_host(out).reshape(n, draws), d_ref)
    got = to_host(dirs).reshape(n, 3)
    # cos/sin are library functions on both sides: allow 2 ulp
    np.testing.assert_array_max_ulp(got, dir_ref, maxulp=2)


# ------------------------------------------------------------------ keys

def test_keys_sort_contract_golden(cuda, olc):
    import torch

    d = np.load(os.path.join(GOLDEN, "sort_contract.npz"))
    pos = d["pos"]
    n = len(pos)
    x, y, z = (to_dev(np.ascontiguousarray(pos[:, k]), cuda) for k in range(3))
    keys = torch.empty(n, dtype=torch.int32, device=cuda)
    g = geom(tuple(int(v) for v in d["dims"]), float(d["vs"]))
    _lib.check(olc.olc_stage_keys(dptr(x), dptr(y), dptr(z), None, n, C.byref(g), dptr(keys), None))
    np.testing.assert_array_equal(to_host(keys, np.uint32), d["keys"])


def test_keys_edge_positions_and_dead(cuda, olc):
    import torch

    rng = np.random.default_rng(5)
    dims, vs = (26, 26, 26), 10.0
    n = 20000
    pos = rng.uniform(-20.0, 280.0, size=(n, 3)).astype(np.float32)
    pos[:10] = [[0, 0, 0], [259.99998, 0, 0], [260, 260, 260], [-0.0, 5, 5], [9.999999, 10, 10.000001],
                [np.nan, 1, 1], [np.inf, -np.inf, 3], [1e30, -1e30, 0], [130, 130, 130], [255.0, 1.0, 2.0]]
    dead = (rng.random(n) < 0.1).astype(np.uint8)
    ref = oracle.keys(pos, dims, vs, dead)
    x, y, z = (to_dev(np.ascontiguousarray(pos[:, k]), cuda) for k in range(3))
    dd = to_dev(dead, cuda)
    keys = torch.empty(n, dtype=torch.int32, device=cuda)
    g = geom(dims, vs)
    _lib.check(olc.olc_stage_keys(dptr(x), dptr(y), dptr(z), dptr(dd), n, C.byref(g), dptr(keys), None))
    got = to_host(keys, np.uint32)
    np.testing.assert_array_equal(got, ref)
    assert np.all(got[dead == 1] == oracle.tissue_key(*dims))


# ------------------------------------------------------------------ sort

def _gpu_sort(olc, cuda, k: np.ndarray, bits: int, v: np.ndarray | None = None):
    import torch

    n = len(k)
    kin = to_dev(k, cuda)
    vin = to_dev(v, cuda) if v is not None else None
    kout = torch.empty(max(n, 1), dtype=torch.int32, device=cuda)
    vout = torch.empty(max(n, 1), dtype=torch.int32, device=cuda)
    nbytes = olc.olc_sort_scratch_bytes(n, bits)
    scratch = torch.empty(nbytes, dtype=torch.uint8, device=cuda)
    _lib.check(olc.olc_stage_sort_pairs(dptr(kin), dptr(vin) if vin is not None else None, dptr(kout), dptr(vout),
                                        n, bits, dptr(scratch), nbytes, None))
    return to_host(kout, np.uint32)[:n], to_host(vout, np.uint32)[:n]


@pytest.mark.parametrize("n,bits", [(1, 8), (100, 8), (4095, 13), (4096, 16), (4097, 21), (65537, 24),
                                    (1_000_003, 21), (300_000, 32), (2_500_000, 24)])
def test_sort_pairs_bit_exact(cuda, olc, n, bits):
    rng = np.random.default_rng(n + bits)
    hi = (1 << bits) if bits < 32 else (1 << 32)
    # few distinct keys for small widths: exercises stability heavily
    k = rng.integers(0, min(hi, max(2, n // 7)), size=n, dtype=np.uint64).astype(np.uint32)
    if bits == 32:
        k = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
    ko, vo = _gpu_sort(olc, cuda, k, bits)
    rk, rv = oracle.sort_pairs(k)
    np.testing.assert_array_equal(ko, rk)
    np.testing.assert_array_equal(vo, rv)


def test_sort_pairs_with_values_and_nearly_sorted_keys(cuda, olc):
    rng = np.random.default_rng(9)
    n = 777_777
    k = np.sort(rng.integers(0, 2_064_833, size=n)).astype(np.uint32)
    swap = rng.integers(0, n - 1, size=n // 50)
    k[swap], k[swap + 1] = k[swap + 1].copy(), k[swap].copy()
    v = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
    ko, vo = _gpu_sort(olc, cuda, k, 21, v)
    rk, rv = oracle.sort_pairs(k, v)
    np.testing.assert_array_equal(ko, rk)
    np.testing.assert_array_equal(vo, rv)


def test_sort_contract_golden_ids(cuda, olc):
    """framework/tests/test_gpu.py:54-61 on the GPU sort: per-key id sets."""
    d = np.load(os.path.join(GOLDEN, "sort_contract.npz"))
    keys = d["keys"]
    bits = int(np.ceil(np.log2(int(d["n_table"]))))
    ko, vo = _gpu_sort(olc, cuda, keys, bits)
    assert sorted(vo.tolist()) == list(range(len(keys)))
    np.testing.assert_array_equal(keys[vo], ko)
    rk, rv = oracle.sort_pairs(keys)
    np.testing.assert_array_equal(vo, rv)


def test_sort_is_deterministic(cuda, olc):
    rng = np.random.default_rng(4)
    k = rng.integers(0, 5000, size=300_001).astype(np.uint32)
    runs = [_gpu_sort(olc, cuda, k, 13) for _ in range(3)]
    for ko, vo in runs[1:]:
        np.testing.assert_array_equal(ko, runs[0][0])
        np.testing.assert_array_equal(vo, runs[0][1])


# ------------------------------------------------------------------ bin table

def test_bin_ranges_bit_exact(cuda, olc):
    import torch

    rng = np.random.default_rng(2)
    n_table = 32313
    k = np.sort(rng.integers(0, n_table + 5, size=200_000)).astype(np.uint32)
    kd = to_dev(k, cuda)
    rg = torch.empty(2 * n_table, dtype=torch.int32, device=cuda)
    _lib.check(olc.olc_stage_bin_ranges(dptr(kd), len(k), n_table, dptr(rg), None))
    np.testing.assert_array_equal(to_host(rg, np.uint32), oracle.bin_ranges(k, n_table))


# ------------------------------------------------------------------ diffusion

@pytest.mark.parametrize("dims,substeps,decay,with_sink", [((32, 24, 20), 5, 0.0, True),
                                                          ((64, 64, 64), 8, 0.1, False),
                                                          ((33, 17, 9), 3, 0.05, True)])
def test_diffuse_bit_exact(cuda, olc, dims, substeps, decay, with_sink):
    import torch

    rng = np.random.default_rng(sum(dims))
    nx, ny, nz = dims
    f = rng.random((nz, ny, nx), dtype=np.float32)
    sink = None
    if with_sink:
        sink = np.zeros_like(f)
        m = rng.random(f.shape) < 0.1
        sink[m] = rng.random(int(m.sum())).astype(np.float32) * 0.5
    dx, dt, D = 4.0, 0.1, 2000.0
    S = substeps
    D = min(D, (1.0 / 6.0) * dx * dx * S / dt * 0.999)
    ref = oracle.diffuse(f, sink, dx=dx, dt=dt, D=D, decay=decay, boundary=0.7, substeps=S)
    fd = to_dev(f, cuda)
    tmp = torch.empty_like(fd)
    sd = to_dev(sink, cuda) if sink is not None else None
    spec = _lib.OlcDiffusion(diffusion=D, decay=decay, boundary=0.7, substeps=S, has_sink=int(with_sink))
    dims_c = (C.c_int32 * 3)(nx, ny, nz)
    _lib.check(olc.olc_stage_diffuse(dptr(fd), dptr(tmp), dptr(sd) if sd is not None else None, C.byref(dims_c),
                                     dx, dt, C.byref(spec), None))
    np.testing.assert_array_equal(to_host(fd), ref)
    if sd is not None:
        assert float(to_host(sd).max()) == 0.0


# (stencil tile, (threads, planes) of the two-substeps-per-pass kernel): every
# single-pass tile, and the pair kernel at each CTA size, with the planes per
# CTA chosen by occupancy (0) and forced small and odd (ragged z chunks)
STENCIL_CHOICES = ([(tile, (0, 0), 0) for tile in ((8, 8), (16, 8), (8, 16), (16, 4))]
                   + [((8, 8), pair, 0) for pair in ((1024, 0), (512, 0), (256, 0), (128, 0), (1024, 9), (512, 13),
                                                     (256, 5), (128, 8))]
                   + [((16, 4), (256, 3), 0)]
                   + [((8, 8), (0, 0), keep) for keep in (30, 60, 100)] + [((16, 8), (0, 0), 45)])


@pytest.mark.parametrize("substeps", [7, 8])
@pytest.mark.parametrize("dims", [(68, 41, 37), (128, 34, 19), (64, 64, 70), (256, 30, 21), (66, 23, 17)])
def test_diffuse_every_stencil_choice_bit_exact(cuda, olc, dims, substeps):
    """Every single-pass tile (with and without a slab of planes kept in L2
    by eviction hints) and every two-substeps-per-pass shape
    (olc_stage_diffuse_tuned) gives the oracle's bits: odd and even substep
    counts (a pair kernel's odd substep is a single pass), ragged tiles and z
    chunks in every direction, rows of 256 voxels where the smallest pair CTA
    does not apply, and an x extent the TMA cannot map (66: the plain
    register-column kernel runs for every choice)."""
    import torch

    rng = np.random.default_rng(77 + substeps)
    nx, ny, nz = dims
    f = rng.random((nz, ny, nx), dtype=np.float32)
    spec = _lib.OlcDiffusion(diffusion=1.0, decay=0.02, boundary=0.4, substeps=substeps, has_sink=0)
    dims_c = (C.c_int32 * 3)(nx, ny, nz)
    ref = oracle.diffuse(f, None, dx=1.0, dt=0.5 * substeps / 7, D=1.0, decay=0.02, boundary=0.4, substeps=substeps)
    for tile, pair, keep in STENCIL_CHOICES:
        t = _lib.OlcTuning(tile[0], tile[1], 0, 16, pair[0], pair[1], keep)
        fd = to_dev(f, cuda)
        tmp = torch.empty_like(fd)
        _lib.check(olc.olc_stage_diffuse_tuned(dptr(fd), dptr(tmp), None, C.byref(dims_c), 1.0, 0.5 * substeps / 7,
                                               C.byref(spec), C.byref(t), None))
        np.testing.assert_array_equal(to_host(fd), ref, err_msg=f"tile {tile} pair {pair} keep {keep}")


def test_diffuse_tuned_rejects_unknown_shapes(cuda, olc):
    import torch

    f = torch.zeros(16 * 16 * 16, dtype=torch.float32, device="cuda")
    tmp = torch.empty_like(f)
    spec = _lib.OlcDiffusion(diffusion=1.0, decay=0.0, boundary=0.4, substeps=2, has_sink=0)
    dims_c = (C.c_int32 * 3)(16, 16, 16)
    for t in (_lib.OlcTuning(8, 8, 0, 16, 64, 0, 0), _lib.OlcTuning(4, 4, 0, 16, 0, 0, 0),
              _lib.OlcTuning(8, 8, 0, 16, 256, -1, 0), _lib.OlcTuning(8, 8, 0, 16, 0, 0, 101)):
        rc = olc.olc_stage_diffuse_tuned(dptr(f), dptr(tmp), None, C.byref(dims_c), 1.0, 0.5, C.byref(spec),
                                         C.byref(t), None)
        assert rc == _lib.OLC_ERR_ARG


def test_diffuse_pinned_voxels_bit_exact(cuda, olc):
    """Pinned voxels (the engine's vessel mask): a cylinder of voxels held at
    1.0 after every substep, on the TMA path, against orc_diffuse_pinned."""
    import torch

    rng = np.random.default_rng(12)
    nx, ny, nz = 64, 40, 48
    f = rng.random((nz, ny, nx), dtype=np.float32) * np.float32(0.5)
    zz, xx = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
    inside = (xx + 0.5 - 30.0) ** 2 + (zz + 0.5 - 20.0) ** 2 <= 6.0 ** 2
    z, x = np.nonzero(inside)
    pins = np.sort(((z[:, None] * ny + np.arange(ny)[None, :]) * nx + x[:, None]).ravel()).astype(np.uint32)
    spec = _lib.OlcDiffusion(diffusion=1.0, decay=0.02, boundary=0.4, substeps=7, has_sink=0, storage=0)
    fd = to_dev(f.ravel(), cuda)
    tmp = torch.zeros_like(fd)
    pd = to_dev(pins, cuda)
    dims_c = (C.c_int32 * 3)(nx, ny, nz)
    _lib.check(olc.olc_stage_diffuse_pinned(dptr(fd), dptr(tmp), None, C.byref(dims_c), 1.0, 0.5, C.byref(spec),
                                            dptr(pd), len(pins), 1.0, None))
    ref = oracle.diffuse_pinned(f, None, 1.0, 0.5, 1.0, 0.02, 0.4, 7, pins, 1.0)
    got = to_host(fd).reshape(nz, ny, nx)
    np.testing.assert_array_equal(got, ref)
    assert np.all(got.ravel()[pins] == 1.0)
    plain = oracle.diffuse(f, None, dx=1.0, dt=0.5, D=1.0, decay=0.02, boundary=0.4, substeps=7)
    assert np.abs(got - plain).max() > 0.1  # the vessel feeds its neighbourhood


# ------------------------------------------------------------------ contact

def test_contact_bit_exact(cuda, olc):
    import torch

    rng = np.random.default_rng(8)
    dims, vs = (20, 20, 20), 10.0
    n = 30000
    pos = rng.normal(100.0, 25.0, size=(n, 3)).astype(np.float32)
    pos = np.clip(pos, 0.0, 199.0).astype(np.float32)
    pos[5] = pos[6]  # a coincident pair
    radius = rng.uniform(4.0, 6.0, size=n).astype(np.float32)
    k = oracle.keys(pos, dims, vs)
    ks, perm = oracle.sort_pairs(k)
    n_table = oracle.tissue_key(*dims)
    ranges = oracle.bin_ranges(ks, n_table)
    posr = np.concatenate([pos[perm], radius[perm, None]], axis=1).astype(np.float32)
    posr[rng.random(n) < 0.02, 3] = -1.0  # a few dead rows
    params = dict(stiffness=1.0, mobility=10.0, max_disp=1.0, dt=0.1)
    lo, hi = (0.1, 0.1, 0.1), (199.9, 199.9, 199.9)
    ref = oracle.contact(posr, ranges, dims, vs, params["stiffness"], params["mobility"], params["max_disp"],
                         params["dt"], lo, hi)
    pr = to_dev(posr, cuda)
    rg = to_dev(ranges, cuda)
    x = to_dev(np.ascontiguousarray(posr[:, 0]), cuda)
    y = to_dev(np.ascontiguousarray(posr[:, 1]), cuda)
    z = to_dev(np.ascontiguousarray(posr[:, 2]), cuda)
    g = geom(dims, vs, lo=(0, 0, 0), hi=(200, 200, 200))
    spec = _lib.OlcContact(enabled=1, radius_field=-1, radius_const=0.0, stiffness=params["stiffness"],
                           mobility=params["mobility"], max_disp=params["max_disp"], margin=0.1)
    _lib.check(olc.olc_stage_contact(dptr(pr), dptr(rg), n, C.byref(g), C.byref(spec), params["dt"], dptr(x),
                                     dptr(y), dptr(z), None))
    got = np.stack([to_host(x), to_host(y), to_host(z)], axis=1)
    np.testing.assert_array_equal(got, ref)
    moved = np.any(got != posr[:, :3], axis=1)
    assert moved.sum() > n // 2


@pytest.mark.parametrize("variant", [_lib.OLC_CONTACT_FLAT, _lib.OLC_CONTACT_NESTED])
@pytest.mark.parametrize("case", ["sparse", "dense", "moved", "cluster"])
def test_contact_walks_bit_exact(cuda, olc, variant, case):
    """Every contact walk (olc_stage_contact_tuned) against orc_contact:
    a sparse population; a dense one; agents moved after the sort (a rule's displacement), whose current
    bin differs from the one they are sorted in; and a cluster of 50 agents
    in one bin of a sparse neighbourhood.  Coincident points and dead rows in
    each."""
    rng = np.random.default_rng(31)
    dims, vs = (20, 20, 20), 10.0
    n, sd = {"sparse": (30000, 25.0), "dense": (40000, 16.0), "moved": (30000, 20.0), "cluster": (8000, 40.0)}[case]
    pos = np.clip(rng.normal(100.0, sd, size=(n, 3)), 0.0, 199.0).astype(np.float32)
    if case == "cluster":
        pos[:50] = rng.uniform(100.5, 109.5, size=(50, 3)).astype(np.float32)
    pos[5] = pos[6]
    radius = rng.uniform(4.0, 6.0, size=n).astype(np.float32)
    k = oracle.keys(pos, dims, vs)
    ks, perm = oracle.sort_pairs(k)
    ranges = oracle.bin_ranges(ks, oracle.tissue_key(*dims))
    posr = np.concatenate([pos[perm], radius[perm, None]], axis=1).astype(np.float32)
    posr[rng.random(n) < 0.02, 3] = -1.0
    if case == "moved":
        m = rng.random(n) < 0.05
        posr[m, :3] = np.clip(posr[m, :3] + rng.normal(0.0, 6.0, size=(int(m.sum()), 3)), 0.0, 199.0)
    lo, hi = (0.1, 0.1, 0.1), (199.9, 199.9, 199.9)
    ref = oracle.contact(posr, ranges, dims, vs, 1.0, 10.0, 1.0, 0.1, lo, hi)
    pr, rg = to_dev(posr, cuda), to_dev(ranges, cuda)
    x, y, z = (to_dev(np.ascontiguousarray(posr[:, a]), cuda) for a in range(3))
    g = geom(dims, vs, lo=(0, 0, 0), hi=(200, 200, 200))
    spec = _lib.OlcContact(enabled=1, radius_field=-1, radius_const=0.0, stiffness=1.0, mobility=10.0,
                           max_disp=1.0, margin=0.1)
    _lib.check(olc.olc_stage_contact_tuned(dptr(pr), dptr(rg), n, C.byref(g), C.byref(spec), 0.1, variant, dptr(x),
                                           dptr(y), dptr(z), None))
    got = np.stack([to_host(x), to_host(y), to_host(z)], axis=1)
    np.testing.assert_array_equal(got, ref)
    counts = ranges[1::2] - ranges[0::2]
    if case == "dense":
        assert counts.max() > 64  # dense bins
    if case == "cluster":
        assert 32 < counts.max() <= 64


@pytest.mark.parametrize("adhesion,velocity", [(False, True), (True, False), (True, True)])
def test_contact_mechanics_matches_the_oracle(cuda, olc, adhesion, velocity):
    """The engine's force-law extras (necrotic factor, adhesion, damped
    velocity; tumor_sim.wgsl:505-628) against orc_contact_mech.  Without
    adhesion every operation is + - * / sqrt and the bits agree; the
    adhesion falloff calls cosf, which CUDA and the host C library may round
    differently by an ulp, so those cases agree to 1e-5 um."""
    rng = np.random.default_rng(21)
    dims, vs = (16, 16, 16), 10.0
    n = 20000
    pos = np.clip(rng.normal(80.0, 22.0, size=(n, 3)), 0.0, 159.0).astype(np.float32)
    pos[7] = pos[8]  # a coincident pair
    radius = rng.uniform(4.0, 6.0, size=n).astype(np.float32)
    k = oracle.keys(pos, dims, vs)
    ks, perm = oracle.sort_pairs(k)
    ranges = oracle.bin_ranges(ks, oracle.tissue_key(*dims))
    posr = np.concatenate([pos[perm], radius[perm, None]], axis=1).astype(np.float32)
    posr[rng.random(n) < 0.02, 3] = -1.0
    state = rng.choice(np.array([1, 2, 3], np.int32), size=n, p=[0.5, 0.3, 0.2]).astype(np.int32)
    vel = rng.normal(0.0, 2.0, size=(n, 3)).astype(np.float32) if velocity else None
    prm = dict(stiffness=1.0, mobility=10.0, max_disp=1.0, dt=0.1)
    mech = dict(necrotic_factor=0.3, adh_k=0.4 if adhesion else 0.0, adh_range=2.5 if adhesion else 0.0,
                damping=1.5, max_speed=8.0)
    lo, hi = (0.1, 0.1, 0.1), (159.9, 159.9, 159.9)
    ref, ref_v = oracle.contact_mech(posr, ranges, dims, vs, prm["stiffness"], prm["mobility"], prm["max_disp"],
                                     prm["dt"], lo, hi, state=state, vel=vel, **mech)
    pr, rg = to_dev(posr, cuda), to_dev(ranges, cuda)
    x, y, z = (to_dev(np.ascontiguousarray(posr[:, c]), cuda) for c in range(3))
    st = to_dev(state, cuda)
    vd = [to_dev(np.ascontiguousarray(vel[:, c]), cuda) for c in range(3)] if velocity else [None] * 3
    g = geom(dims, vs, lo=(0, 0, 0), hi=(160, 160, 160))
    spec = _lib.OlcContact(enabled=1, radius_field=-1, radius_const=0.0, stiffness=prm["stiffness"],
                           mobility=prm["mobility"], max_disp=prm["max_disp"], margin=0.1)
    m = _lib.OlcMechanics(state_field=0, necrotic_factor=mech["necrotic_factor"], adhesion_stiffness=mech["adh_k"],
                          adhesion_range=mech["adh_range"], velocity_field=0 if velocity else -1,
                          damping=mech["damping"], max_speed=mech["max_speed"], enabled=1)
    _lib.check(olc.olc_stage_contact_mech(dptr(pr), dptr(rg), n, C.byref(g), C.byref(spec), C.byref(m), dptr(st),
                                          *(dptr(v) if v is not None else None for v in vd), prm["dt"], dptr(x),
                                          dptr(y), dptr(z), None))
    got = np.stack([to_host(x), to_host(y), to_host(z)], axis=1)
    if adhesion:
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-5)
        assert np.mean(got == ref) > 0.9
    else:
        np.testing.assert_array_equal(got, ref)
    if velocity:
        got_v = np.stack([to_host(v) for v in vd], axis=1)
        if adhesion:
            np.testing.assert_allclose(got_v, ref_v, rtol=0, atol=1e-4)
        else:
            np.testing.assert_array_equal(got_v, ref_v)
        assert np.abs(got_v).max() <= mech["max_speed"] * (1 + 1e-6)
    # the extras change the result: necrotic pairs repel less, adhesion pulls
    plain = oracle.contact(posr, ranges, dims, vs, prm["stiffness"], prm["mobility"], prm["max_disp"], prm["dt"],
                           lo, hi)
    assert np.any(got != plain)


def test_contact_active_motion_matches_the_oracle(cuda, olc):
    """The engine's chemotaxis and random motility (tumor_sim.wgsl:584-604)
    on top of the force law, per species: RNG states exact; positions and
    velocities to 1e-4 (the random direction calls cosf/sinf)."""
    rng = np.random.default_rng(33)
    dims, vs = (16, 16, 16), 10.0
    cd, cvs = (32, 32, 32), 5.0
    n = 20000
    pos = np.clip(rng.normal(80.0, 22.0, size=(n, 3)), 0.0, 159.0).astype(np.float32)
    radius = rng.uniform(4.0, 6.0, size=n).astype(np.float32)
    k = oracle.keys(pos, dims, vs)
    ks, perm = oracle.sort_pairs(k)
    ranges = oracle.bin_ranges(ks, oracle.tissue_key(*dims))
    posr = np.concatenate([pos[perm], radius[perm, None]], axis=1).astype(np.float32)
    state = rng.choice(np.array([1, 2, 3], np.int32), size=n, p=[0.6, 0.3, 0.1]).astype(np.int32)
    species = rng.integers(-1, 5, size=n).astype(np.int32)  # out-of-range ids clamp
    states = (rng.integers(1, 2 ** 32, size=n, dtype=np.uint64)).astype(np.uint32)
    vel = rng.normal(0.0, 1.0, size=(n, 3)).astype(np.float32)
    zz, yy, xx = np.meshgrid(*(np.arange(d, dtype=np.float32) for d in cd[::-1]), indexing="ij")
    o2 = (0.5 + 0.4 * np.sin(xx / 5.0) * np.cos(yy / 7.0)).astype(np.float32).ravel()
    glu = (zz / cd[2]).astype(np.float32).ravel()
    table = ((1.5, 0.0, 0.3), (0.0, 2.0, 0.8), (-1.0, 0.5, 0.0))
    prm = dict(stiffness=1.0, mobility=10.0, max_disp=1.0, dt=0.1)
    lo, hi = (0.1, 0.1, 0.1), (159.9, 159.9, 159.9)
    ref, ref_v, ref_rng = oracle.contact_motion(posr, ranges, dims, vs, prm["stiffness"], prm["mobility"],
                                                prm["max_disp"], prm["dt"], lo, hi, state=state,
                                                necrotic_factor=0.3, vel=vel, damping=1.5, max_speed=8.0,
                                                species=species, rng=states, o2=o2, glu=glu, cdims=cd, cvs=cvs,
                                                chemo_force=2.0, impulse=0.4, table=table)
    pr, rg = to_dev(posr, cuda), to_dev(ranges, cuda)
    x, y, z = (to_dev(np.ascontiguousarray(posr[:, c]), cuda) for c in range(3))
    vd = [to_dev(np.ascontiguousarray(vel[:, c]), cuda) for c in range(3)]
    st, spd, rgd = to_dev(state, cuda), to_dev(species, cuda), to_dev(states, cuda)
    o2d, glud = to_dev(o2, cuda), to_dev(glu, cuda)
    g = geom(dims, vs, lo=(0, 0, 0), hi=(160, 160, 160))
    g.chem_dims[:] = cd
    g.chem_voxel_size = cvs
    spec = _lib.OlcContact(enabled=1, radius_field=-1, radius_const=0.0, stiffness=prm["stiffness"],
                           mobility=prm["mobility"], max_disp=prm["max_disp"], margin=0.1)
    m = _lib.OlcMechanics(state_field=0, necrotic_factor=0.3, adhesion_stiffness=0.0, adhesion_range=0.0,
                          velocity_field=0, damping=1.5, max_speed=8.0, enabled=1, chemo_force=2.0,
                          motility_impulse=0.4, n_species=len(table))
    for i, (a, b, c) in enumerate(table):
        m.species[i].chemotaxis_o2, m.species[i].chemotaxis_glucose, m.species[i].move_prob = a, b, c
    _lib.check(olc.olc_stage_contact_motion(dptr(pr), dptr(rg), n, C.byref(g), C.byref(spec), C.byref(m), dptr(st),
                                            *(dptr(v) for v in vd), dptr(spd), dptr(rgd), dptr(o2d), dptr(glud),
                                            prm["dt"], dptr(x), dptr(y), dptr(z), None))
    got = np.stack([to_host(x), to_host(y), to_host(z)], axis=1)
    np.testing.assert_array_equal(to_host(rgd, np.uint32), ref_rng)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-4)
    np.testing.assert_allclose(np.stack([to_host(v) for v in vd], axis=1), ref_v, rtol=0, atol=1e-4)
    # necrotic agents draw nothing; the others advance their RNG by two draws
    assert np.array_equal(ref_rng[state == 3], states[state == 3])
    assert np.all(ref_rng[state != 3] != states[state != 3])
    still, _, _ = oracle.contact_motion(posr, ranges, dims, vs, prm["stiffness"], prm["mobility"], prm["max_disp"],
                                        prm["dt"], lo, hi, state=state, necrotic_factor=0.3, vel=vel, damping=1.5,
                                        max_speed=8.0, table=())
    assert np.abs(got - still).max() > 1e-3


# ------------------------------------------------------------------ 16-bit field storage

@pytest.mark.parametrize("encoding", [0, 1, 2])
@pytest.mark.parametrize("storage", [1, 2, 3, 4])
@pytest.mark.parametrize("dims,substeps,decay,with_sink", [((32, 24, 20), 5, 0.0, True),
                                                          ((64, 41, 37), 7, 0.1, True),
                                                          ((136, 17, 9), 3, 0.05, False)])
def test_diffuse16_bit_exact(cuda, olc, storage, encoding, dims, substeps, decay, with_sink):
    """BF16 / FP16 / BF16 with stochastic rounding, each element holding the
    value, the deficit from the boundary value or the value less one of three
    offsets: three steps of reaction (uptake, decay, residual) and substeps
    give the oracle's bits, residuals included."""
    import torch

    rng = np.random.default_rng(sum(dims) + storage + 7 * encoding)
    nx, ny, nz = dims
    lo, span = (0.05, 0.6) if encoding else (0.1, 0.8)  # encoded fields live in [0, boundary = 0.7]
    f = (rng.random((nz, ny, nx), dtype=np.float32) * span + lo).astype(np.float32)
    dx, dt, D = 4.0, 0.1, 2000.0
    D = min(D, (1.0 / 6.0) * dx * dx * substeps / dt * 0.999)
    bits = oracle.to_bits16(f, storage, encoding, 0.7)
    comp = np.zeros_like(f)
    fd = torch.from_numpy(bits.view(np.int16).copy()).to(cuda)
    tmp = torch.empty_like(fd)
    cd = torch.zeros(f.size, dtype=torch.float32, device=cuda)
    spec = _lib.OlcDiffusion(diffusion=D, decay=decay, boundary=0.7, substeps=substeps, has_sink=int(with_sink),
                             storage=storage, encoding=encoding)
    dims_c = (C.c_int32 * 3)(nx, ny, nz)
    for step in range(3):
        sink = None
        sd = None
        if with_sink:
            sink = np.zeros_like(f)
            m = rng.random(f.shape) < 0.2
            sink[m] = rng.random(int(m.sum())).astype(np.float32) * 0.5
            sd = to_dev(sink, cuda)
        bits, comp = oracle.diffuse16(bits, sink, comp, dx, dt, D, decay, 0.7, substeps, storage, step=100 + step,
                                      field=1, encoding=encoding)
        _lib.check(olc.olc_stage_diffuse16(dptr(fd), dptr(tmp), dptr(sd) if sd is not None else None, dptr(cd),
                                           C.byref(dims_c), dx, dt, C.byref(spec), 100 + step, 1, None))
        torch.cuda.synchronize()
        got = fd.cpu().numpy().view(np.uint16).reshape(nz, ny, nx)
        np.testing.assert_array_equal(got, bits, err_msg=f"field bits step {step}")
        np.testing.assert_array_equal(cd.cpu().numpy().reshape(nz, ny, nx), comp, err_msg=f"residual step {step}")
        if sd is not None:
            assert float(to_host(sd).max()) == 0.0
