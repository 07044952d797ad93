"""Hierarchical Morton keys on the host (API of the reference's
framework/src/oncolytica/core/runtime/_geometry.py:14-47), vectorised with
numpy.  The device computes the same keys in csrc/olc_device.cuh."""
from __future__ import annotations

import numpy as np


def interleave_9bit(x):
    x = np.asarray(x, dtype=np.uint32) & np.uint32(0x1FF)
    x = (x | (x << np.uint32(16))) & np.uint32(0x030000FF)
    x = (x | (x << np.uint32(8))) & np.uint32(0x0300F00F)
    x = (x | (x << np.uint32(4))) & np.uint32(0x030C30C3)
    x = (x | (x << np.uint32(2))) & np.uint32(0x09249249)
    return x


def get_chemical_voxel_key(cx, cy, cz):
    k = interleave_9bit(cx) | (interleave_9bit(cy) << np.uint32(1)) | (interleave_9bit(cz) << np.uint32(2))
    return int(k) if np.ndim(k) == 0 else k


def get_sub_voxel_index(sx, sy, sz):
    sx, sy, sz = (np.asarray(v, dtype=np.int64) for v in (sx, sy, sz))
    k = ((sx & 1) | ((sy & 1) << 1) | ((sz & 1) << 2)).astype(np.uint32)
    return int(k) if np.ndim(k) == 0 else k


def get_tissue_voxel_key(sx, sy, sz):
    sx, sy, sz = (np.asarray(v, dtype=np.int64) for v in (sx, sy, sz))
    j = np.asarray(get_chemical_voxel_key(sx // 2, sy // 2, sz // 2), dtype=np.uint32)
    k = (j << np.uint32(3)) | np.asarray(get_sub_voxel_index(sx, sy, sz), dtype=np.uint32)
    return int(k) if np.ndim(k) == 0 else k


def voxel_table_size(tissue_grid_dim) -> int:
    return int(get_tissue_voxel_key(*tissue_grid_dim)) + 1
