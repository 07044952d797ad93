"""Builds libolc.so (the sm_100a CUDA library) in-tree with nvcc.

The library is placed at ``oncolytica_b200/_lib/libolc.so`` so that it travels
with the source tree.  Usage::

    python -m oncolytica_b200.build_lib [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import hashlib
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libolc.so")
REPO = os.path.dirname(HERE)
INCLUDE = os.path.join(REPO, "include")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

SOURCES = ["olc_grid.cu", "olc_field.cu", "olc_field16.cu", "olc_contact.cu", "olc_reduce.cu", "olc_batch.cu", "olc_sim.cu",
           "olc_noalloc.cu", "olc_pool.cu", "olc_metrics.cu", "olc_selftest.cu"]
HEADERS = ["olc_device.cuh", "olc_rule_rt.cuh", "olc_internal.h", "olc_store16.cuh", "olc_arena.h", "olc_stencil.cuh"]

# -fmad=false keeps a*b+c as two roundings everywhere, so the CPU oracle
# (compiled with -ffp-contract=off) reproduces every floating-point stage.
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "--fmad=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
    f"-I{INCLUDE}", f"-I{CSRC}",
]


def _digest() -> str:
    h = hashlib.sha256()
    for name in SOURCES + HEADERS:
        with open(os.path.join(CSRC, name), "rb") as fh:
            h.update(fh.read())
    with open(os.path.join(INCLUDE, "olc.h"), "rb") as fh:
        h.update(fh.read())
    h.update(" ".join(NVCC_FLAGS).encode())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every source for sm_100a and links libolc.so; returns its path."""
    os.makedirs(OUT_DIR, exist_ok=True)
    stamp = os.path.join(OUT_DIR, "libolc.sha256")
    digest = _digest()
    if not force and os.path.exists(LIB) and os.path.exists(stamp):
        with open(stamp) as fh:
            if fh.read().strip() == digest:
                return LIB

    def compile_one(src: str) -> str:
        obj = os.path.join(OUT_DIR, src.replace(".cu", ".o"))
        cmd = [NVCC, *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
        if verbose and res.stderr:
            print(res.stderr, flush=True)
        return obj

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, SOURCES))

    link = [
        NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-cudart", "static",
        *objs, "-o", LIB,
        f"-L{CUDA_HOME}/lib64", "-lnvrtc",
        "-Xlinker", f"-rpath,{CUDA_HOME}/lib64",
    ]
    res = subprocess.run(link, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    for obj in objs:
        os.remove(obj)
    with open(stamp, "w") as fh:
        fh.write(digest)
    return LIB


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    args = ap.parse_args(argv)
    print(build(force=args.force, verbose=args.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
