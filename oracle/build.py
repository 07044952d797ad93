"""Builds the CPU oracle (test infrastructure) into oracle/_build/liboracle.so.

gcc -O2 -fopenmp -ffp-contract=off: no fused multiply-add, so every float
operation rounds exactly as the CUDA kernels' separately rounded operations.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle.so")
SRC = [os.path.join(HERE, "olc_oracle.c")]
HDR = [os.path.join(HERE, "olc_oracle.h")]
FLAGS = ["-O2", "-std=c11", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-Wall"]


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    h = hashlib.sha256()
    for p in SRC + HDR:
        with open(p, "rb") as fh:
            h.update(fh.read())
    h.update(" ".join(FLAGS).encode())
    digest = h.hexdigest()
    stamp = os.path.join(OUT_DIR, "liboracle.sha256")
    if not force and os.path.exists(LIB) and os.path.exists(stamp) and open(stamp).read().strip() == digest:
        return LIB
    cmd = ["gcc", *FLAGS, *SRC, "-o", LIB, "-lm"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")
    with open(stamp, "w") as fh:
        fh.write(digest)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
