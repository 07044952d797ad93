"""Generates struct_layouts.json from the reference itself: the AoS record
layout of its bundles (StructSerializer.update_layout over
optimize_struct_layout, framework/src/oncolytica/gpu/runtime/_memory.py:11-118).

Run in a container that has the reference checked out (nothing at test time
imports the reference):

    python tests/golden/make_bundle_golden.py [/path/to/reference]
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout: the first argument, else $OLC_REFERENCE, else a
# directory named "reference" beside this repository
REF = (sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OLC_REFERENCE")
       or os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(HERE))), "reference"))

CASES = [
    # the tumour cell (with the _rng_state every reference Cell declares first)
    [("_rng_state", "u32"), ("pos", "vec3<f32>"), ("radius", "f32"), ("volume", "f32"), ("state", "i32")],
    # test_gpu.py's MockCell
    [("_rng_state", "u32"), ("pos", "vec3<f32>"), ("id", "i32")],
    # two vec3s, an ivec3 and scalars
    [("_rng_state", "u32"), ("pos", "vec3<f32>"), ("vel", "vec3<f32>"), ("coord", "vec3<i32>"), ("a", "f32"),
     ("b", "i32"), ("c", "u32"), ("d", "f32"), ("e", "i32")],
    # chemistry / tissue records (no _rng_state)
    [("o2", "f32"), ("drug", "f32")],
    [("oxygen", "f32")],
    [("a", "f32"), ("b", "f32"), ("c", "f32"), ("d", "f32"), ("e", "f32")],
    [("v", "vec3<f32>")],
]


def main() -> None:
    sys.path.insert(0, os.path.join(REF, "framework", "src"))
    from oncolytica.gpu.runtime._memory import StructSerializer, optimize_struct_layout  # reference module

    out = []
    for fields in CASES:
        ser = StructSerializer("Case", None)
        ser.update_layout(optimize_struct_layout(list(fields)))
        out.append({"fields": [list(f) for f in fields], "order": [list(f) for f in ser.fields],
                    "offsets": ser.offsets, "stride": ser.stride})
    with open(os.path.join(HERE, "struct_layouts.json"), "w") as fh:
        json.dump({"source": "framework/src/oncolytica/gpu/runtime/_memory.py:11-118", "cases": out}, fh, indent=1)


if __name__ == "__main__":
    main()
