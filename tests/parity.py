"""Comparison helpers shared by the parity tests.

Tolerances: object IDs and depth bit-exact; 8-bit
colour within 1 LSB on >= 99.9% of samples/pixels and within 2 LSB
everywhere.  Colour can differ from the CPU reference only through the IBL
direction->uv mapping, where CUDA's atan2f/asinf and glibc's differ in the
last ulp for some inputs.
"""
import numpy as np

COLOR_MAX_LSB = 2
COLOR_1LSB_FRACTION = 0.999


def color_stats(a, b):
    d = np.abs(a.astype(np.int32) - b.astype(np.int32)).max(axis=-1)
    return {"max": int(d.max()) if d.size else 0,
            "within1": float((d <= 1).mean()) if d.size else 1.0,
            "exact": float((d == 0).mean()) if d.size else 1.0}


def assert_frame_parity(got, ref, label=""):
    ids, dep = got["object_id"], got["depth"]
    bad_id = int((ids != ref["object_id"]).sum())
    bad_dep = int((dep.view(np.uint32) != ref["depth"].view(np.uint32)).sum())
    assert bad_id == 0, f"{label}: {bad_id} object-ID mismatches"
    assert bad_dep == 0, f"{label}: {bad_dep} depth mismatches (bitwise)"
    for key in ("color_full", "color"):
        s = color_stats(got[key], ref[key])
        assert s["max"] <= COLOR_MAX_LSB, f"{label}: {key} max diff {s}"
        assert s["within1"] >= COLOR_1LSB_FRACTION, f"{label}: {key} {s}"
