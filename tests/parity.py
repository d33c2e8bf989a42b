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


def deform_case(seed: int, vertex_count: int, bone_count: int = 64, stride: int = 44):
    """Seeded skinning input in the layout position float3 @0, normal float3
    @12, joints ubyte4 @24, weights float4 @28 (+ padding to `stride`):
    weights of both signs (non-positive ones are skipped), joint indices
    beyond bone_count (skipped), zero normals (not renormalised), and random
    affine bones (column-major)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    vc = vertex_count
    raw = np.zeros((vc, stride), np.uint8)
    f = np.zeros((vc, 11), np.float32)
    f[:, 0:3] = rng.uniform(-3, 3, (vc, 3))
    n = rng.normal(size=(vc, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    n[::17] = 0.0
    f[:, 3:6] = n
    w = rng.uniform(-0.2, 1.0, (vc, 4)).astype(np.float32)
    w /= np.abs(w).sum(1, keepdims=True)
    f[:, 7:11] = w
    raw[:, :44] = f.view(np.uint8).reshape(vc, 44)
    raw[:, 24:28] = rng.integers(0, min(255, bone_count + 8), (vc, 4)).astype(np.uint8)
    bones = np.zeros((bone_count, 16), np.float32)
    for k in range(bone_count):
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        m = np.eye(4)
        m[:3, :3] = q * rng.uniform(0.5, 2.0)
        m[:3, 3] = rng.uniform(-1, 1, 3)
        bones[k] = m.T.reshape(-1)
    return raw.reshape(-1), bones
