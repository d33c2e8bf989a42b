""".mop v2 scene files (reference src/loader/mop_scene.c) on the CPU.

* the product-side writer (scene_file.save) produces the reference's own
  mop_scene_save bytes, raw and quantized — against committed files the
  reference wrote (tests/golden/make_golden.py scene_files) and, when the
  reference library is built, live on more scenes;
* the oracle's decode (mop_scene_get_mesh restated) equals the reference's
  decode bit for bit;
* the C ABI's file checks (mopcuda_scene_file_open: magic, version, section
  count, table of contents inside the file) and its section readers — host
  code, no device needed.
"""
import ctypes as C
import dataclasses
import struct
from pathlib import Path

import numpy as np
import pytest

import cpu_oracle
import mopcuda
import refdrive
import scene_file
import scenes

GOLDEN = Path(__file__).resolve().parent / "golden"
GOLDEN_FILES = {"scene_small_quant": (lambda: scenes.small_scene(seed=3), True),
                "scene_coplanar_raw": (lambda: scenes.coplanar_scene(), False)}


@pytest.mark.parametrize("name", list(GOLDEN_FILES))
def test_writer_matches_golden(tmp_path, name):
    make, quant = GOLDEN_FILES[name]
    path = tmp_path / "ours.mop"
    scene_file.save(make(), path, quant)
    assert path.read_bytes() == (GOLDEN / f"{name}.mop").read_bytes()


@pytest.mark.parametrize("name", list(GOLDEN_FILES))
def test_oracle_decode_matches_golden(name):
    got = cpu_oracle.scene_file_meshes(GOLDEN / f"{name}.mop")
    want = np.load(GOLDEN / f"{name}_decoded.npz")
    assert len(got) == len([k for k in want.files if k.startswith("v")])
    for k, (v, i, bb) in enumerate(got):
        assert v.tobytes() == want[f"v{k}"].tobytes(), f"mesh {k} vertices"
        assert (i == want[f"i{k}"]).all() and bb.tobytes() == want[f"b{k}"].tobytes()


LIVE = {
    "mixed_ssaa2": lambda: scenes.small_scene(seed=4, ssaa=2, width=100, height=60),
    "config2_small": lambda: scenes.config2(width=64, height=36, instances=3, tex_size=8),
    # one mesh above 65535 vertices: 32-bit indices; non-unit normals and
    # tiled UVs exercise the quantizer's clamps and wraps
    "wide": lambda: _wide_scene(),
}


def _wide_scene():
    sc = scenes.small_scene(seed=5, n_meshes=2)
    v, i = scenes.uv_sphere(300, 240, 1.3, (0.2, 0.5, 0.9, 1.0))
    v = v.copy()
    v[:, 3:6] *= 1.7
    v[:, 10:12] = v[:, 10:12] * 3.0 - 1.0
    sc.meshes.append(scenes.Mesh(v, i, 99, scenes.mat_identity()))
    return sc


@pytest.mark.skipif(not refdrive.available(), reason="reference library not built")
@pytest.mark.parametrize("name", list(LIVE))
@pytest.mark.parametrize("quant", [False, True])
def test_writer_and_decode_match_reference_live(tmp_path, name, quant):
    sc = LIVE[name]()
    ref_path, our_path = tmp_path / "ref.mop", tmp_path / "ours.mop"
    r = refdrive.Reference(sc, serial=True)
    r.save_scene(ref_path, quant)
    r.close()
    scene_file.save(sc, our_path, quant)
    assert our_path.read_bytes() == ref_path.read_bytes()
    for k, (v, i, bb) in enumerate(cpu_oracle.scene_file_meshes(ref_path)):
        rv, ri, rb = refdrive.scene_file_mesh(ref_path, k)
        assert v.tobytes() == rv.tobytes() and (i == ri).all() and bb.tobytes() == rb.tobytes()


def _open(path):
    return mopcuda.lib().mopcuda_scene_file_open(str(path).encode())


def test_loader_reads_sections():
    L = mopcuda.lib()
    sc = GOLDEN_FILES["scene_small_quant"][0]()
    f = _open(GOLDEN / "scene_small_quant.mop")
    assert f
    try:
        assert L.mopcuda_scene_file_mesh_count(f) == len(sc.meshes)
        n_lights = L.mopcuda_scene_file_light_count(f)
        assert n_lights == sum(1 for l in sc.lights if l.active)
        eye, tgt, up = (C.c_float * 3)(), (C.c_float * 3)(), (C.c_float * 3)()
        fov, near, far = C.c_float(), C.c_float(), C.c_float()
        assert L.mopcuda_scene_file_camera(f, eye, tgt, up, C.byref(fov), C.byref(near),
                                           C.byref(far)) == 0
        assert np.allclose(list(eye), sc.eye) and np.allclose(list(tgt), sc.target)
        assert np.isclose(fov.value, np.deg2rad(sc.fov_deg)) and near.value == np.float32(sc.near)
        for k in range(n_lights):
            lt = mopcuda.MopCudaLight()
            assert L.mopcuda_scene_file_light(f, k, C.byref(lt)) == 0
            assert lt.type == sc.lights[k].type
            assert np.float32(lt.intensity) == np.float32(sc.lights[k].intensity)
        assert L.mopcuda_scene_file_light(f, n_lights, C.byref(mopcuda.MopCudaLight())) != 0
    finally:
        L.mopcuda_scene_file_close(f)


@pytest.mark.parametrize("patch,why", [
    (lambda b: struct.pack_into("<I", b, 0, 0x4D4F5001), "bad magic"),
    (lambda b: struct.pack_into("<I", b, 4, 3), "unsupported version"),
    (lambda b: struct.pack_into("<I", b, 8, 257), "more than 256 sections"),
    (lambda b: struct.pack_into("<I", b, 8, 200), "table of contents beyond the file"),
])
def test_loader_rejects_bad_headers(tmp_path, patch, why):
    data = bytearray((GOLDEN / "scene_coplanar_raw.mop").read_bytes())
    patch(data)
    path = tmp_path / "bad.mop"
    path.write_bytes(bytes(data))
    assert not _open(path)
    assert why in mopcuda.last_error()


def test_loader_rejects_short_file(tmp_path):
    path = tmp_path / "short.mop"
    path.write_bytes((GOLDEN / "scene_coplanar_raw.mop").read_bytes()[:40])
    assert not _open(path)
    assert not _open(tmp_path / "missing.mop")
