""".mop v2 meshes decoded on the device (mopcuda_scene_file_upload_mesh)
against mop_scene_get_mesh's host decode — the oracle's restatement and the
committed arrays the reference itself decoded — byte for byte, for raw and
quantized vertices and 16- and 32-bit indices, mesh by mesh and for the whole
file in one pass; the host copy kept on request;
a truncated section rejected; and a frame rendered from the device-decoded
buffers against the oracle's frame of the decoded meshes."""
import ctypes as C
import dataclasses
import struct
from pathlib import Path

import numpy as np
import pytest

import cpu_oracle
import mopcuda
import scene_file
import scenes
from parity import assert_frame_parity

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def _device_meshes(dev, path, host_shadow=False, whole_file=False):
    if whole_file:
        bufs = scene_file.upload_all(dev, path, host_shadow)
        for b, (_, _, bb) in zip(bufs, cpu_oracle.scene_file_meshes(path)):
            b["bbox_min"], b["bbox_max"] = tuple(bb[:3]), tuple(bb[3:])
    else:
        bufs = scene_file.upload(dev, path, host_shadow)
    L = dev.L
    out = []
    for b in bufs:
        v = np.zeros((b["vertex_count"], 12), np.float32)
        i = np.zeros(b["index_count"], np.uint32)
        if host_shadow:
            pv = L.mopcuda_buffer_read(b["vertices"])
            pi = L.mopcuda_buffer_read(b["indices"])
            C.memmove(v.ctypes.data, pv, v.nbytes)
            C.memmove(i.ctypes.data, pi, i.nbytes)
        else:
            assert not L.mopcuda_buffer_read(b["vertices"])
            v, i = _read_device(dev, b, v, i)
        out.append((v, i, np.array(b["bbox_min"] + b["bbox_max"], np.float32)))
        L.mopcuda_buffer_destroy(dev.h, b["vertices"])
        L.mopcuda_buffer_destroy(dev.h, b["indices"])
    return out


def _read_device(dev, b, v, i):
    L = dev.L
    assert L.mopcuda_buffer_copy_to_host(dev.h, b["vertices"], 0, v.ctypes.data, v.nbytes) == 0
    assert L.mopcuda_buffer_copy_to_host(dev.h, b["indices"], 0, i.ctypes.data, i.nbytes) == 0
    return v, i


def _same(got, want):
    assert len(got) == len(want)
    for k, ((v, i, bb), (rv, ri, rb)) in enumerate(zip(got, want)):
        assert v.tobytes() == rv.tobytes(), f"mesh {k}: vertices differ"
        assert (i == ri).all(), f"mesh {k}: indices differ"
        assert bb.tobytes() == rb.tobytes()


@pytest.mark.parametrize("name", ["scene_small_quant", "scene_coplanar_raw"])
@pytest.mark.parametrize("host_shadow", [True, False])
@pytest.mark.parametrize("whole_file", [False, True])
def test_device_decode_matches_reference(cuda_device, name, host_shadow, whole_file):
    want = np.load(GOLDEN / f"{name}_decoded.npz")
    n = len([k for k in want.files if k.startswith("v")])
    ref = [(want[f"v{k}"], want[f"i{k}"], want[f"b{k}"]) for k in range(n)]
    _same(_device_meshes(cuda_device, GOLDEN / f"{name}.mop", host_shadow, whole_file), ref)


@pytest.mark.parametrize("quant", [False, True])
def test_device_decode_wide_mesh(cuda_device, tmp_path, quant):
    """A mesh above 65535 vertices (32-bit indices), non-unit normals and
    tiled UVs, against the oracle's decode."""
    sc = scenes.small_scene(seed=5, n_meshes=2)
    v, i = scenes.uv_sphere(300, 240, 1.3, (0.2, 0.5, 0.9, 1.0))
    v = v.copy()
    v[:, 3:6] *= 1.7
    v[:, 10:12] = v[:, 10:12] * 3.0 - 1.0
    sc.meshes.append(scenes.Mesh(v, i, 99, scenes.mat_identity()))
    path = tmp_path / "wide.mop"
    scene_file.save(sc, path, quant)
    want = cpu_oracle.scene_file_meshes(path)
    _same(_device_meshes(cuda_device, path, True), want)
    _same(_device_meshes(cuda_device, path, False, whole_file=True), want)


def test_truncated_section_rejected(cuda_device, tmp_path):
    data = bytearray((GOLDEN / "scene_coplanar_raw.mop").read_bytes())
    kind, _, off, size = struct.unpack_from("<IIQQ", data, 64 + 24 * 10)  # a mesh entry
    assert kind == 1
    struct.pack_into("<I", data, off, 1000)  # vertex count beyond the section
    path = tmp_path / "bad.mop"
    path.write_bytes(bytes(data))
    with pytest.raises(RuntimeError, match="shorter than"):
        scene_file.upload(cuda_device, path)
    with pytest.raises(RuntimeError, match="shorter than"):
        scene_file.upload_all(cuda_device, path)


@pytest.mark.parametrize("quant,whole_file", [(False, False), (True, False), (True, True)])
def test_frame_from_device_decoded_scene(cuda_device, tmp_path, quant, whole_file):
    sc = scenes.small_scene(seed=6, width=160, height=120)
    path = tmp_path / "scene.mop"
    scene_file.save(sc, path, quant)
    decoded = cpu_oracle.scene_file_meshes(path)
    sc_dec = dataclasses.replace(sc, meshes=[dataclasses.replace(m, vertices=d[0], indices=d[1])
                                             for m, d in zip(sc.meshes, decoded)])
    ref = cpu_oracle.render(sc_dec)
    up = scene_file.upload_all if whole_file else scene_file.upload
    r = mopcuda.SceneRenderer(cuda_device, sc_dec, None, preloaded=up(cuda_device, path))
    try:
        r.render()
        got = {"object_id": r.object_id(), "depth": r.depth(), "color_full": r.color_full(),
               "color": r.color()}
        assert_frame_parity(got, ref, f"scene file quant={quant}")
    finally:
        r.close()
