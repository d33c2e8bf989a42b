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


def test_per_mesh_buffers_across_chunks(cuda_device, tmp_path):
    """Per-mesh uploads carve their buffers from 64 MiB device chunks: uploads
    that fill several chunks, a mesh larger than a chunk (an allocation of
    its own), buffers destroyed out of order while others stay live, and
    uploads after that all keep every buffer's bytes equal to the oracle's
    decode."""
    big_v, big_i = scenes.uv_sphere(1200, 1200, 1.0, (0.8, 0.3, 0.2, 1.0))  # 1.45 M vertices
    sc = scenes.small_scene(seed=9, n_meshes=1)
    v, i = scenes.uv_sphere(300, 240, 1.1, (0.2, 0.5, 0.9, 1.0))  # 3.5 MB decoded
    sc.meshes = [scenes.Mesh(v, i, 11, scenes.mat_identity())]
    path = tmp_path / "mid.mop"
    scene_file.save(sc, path, True)
    want = cpu_oracle.scene_file_meshes(path)[0]
    sc_big = scenes.small_scene(seed=9, n_meshes=1)
    sc_big.meshes = [scenes.Mesh(big_v, big_i, 12, scenes.mat_identity())]
    big_path = tmp_path / "big.mop"
    scene_file.save(sc_big, big_path, True)
    want_big = cpu_oracle.scene_file_meshes(big_path)[0]
    assert want_big[0].nbytes > 64 << 20
    L = cuda_device.L
    live = []

    def check(b, w):
        v = np.zeros((b["vertex_count"], 12), np.float32)
        i = np.zeros(b["index_count"], np.uint32)
        _read_device(cuda_device, b, v, i)
        assert v.tobytes() == w[0].tobytes() and (i == w[1]).all()

    def drop(b):
        L.mopcuda_buffer_destroy(cuda_device.h, b["vertices"])
        L.mopcuda_buffer_destroy(cuda_device.h, b["indices"])

    try:
        for _ in range(40):  # about 140 MB: three chunks
            live.append((scene_file.upload(cuda_device, path)[0], want))
        live.append((scene_file.upload(cuda_device, big_path)[0], want_big))
        for b, w in live:
            check(b, w)
        for k in sorted(range(len(live)), key=lambda k: (k * 7) % 11)[:25]:
            drop(live[k][0])
            live[k] = None
        live = [x for x in live if x is not None]
        for _ in range(20):
            live.append((scene_file.upload(cuda_device, path)[0], want))
        for b, w in live:
            check(b, w)
    finally:
        for x in live:
            drop(x[0])


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
