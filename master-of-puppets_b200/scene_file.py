""".mop v2 scene files (reference src/loader/mop_scene.c).

``save`` writes a scenes.Scene in the layout mop_scene_save produces for the
same viewport (mop_scene.c:544-766): 64-byte header, a table of contents with
one entry reserved per scene mesh, light and the camera, then the camera
section, the light sections and the mesh sections, each 8-byte aligned; mesh
vertices raw (48-byte MopVertex) or quantized (18-byte MopQuantizedVertex:
position on the mesh bbox, octahedral normal, RGBA8, UV), indices 16-bit when
the mesh has fewer than 65536 vertices.  The quantization restates
quantize_vertex / oct_encode (mop_scene.c:122-196) in float32 with the x86
build's float-to-integer conversions (truncation through int32, then the low
bits).

``upload`` reads one back straight into device memory through the C ABI
(mopcuda_scene_file_*): the stored bytes cross PCIe and are decoded on the
device.
"""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np

MAGIC = 0x4D4F5002
VERSION = 2
SAVE_QUANTIZE = 0x01
SECTION_MESH, SECTION_CAMERA, SECTION_LIGHT = 1, 2, 3
CHROME_ID_FLOOR = 0xFFFD0000
MAX_SECTIONS = 256
DEG2RAD = np.float32(np.float32(3.14159265358979323846) / np.float32(180.0))


def _align8(n: int) -> int:
    return (n + 7) & ~7


def _trunc_bits(x, bits):
    """(uintN_t)(float) as the x86-64 build converts: truncate to int32, keep
    the low bits (values here are far inside int32)."""
    return (np.trunc(np.asarray(x, np.float64)).astype(np.int64) & ((1 << bits) - 1))


def _first_extreme(p, smaller):
    """The running min/max of mop_scene_save's bbox loop (strict compare:
    the first of equal values stays, which decides the sign of a zero)."""
    m = p.min() if smaller else p.max()
    hits = np.flatnonzero(p == m)
    return p[hits[0]]


def _bbox(pos):
    bmin = np.array([_first_extreme(pos[:, j], True) for j in range(3)], np.float32)
    bmax = np.array([_first_extreme(pos[:, j], False) for j in range(3)], np.float32)
    return bmin, bmax


def _oct_encode(n):
    n = np.asarray(n, np.float32)
    nx, ny, nz = n[:, 0], n[:, 1], n[:, 2]
    s = (np.abs(nx) + np.abs(ny)) + np.abs(nz)
    s = np.where(s < np.float32(1e-8), np.float32(1e-8), s).astype(np.float32)
    ox = (nx / s).astype(np.float32)
    oy = (ny / s).astype(np.float32)
    one = np.float32(1.0)
    sx = np.where(ox >= 0, one, -one).astype(np.float32)
    sy = np.where(oy >= 0, one, -one).astype(np.float32)
    fx = ((one - np.abs(oy)) * sx).astype(np.float32)
    fy = ((one - np.abs(ox)) * sy).astype(np.float32)
    neg = nz < 0
    ox = np.where(neg, fx, ox).astype(np.float32)
    oy = np.where(neg, fy, oy).astype(np.float32)
    k = np.float32(32767.0)
    return (np.trunc((ox * k).astype(np.float64)).astype(np.int32).astype(np.int16),
            np.trunc((oy * k).astype(np.float64)).astype(np.int32).astype(np.int16))


def quantize(vertices, bmin, bmax) -> bytes:
    v = np.asarray(vertices, np.float32)
    n = v.shape[0]
    out = np.zeros((n, 9), np.uint16)
    for i in range(3):
        rng = np.float32(bmax[i] - bmin[i])
        if rng > np.float32(1e-8):
            t = ((v[:, i] - bmin[i]) / rng).astype(np.float32)
        else:
            t = np.zeros(n, np.float32)
        t = np.clip(t, np.float32(0.0), np.float32(1.0)).astype(np.float32)
        out[:, i] = _trunc_bits((t * np.float32(65535.0) + np.float32(0.5)).astype(np.float32), 16)
    nx, ny = _oct_encode(v[:, 3:6])
    out[:, 3] = nx.view(np.uint16)
    out[:, 4] = ny.view(np.uint16)
    c = _trunc_bits((v[:, 6:10] * np.float32(255.0) + np.float32(0.5)).astype(np.float32), 8)
    out[:, 5] = c[:, 0] | (c[:, 1] << 8)
    out[:, 6] = c[:, 2] | (c[:, 3] << 8)
    uv = _trunc_bits((v[:, 10:12] * np.float32(65535.0) + np.float32(0.5)).astype(np.float32), 16)
    out[:, 7] = uv[:, 0]
    out[:, 8] = uv[:, 1]
    return out.astype('<u2').tobytes()


def save(scene, path, quantize_vertices: bool = False) -> None:
    """Writes scene as mop_scene_save would for the viewport the reference
    harness builds from it (camera as set, lights, then the scene meshes)."""
    meshes = [m for m in scene.meshes if m.object_id != 0 and m.object_id < CHROME_ID_FLOOR]
    n_active = sum(1 for l in scene.lights if l.active)
    nsec = len(meshes) + 1 + n_active
    if nsec > MAX_SECTIONS:  # mop_scene_save refuses these too (mop_scene.c:556-559)
        raise ValueError(f"{nsec} sections: the format holds at most {MAX_SECTIONS}")
    body = bytearray()
    toc = []
    start = _align8(64 + 24 * nsec)

    def put(kind, flags, data):
        toc.append(struct.pack("<IIQQ", kind, flags, start + len(body), len(data)))
        body.extend(data)
        body.extend(b"\0" * (_align8(len(body)) - len(body)))

    f32 = np.float32
    cam = np.array(list(scene.eye) + list(scene.target) + list(scene.up) +
                   [f32(scene.fov_deg) * DEG2RAD, scene.near, scene.far,
                    f32(scene.width) / f32(scene.height)], np.float32)
    put(SECTION_CAMERA, 0, cam.tobytes() + b"\0" * 4)
    # mop_scene_save visits light slots 0..(active count - 1) and skips an
    # inactive slot (mop_scene.c:616-648)
    for l in scene.lights[:n_active]:
        if not l.active:
            continue
        vals = np.array(list(l.position) + list(l.direction) + list(l.color) +
                        [l.intensity, l.range, l.spot_inner_cos, l.spot_outer_cos], np.float32)
        put(SECTION_LIGHT, 0, struct.pack("<I", l.type) + vals.tobytes() + b"\0" * 4)
    for m in meshes:
        v = np.ascontiguousarray(m.vertices, np.float32)
        idx = np.ascontiguousarray(m.indices, np.uint32)
        if v.shape[0] == 0:
            continue
        bmin, bmax = _bbox(v[:, :3])
        isz = 2 if v.shape[0] < 65536 else 4
        enc = 1 if quantize_vertices else 0
        hdr = struct.pack("<IIII", v.shape[0], idx.size, enc, isz) + bmin.tobytes() + \
            bmax.tobytes() + b"\0" * 8
        vb = quantize(v, bmin, bmax) if quantize_vertices else v.tobytes()
        ib = idx.astype("<u2").tobytes() if isz == 2 else idx.astype("<u4").tobytes()
        put(SECTION_MESH, enc, hdr + vb + b"\0" * (_align8(48 + len(vb)) - 48 - len(vb)) + ib)
    head = struct.pack("<IIII", MAGIC, VERSION, len(toc), SAVE_QUANTIZE if quantize_vertices
                       else 0) + b"\0" * 48
    toc_bytes = b"".join(toc) + b"\0" * (24 * (nsec - len(toc)))
    with open(path, "wb") as fp:
        fp.write(head + toc_bytes + b"\0" * (start - 64 - len(toc_bytes)) + bytes(body))


def upload_all(device, path, host_shadow: bool = False):
    """upload's result through mopcuda_scene_file_upload_all: one copy, two
    decode launches, one device allocation for every mesh (bbox not
    returned)."""
    import mopcuda
    L = device.L
    f = L.mopcuda_scene_file_open(str(path).encode())
    if not f:
        raise RuntimeError(f"scene_file_open: {mopcuda.last_error()}")
    try:
        n = L.mopcuda_scene_file_mesh_count(f)
        vbs, ibs = (C.c_void_p * max(1, n))(), (C.c_void_p * max(1, n))()
        vcs, ics = (C.c_uint32 * max(1, n))(), (C.c_uint32 * max(1, n))()
        if L.mopcuda_scene_file_upload_all(device.h, f, 1 if host_shadow else 0, vbs, ibs, vcs,
                                           ics) != 0:
            raise RuntimeError(f"scene_file_upload_all: {mopcuda.last_error()}")
        return [{"vertices": vbs[k], "indices": ibs[k], "vertex_count": vcs[k],
                 "index_count": ics[k]} for k in range(n)]
    finally:
        L.mopcuda_scene_file_close(f)


def upload(device, path, host_shadow: bool = False):
    """Every mesh of the file in device memory: a list of dicts with the
    vertex / index buffers (C-ABI handles), counts and bbox."""
    import mopcuda
    L = device.L
    f = L.mopcuda_scene_file_open(str(path).encode())
    if not f:
        raise RuntimeError(f"scene_file_open: {mopcuda.last_error()}")
    out = []
    try:
        for k in range(L.mopcuda_scene_file_mesh_count(f)):
            vb, ib = C.c_void_p(), C.c_void_p()
            vc, ic = C.c_uint32(), C.c_uint32()
            bmin, bmax = (C.c_float * 3)(), (C.c_float * 3)()
            rc = L.mopcuda_scene_file_upload_mesh(device.h, f, k, 1 if host_shadow else 0,
                                                  C.byref(vb), C.byref(ib), C.byref(vc),
                                                  C.byref(ic), bmin, bmax)
            if rc != 0:
                raise RuntimeError(f"scene_file_upload_mesh: {mopcuda.last_error()}")
            out.append({"vertices": vb.value, "indices": ib.value, "vertex_count": vc.value,
                        "index_count": ic.value, "bbox_min": tuple(bmin), "bbox_max": tuple(bmax)})
        return out
    except Exception:
        for b in out:
            L.mopcuda_buffer_destroy(device.h, b["vertices"])
            L.mopcuda_buffer_destroy(device.h, b["indices"])
        raise
    finally:
        L.mopcuda_scene_file_close(f)
