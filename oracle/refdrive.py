"""ctypes driver for the reference library built into oracle/_ref/libmopref.so.

Test infrastructure only: tests/ use it to pin the C oracle against the
reference itself, and bench.py's CPU-baseline leg uses it to time the
reference CPU backend.  Structures mirror oracle/ref_harness.h.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_SO = HERE / "_ref" / "libmopref.so"


class RefMesh(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("vertex_count", C.c_uint32),
                ("indices", C.c_void_p), ("index_count", C.c_uint32),
                ("object_id", C.c_uint32), ("transform", C.c_float * 16),
                ("metallic", C.c_float), ("roughness", C.c_float),
                ("has_material", C.c_int32), ("texture", C.c_int32),
                ("opacity", C.c_float), ("blend_mode", C.c_int32)]


class RefLight(C.Structure):
    _fields_ = [("type", C.c_int32), ("position", C.c_float * 3),
                ("direction", C.c_float * 3), ("color", C.c_float * 4),
                ("intensity", C.c_float), ("range", C.c_float),
                ("spot_inner_cos", C.c_float), ("spot_outer_cos", C.c_float),
                ("active", C.c_int32), ("cast_shadows", C.c_int32)]


class RefInstanced(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("vertex_count", C.c_uint32),
                ("indices", C.c_void_p), ("index_count", C.c_uint32),
                ("object_id", C.c_uint32), ("transforms", C.c_void_p),
                ("instance_count", C.c_uint32)]


class RefScene(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("ssaa", C.c_int32),
                ("clear_color", C.c_float * 4), ("eye", C.c_float * 3),
                ("target", C.c_float * 3), ("up", C.c_float * 3),
                ("fov_deg", C.c_float), ("near_plane", C.c_float), ("far_plane", C.c_float),
                ("ambient", C.c_float), ("exposure", C.c_float),
                ("post_effects", C.c_uint32), ("mesh_count", C.c_uint32),
                ("meshes", C.POINTER(RefMesh)), ("texture_count", C.c_uint32),
                ("tex_w", C.POINTER(C.c_int32)), ("tex_h", C.POINTER(C.c_int32)),
                ("tex_data", C.POINTER(C.c_void_p)), ("light_count", C.c_uint32),
                ("lights", C.POINTER(RefLight)), ("env", C.c_int32),
                ("sun_dir", C.c_float * 3), ("turbidity", C.c_float),
                ("ground_albedo", C.c_float), ("env_rotation", C.c_float),
                ("env_intensity", C.c_float), ("serial", C.c_int32),
                ("flat", C.c_int32), ("workers", C.c_int32),
                ("backend", C.c_int32), ("fog_on", C.c_int32),
                ("fog_color", C.c_float * 4), ("fog_near", C.c_float),
                ("fog_far", C.c_float), ("instanced_count", C.c_uint32),
                ("instanced", C.POINTER(RefInstanced)), ("tex_format", C.POINTER(C.c_int32)),
                ("tex_bytes", C.POINTER(C.c_uint32)), ("render_target", C.c_int32),
                ("env_background", C.c_int32), ("wireframe", C.c_int32)]


class RefFrame(C.Structure):
    _fields_ = [("color", C.c_void_p), ("color_full", C.c_void_p),
                ("depth", C.c_void_p), ("object_id", C.c_void_p),
                ("view", C.c_float * 16), ("proj", C.c_float * 16),
                ("eye", C.c_float * 3), ("triangle_count", C.c_uint32),
                ("frame_ms", C.c_double)]


def light_struct(L, cls=RefLight):
    s = cls()
    s.type = L.type
    s.position[:] = L.position
    s.direction[:] = L.direction
    s.color[:] = L.color
    s.intensity = L.intensity
    s.range = L.range
    s.spot_inner_cos = L.spot_inner_cos
    s.spot_outer_cos = L.spot_outer_cos
    s.active = 1 if L.active else 0
    s.cast_shadows = 1 if getattr(L, "cast_shadows", False) else 0
    return s


_libs = {}
REF_CUDA_SO = HERE / "_ref" / "libmopref_cuda.so"
BACKEND_CUDA = 4  # MOP_BACKEND_CUDA in the integration patch


def available() -> bool:
    return REF_SO.exists()


def lib(kind: str = "cpu"):
    so = REF_SO if kind == "cpu" else REF_CUDA_SO
    if kind not in _libs:
        if not so.exists():
            raise FileNotFoundError(f"reference library not built: {so}")
        _lib = _libs[kind] = C.CDLL(str(so))
        _lib.refh_create.restype = C.c_void_p
        _lib.refh_create.argtypes = [C.POINTER(RefScene)]
        _lib.refh_render.argtypes = [C.c_void_p, C.POINTER(RefFrame)]
        _lib.refh_pick.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.refh_env_maps.argtypes = [C.c_void_p] + [C.c_void_p] * 9
        _lib.refh_env_hdr.argtypes = [C.c_void_p] * 4
        _lib.refh_scene_save.argtypes = [C.c_void_p, C.c_char_p, C.c_uint32]
        _lib.refh_scene_file_mesh.argtypes = [C.c_char_p, C.c_uint32, C.c_void_p, C.c_uint32,
                                              C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                              C.c_void_p]
        _lib.refh_time_scene_file.restype = C.c_double
        _lib.refh_time_scene_file.argtypes = [C.c_char_p, C.c_int]
        _lib.refh_time_frames.restype = C.c_double
        _lib.refh_time_frames.argtypes = [C.c_void_p, C.c_int, C.c_int]
        _lib.refh_time_environment.restype = C.c_double
        _lib.refh_time_environment.argtypes = [C.c_void_p, C.c_int]
        _lib.refh_num_threads.argtypes = [C.c_void_p]
        _lib.refh_destroy.argtypes = [C.c_void_p]
        _lib.refh_bc_decode.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                        C.c_uint32, C.c_void_p]
        _lib.refh_present_to_texture.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        _lib.refh_read_target.argtypes = [C.c_void_p, C.c_void_p]
        if hasattr(_lib, "refh_deform_probe"):
            _lib.refh_deform_probe.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32,
                                               C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
    return _libs[kind]


class Reference:
    """A reference CPU-backend viewport holding one scene."""

    def __init__(self, scene, serial: bool = True, workers: int = 0, backend: str = "cpu",
                 render_target: bool = False):
        """render_target: the viewport renders into a host texture
        (MopViewportDesc.render_target), read back with read_target()."""
        L = self.L = lib(backend)
        self.render_target = render_target
        self.scene = scene
        self._keep = []
        meshes = (RefMesh * max(1, len(scene.meshes)))()
        for k, m in enumerate(scene.meshes):
            v = np.ascontiguousarray(m.vertices, np.float32)
            i = np.ascontiguousarray(m.indices, np.uint32)
            self._keep += [v, i]
            rm = meshes[k]
            rm.vertices = v.ctypes.data
            rm.vertex_count = v.shape[0]
            rm.indices = i.ctypes.data
            rm.index_count = i.size
            rm.object_id = m.object_id
            rm.transform[:] = [float(x) for x in m.transform]
            rm.metallic = m.metallic
            rm.roughness = m.roughness
            rm.has_material = 1 if m.has_material else 0
            rm.texture = m.texture
            rm.opacity = m.opacity
            rm.blend_mode = getattr(m, "blend_mode", 0)
        lights = (RefLight * max(1, len(scene.lights)))()
        for k, l in enumerate(scene.lights):
            lights[k] = light_struct(l)
        nt = len(scene.textures)
        tw = (C.c_int32 * max(1, nt))()
        th = (C.c_int32 * max(1, nt))()
        td = (C.c_void_p * max(1, nt))()
        tf = (C.c_int32 * max(1, nt))()
        tb = (C.c_uint32 * max(1, nt))()
        for k, t in enumerate(scene.textures):
            if hasattr(t, "format"):  # block-compressed (mop_tex_create)
                d = np.ascontiguousarray(t.data, np.uint8)
                self._keep.append(d)
                th[k], tw[k], tf[k], tb[k] = t.height, t.width, t.format, d.size
                td[k] = d.ctypes.data
                continue
            t = np.ascontiguousarray(t, np.uint8)
            self._keep.append(t)
            th[k], tw[k] = t.shape[0], t.shape[1]
            td[k] = t.ctypes.data
        sc = RefScene()
        sc.width, sc.height, sc.ssaa = scene.width, scene.height, scene.ssaa
        sc.clear_color[:] = scene.clear
        sc.eye[:] = scene.eye
        sc.target[:] = scene.target
        sc.up[:] = scene.up
        sc.fov_deg, sc.near_plane, sc.far_plane = scene.fov_deg, scene.near, scene.far
        sc.ambient, sc.exposure = scene.ambient, scene.exposure
        sc.post_effects = scene.post_effects
        sc.mesh_count = len(scene.meshes)
        sc.meshes = meshes
        sc.texture_count = nt
        sc.tex_w, sc.tex_h, sc.tex_data = tw, th, td
        sc.light_count = len(scene.lights)
        sc.lights = lights
        sc.env = scene.env
        sc.sun_dir[:] = scene.sun_dir
        sc.turbidity, sc.ground_albedo = scene.turbidity, scene.ground_albedo
        sc.env_rotation, sc.env_intensity = scene.env_rotation, scene.env_intensity
        sc.serial = 1 if serial else 0
        sc.flat = 0 if getattr(scene, "smooth", True) else 1
        sc.wireframe = (2 if getattr(scene, "wireframe_grid", False) else 1) \
            if getattr(scene, "wireframe", False) else 0
        sc.workers = int(workers)
        sc.backend = 0 if backend == "cpu" else BACKEND_CUDA
        fog = getattr(scene, "fog", None)
        if fog is not None:
            sc.fog_on = 1
            sc.fog_color[:] = fog[0]
            sc.fog_near, sc.fog_far = fog[1], fog[2]
        inst = getattr(scene, "instanced", [])
        ia = (RefInstanced * max(1, len(inst)))()
        for k, im in enumerate(inst):
            v = np.ascontiguousarray(im.vertices, np.float32)
            i = np.ascontiguousarray(im.indices, np.uint32)
            t = np.ascontiguousarray(im.transforms, np.float32).reshape(-1, 16)
            self._keep += [v, i, t]
            ia[k].vertices, ia[k].vertex_count = v.ctypes.data, v.shape[0]
            ia[k].indices, ia[k].index_count = i.ctypes.data, i.size
            ia[k].object_id = im.object_id
            ia[k].transforms, ia[k].instance_count = t.ctypes.data, t.shape[0]
        sc.instanced_count = len(inst)
        sc.instanced = ia
        sc.tex_format, sc.tex_bytes = tf, tb
        sc.render_target = 1 if render_target else 0
        sc.env_background = 1 if getattr(scene, "env_background", False) else 0
        self._keep += [meshes, lights, tw, th, td, tf, tb, sc, ia]
        self.h = L.refh_create(C.byref(sc))
        if not self.h:
            raise RuntimeError("refh_create failed")

    def render(self):
        s = self.scene
        S = s.samples
        out = {
            "color": np.zeros((s.height, s.width, 4), np.uint8),
            "color_full": np.zeros((s.height * s.ssaa, s.width * s.ssaa, 4), np.uint8),
            "depth": np.zeros((s.height * s.ssaa, s.width * s.ssaa), np.float32),
            "object_id": np.zeros((s.height * s.ssaa, s.width * s.ssaa), np.uint32),
        }
        f = RefFrame()
        f.color = out["color"].ctypes.data
        f.color_full = out["color_full"].ctypes.data
        f.depth = out["depth"].ctypes.data
        f.object_id = out["object_id"].ctypes.data
        rc = self.L.refh_render(self.h, C.byref(f))
        if rc != 0:
            raise RuntimeError(f"refh_render failed: {rc}")
        out["view"] = np.array(f.view[:], np.float32)
        out["proj"] = np.array(f.proj[:], np.float32)
        out["eye"] = np.array(f.eye[:], np.float32)
        out["triangle_count"] = f.triangle_count
        assert S == out["depth"].size
        return out

    def present_to_texture(self, tw: int, th: int):
        """mop_viewport_present_to_texture into a new tw x th RGBA8 texture:
        its pixels, or None when the core refused the present."""
        out = np.zeros((th, tw, 4), np.uint8)
        rc = self.L.refh_present_to_texture(self.h, tw, th, out.ctypes.data)
        if rc < 0:
            raise RuntimeError(f"refh_present_to_texture failed: {rc}")
        return out if rc == 1 else None

    def read_target(self):
        """The render target texture's pixels (render_target viewports)."""
        s = self.scene
        out = np.zeros((s.height, s.width, 4), np.uint8)
        rc = self.L.refh_read_target(self.h, out.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"refh_read_target failed: {rc}")
        return out

    def pick(self, xy: np.ndarray):
        xy = np.ascontiguousarray(xy, np.int32)
        n = xy.shape[0]
        ids = np.zeros(n, np.uint32)
        dep = np.zeros(n, np.float32)
        hits = np.zeros(n, np.int32)
        self.L.refh_pick(self.h, n, xy.ctypes.data, ids.ctypes.data, dep.ctypes.data, hits.ctypes.data)
        return ids, dep, hits

    def env_maps(self):
        ptrs = [C.c_void_p() for _ in range(3)]
        ints = [C.c_int32() for _ in range(7)]
        irr, pf, brdf = ptrs
        iw, ih, pw, ph, lv, bs = ints[:6]
        rc = self.L.refh_env_maps(self.h, C.byref(irr), C.byref(iw), C.byref(ih), C.byref(pf),
                                 C.byref(pw), C.byref(ph), C.byref(lv), C.byref(brdf), C.byref(bs))
        if rc != 0:
            return None

        def arr(p, n):
            return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_float)), shape=(n,)).copy()

        pf_total = 0
        for l in range(lv.value):
            pf_total += max(1, pw.value >> l) * max(1, ph.value >> l)
        return {
            "irr": arr(irr, iw.value * ih.value * 4), "irr_w": iw.value, "irr_h": ih.value,
            "pf": arr(pf, pf_total * 4), "pf_w": pw.value, "pf_h": ph.value, "pf_levels": lv.value,
            "brdf": arr(brdf, bs.value * bs.value * 4), "brdf_size": bs.value,
            "rotation": self.scene.env_rotation,
            "intensity": self.scene.env_intensity if self.scene.env_intensity > 0 else 1.0,
        }

    def save_scene(self, path, quantize: bool) -> None:
        """mop_scene_save of this viewport."""
        if self.L.refh_scene_save(self.h, str(path).encode(), 1 if quantize else 0) != 0:
            raise RuntimeError("mop_scene_save failed")

    def env_hdr(self):
        """The environment map the reference computed its IBL maps from
        (float32 [h, w, 4]), or None."""
        p, w, h = C.c_void_p(), C.c_int32(), C.c_int32()
        if self.L.refh_env_hdr(self.h, C.byref(p), C.byref(w), C.byref(h)) != 0:
            return None
        n = w.value * h.value * 4
        a = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_float)), shape=(n,)).copy()
        return a.reshape(h.value, w.value, 4)

    def time_environment(self, reps: int) -> float:
        return self.L.refh_time_environment(self.h, reps)

    def time_frames(self, warm: int, frames: int) -> float:
        return self.L.refh_time_frames(self.h, warm, frames)

    @property
    def threads(self) -> int:
        return self.L.refh_num_threads(self.h)

    def close(self):
        if self.h:
            self.L.refh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def deform_probe(vertices: np.ndarray, vertex_count: int, bones=None, targets=None,
                 weights=None) -> np.ndarray:
    """The reference core's own skinning / morph of one mesh (layout: position
    @0, normal @12, joints ubyte4 @24, weights float4 @28, stride 44), read
    back from the CPU backend's vertex buffer."""
    L = lib()
    v = np.ascontiguousarray(vertices, np.uint8)
    out = np.zeros(vertex_count * 44, np.uint8)
    b = None if bones is None else np.ascontiguousarray(bones, np.float32).reshape(-1)
    t = None if targets is None else np.ascontiguousarray(targets, np.float32).reshape(-1)
    w = None if weights is None else np.ascontiguousarray(weights, np.float32)
    rc = L.refh_deform_probe(v.ctypes.data, vertex_count,
                             b.ctypes.data if b is not None else None,
                             b.size // 16 if b is not None else 0,
                             t.ctypes.data if t is not None else None,
                             w.ctypes.data if w is not None else None,
                             w.size if w is not None else 0, out.ctypes.data)
    if rc != 0:
        raise RuntimeError("refh_deform_probe failed")
    return out


def scene_file_mesh(path, idx: int, vcap: int = 1 << 22, icap: int = 1 << 24):
    """mop_scene_load + mop_scene_get_mesh(idx) of the reference: (vertices
    float32 [V, 12], indices uint32, bbox float32 [6])."""
    v = np.zeros((vcap, 12), np.float32)
    i = np.zeros(icap, np.uint32)
    vc, ic = C.c_uint32(), C.c_uint32()
    bb = np.zeros(6, np.float32)
    rc = lib().refh_scene_file_mesh(str(path).encode(), idx, v.ctypes.data, vcap, i.ctypes.data,
                                    icap, C.byref(vc), C.byref(ic), bb.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"reference mop_scene_get_mesh failed ({rc})")
    return v[:vc.value].copy(), i[:ic.value].copy(), bb


def time_scene_file(path, reps: int = 3) -> float:
    """Median ms of the reference's mop_scene_load + every mop_scene_get_mesh."""
    return lib().refh_time_scene_file(str(path).encode(), reps)


def bc_decode(t, backend: str = "cpu"):
    """A scenes.CompressedTexture through the backend's texture_create_ex and
    texture_read_rgba8 (the reference CPU backend, or the CUDA backend's RHI
    table in the drop-in library): RGBA8 [h, w, 4], or None when the backend
    refuses the format."""
    L = lib(backend)
    out = np.zeros((t.height, t.width, 4), np.uint8)
    d = np.ascontiguousarray(t.data, np.uint8)
    rc = L.refh_bc_decode(0 if backend == "cpu" else BACKEND_CUDA, t.format, t.width, t.height,
                          d.ctypes.data, d.size, out.ctypes.data)
    return out if rc == 0 else None
