"""ctypes binding of the CUDA backend's C ABI (include/mop_cuda.h).

This is the host-side mirror of the reference's viewport/RHI usage for the
frame path: a ``SceneRenderer`` uploads a scene once (mop_viewport_add_mesh ->
buffer_create, mop_viewport_create_texture -> texture_create), then each frame
issues frame_begin / one draw per mesh (EMIT_DRAW, reference
src/core/viewport.c:2015-2088) / frame_end, and reads back colour, depth,
object IDs and picks.  All arithmetic runs in libmopcuda.so; there is no
Python or CPU fallback — if the native library or a GPU is missing, this
module raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libmopcuda.so"

OK, EINVAL, ENOMEM, ECUDA, ETIMEOUT, EUNSUPPORTED = 0, -1, -2, -3, -4, -5
POST_GAMMA, POST_TONEMAP, POST_VIGNETTE, POST_FXAA = 1, 2, 4, 16
DEFAULT_LIGHT_DIR = (0.3, 1.0, 0.5)  # viewport default light_dir (viewport.c:641)


class MopCudaLight(C.Structure):
    _fields_ = [("type", C.c_int32), ("position", C.c_float * 3), ("direction", C.c_float * 3),
                ("color", C.c_float * 4), ("intensity", C.c_float), ("range", C.c_float),
                ("spot_inner_cos", C.c_float), ("spot_outer_cos", C.c_float),
                ("active", C.c_int32)]


class MopCudaVertexLayout(C.Structure):
    _fields_ = [("stride", C.c_uint32), ("position_offset", C.c_int32),
                ("position_components", C.c_int32), ("normal_offset", C.c_int32),
                ("normal_components", C.c_int32), ("color_offset", C.c_int32),
                ("color_components", C.c_int32), ("uv_offset", C.c_int32),
                ("uv_components", C.c_int32)]


class MopCudaDraw(C.Structure):
    _fields_ = [("vertex_buffer", C.c_void_p), ("index_buffer", C.c_void_p),
                ("vertex_count", C.c_uint32), ("index_count", C.c_uint32),
                ("object_id", C.c_uint32), ("model", C.c_float * 16), ("mvp", C.c_float * 16),
                ("light_dir", C.c_float * 3), ("ambient", C.c_float), ("opacity", C.c_float),
                ("metallic", C.c_float), ("roughness", C.c_float), ("depth_bias", C.c_float),
                ("cam_eye", C.c_float * 3), ("smooth", C.c_int32), ("wireframe", C.c_int32),
                ("depth_test", C.c_int32), ("depth_write", C.c_int32),
                ("backface_cull", C.c_int32), ("blend_mode", C.c_int32),
                ("texture", C.c_void_p), ("lights", C.POINTER(MopCudaLight)),
                ("light_count", C.c_uint32), ("layout", C.POINTER(MopCudaVertexLayout))]


class MopCudaShadowCaster(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("vertex_count", C.c_uint32), ("stride", C.c_uint32),
                ("indices", C.c_void_p), ("index_count", C.c_uint32), ("model", C.c_float * 16)]


# the model matrices of a MopCudaShadowCaster array, as a numpy view
_CASTER_MODELS = np.dtype({"names": ["model"], "formats": [(np.float32, 16)],
                           "offsets": [MopCudaShadowCaster.model.offset],
                           "itemsize": C.sizeof(MopCudaShadowCaster)})


class MopCudaDeformLayout(C.Structure):
    _fields_ = [("stride", C.c_uint32), ("position_offset", C.c_int32),
                ("normal_offset", C.c_int32), ("joints_offset", C.c_int32),
                ("weights_offset", C.c_int32)]


class MopCudaView(C.Structure):
    _fields_ = [("view", C.c_float * 16), ("proj", C.c_float * 16), ("eye", C.c_float * 3),
                ("width", C.c_int), ("height", C.c_int), ("ssaa", C.c_int),
                ("clear", C.c_float * 4)]


class MopCudaBatchConfig(C.Structure):
    _fields_ = [("small_side", C.c_int), ("small_area", C.c_int), ("vertex_block", C.c_int),
                ("setup_block", C.c_int), ("raster_block", C.c_int), ("large_block", C.c_int),
                ("shade_block", C.c_int), ("grid_mul", C.c_int)]


BATCH_COLOR, BATCH_PRESENTED, BATCH_DEPTH, BATCH_IDS = 0, 1, 2, 3
REQ_RENDER, REQ_PICK = 0, 1


class MopCudaServerConfig(C.Structure):
    _fields_ = [("hbm_budget", C.c_uint64), ("max_views", C.c_uint32),
                ("max_inflight", C.c_uint32), ("batch_window_us", C.c_uint32),
                ("max_launch_samples", C.c_uint64)]


class MopCudaRequest(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("scene", C.c_uint32), ("view", MopCudaView),
                ("color", C.c_void_p), ("ids", C.c_void_p), ("depth", C.c_void_p),
                ("pick_xy", C.c_void_p), ("pick_n", C.c_uint32), ("pick_ids", C.c_void_p),
                ("pick_depths", C.c_void_p), ("pick_hits", C.c_void_p)]


class MopCudaServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("launches", C.c_uint64), ("launched_views", C.c_uint64),
                ("reruns", C.c_uint64), ("peak_inflight_bytes", C.c_uint64),
                ("device_bytes", C.c_uint64), ("max_views_in_launch", C.c_uint32),
                ("pad", C.c_uint32)]

# (name, restype, argtypes) for every entry point of include/mop_cuda.h
_P = C.c_void_p
SIGNATURES = [
    ("mopcuda_device_create", _P, [C.c_int]),
    ("mopcuda_device_destroy", None, [_P]),
    ("mopcuda_last_error", C.c_char_p, []),
    ("mopcuda_launch_count", C.c_uint64, [_P]),
    ("mopcuda_buffer_create", _P, [_P, _P, C.c_size_t]),
    ("mopcuda_buffer_destroy", None, [_P, _P]),
    ("mopcuda_buffer_update", C.c_int, [_P, _P, _P, C.c_size_t, C.c_size_t]),
    ("mopcuda_buffer_read", _P, [_P]),
    ("mopcuda_buffer_copy_to_host", C.c_int, [_P, _P, C.c_size_t, _P, C.c_size_t]),
    ("mopcuda_buffer_size", C.c_size_t, [_P]),
    ("mopcuda_texture_create", _P, [_P, C.c_int, C.c_int, _P]),
    ("mopcuda_texture_create_hdr", _P, [_P, C.c_int, C.c_int, _P]),
    ("mopcuda_texture_destroy", None, [_P, _P]),
    ("mopcuda_texture_read_rgba8", C.c_int, [_P, _P, _P, C.c_size_t]),
    ("mopcuda_texture_create_ex", _P, [_P, C.c_int, C.c_int, C.c_int, C.c_int, _P, C.c_size_t]),
    ("mopcuda_framebuffer_create", _P, [_P, C.c_int, C.c_int]),
    ("mopcuda_framebuffer_destroy", None, [_P, _P]),
    ("mopcuda_framebuffer_resize", C.c_int, [_P, _P, C.c_int, C.c_int]),
    ("mopcuda_framebuffer_set_ssaa", C.c_int, [_P, C.c_int]),
    ("mopcuda_framebuffer_copy_to_texture", C.c_int, [_P, _P, _P]),
    ("mopcuda_framebuffer_create_from_texture", _P, [_P, _P, C.c_int, C.c_int]),
    ("mopcuda_set_exposure", None, [_P, C.c_float]),
    ("mopcuda_set_post_effects", None, [_P, C.c_uint32]),
    ("mopcuda_set_fog", C.c_int, [_P, C.POINTER(C.c_float), C.c_float, C.c_float]),
    ("mopcuda_set_ibl", C.c_int, [_P, _P, C.c_int, C.c_int, _P, C.c_int, C.c_int, C.c_int, _P,
                                  C.c_int, C.c_float, C.c_float]),
    ("mopcuda_skin_apply", C.c_int, [_P, _P, _P, C.c_uint32, C.POINTER(MopCudaDeformLayout),
                                     _P, C.c_uint32]),
    ("mopcuda_morph_apply", C.c_int, [_P, _P, _P, C.c_uint32, C.POINTER(MopCudaDeformLayout),
                                      _P, _P, C.c_uint32]),
    ("mopcuda_ibl_from_env", C.c_int, [_P, _P, C.c_int, C.c_int, C.c_float, C.c_float]),
    ("mopcuda_ibl_procedural_sky", C.c_int, [_P, _P, C.c_float, C.c_float, C.c_float,
                                             C.c_float]),
    ("mopcuda_ibl_gpu_time_ms", C.c_float, [_P]),
    ("mopcuda_ibl_read", C.c_int, [_P, _P, C.c_size_t, _P, C.c_size_t, _P, C.c_size_t, _P,
                                   C.c_size_t]),
    ("mopcuda_scene_file_open", _P, [C.c_char_p]),
    ("mopcuda_scene_file_close", None, [_P]),
    ("mopcuda_scene_file_mesh_count", C.c_uint32, [_P]),
    ("mopcuda_scene_file_light_count", C.c_uint32, [_P]),
    ("mopcuda_scene_file_camera", C.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    ("mopcuda_scene_file_light", C.c_int, [_P, C.c_uint32, C.POINTER(MopCudaLight)]),
    ("mopcuda_scene_file_upload_mesh", C.c_int, [_P, _P, C.c_uint32, C.c_uint32,
                                                 C.POINTER(_P), C.POINTER(_P),
                                                 C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                                 _P, _P]),
    ("mopcuda_scene_file_upload_all", C.c_int, [_P, _P, C.c_uint32, _P, _P, _P, _P]),
    ("mopcuda_shadow_begin", C.c_int, [_P, C.c_int, _P]),
    ("mopcuda_shadow_draw", C.c_int, [_P, _P, C.c_uint32, C.c_uint32, _P, C.c_uint32, _P]),
    ("mopcuda_shadow_draw_list", C.c_int, [_P, C.POINTER(MopCudaShadowCaster), C.c_uint32]),
    ("mopcuda_shadow_end", C.c_int, [_P]),
    ("mopcuda_shadow_clear", C.c_int, [_P]),
    ("mopcuda_shadow_gpu_time_ms", C.c_float, [_P]),
    ("mopcuda_shadow_read", C.c_int, [_P, _P, C.c_size_t]),
    ("mopcuda_frame_begin", C.c_int, [_P, _P, _P]),
    ("mopcuda_draw", C.c_int, [_P, _P, C.POINTER(MopCudaDraw)]),
    ("mopcuda_draw_list", C.c_int, [_P, _P, _P, C.c_uint32]),
    ("mopcuda_draw_instanced", C.c_int, [_P, _P, C.POINTER(MopCudaDraw), _P, _P, _P, C.c_uint32]),
    ("mopcuda_draw_background", C.c_int, [_P, _P, _P, _P, _P, _P, C.c_float, C.c_float,
                                          C.c_float]),
    ("mopcuda_draw_skybox", C.c_int, [_P, _P, _P, _P, _P, C.c_float, C.c_float]),
    ("mopcuda_frame_end", C.c_int, [_P, _P]),
    ("mopcuda_frame_wait", C.c_int, [_P, C.c_int]),
    ("mopcuda_frame_gpu_time_ms", C.c_float, [_P]),
    ("mopcuda_read_color", _P, [_P, _P, _P, _P]),
    ("mopcuda_read_object_id", _P, [_P, _P, _P, _P]),
    ("mopcuda_read_depth", _P, [_P, _P, _P, _P]),
    ("mopcuda_read_color_resolved", C.c_int, [_P, _P, C.c_int, _P, C.c_size_t]),
    ("mopcuda_read_color_resolved_async", C.c_int, [_P, _P, C.c_int, _P, C.c_size_t]),
    ("mopcuda_readback_wait", C.c_int, [_P, _P, C.c_int]),
    ("mopcuda_pick_read_id", C.c_uint32, [_P, _P, C.c_int, C.c_int]),
    ("mopcuda_pick_read_depth", C.c_float, [_P, _P, C.c_int, C.c_int]),
    ("mopcuda_pick_batch", C.c_int, [_P, _P, C.c_int, _P, C.c_uint32, _P, _P, _P]),
    ("mopcuda_pick_batch_noalloc", C.c_int, [_P, _P, C.c_int, _P, C.c_uint32, _P, _P, _P]),
    ("mopcuda_set_stage_timing", None, [_P, C.c_int]),
    ("mopcuda_stage_times", C.c_int, [_P, _P, C.c_int]),
    ("mopcuda_measure_fp32_peak", C.c_int, [_P, C.POINTER(C.c_double)]),
    ("mopcuda_frame_io_bytes", C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("mopcuda_scene_create", _P, [_P]),
    ("mopcuda_scene_set_shadow", C.c_int, [_P, C.c_int, _P]),
    ("mopcuda_scene_destroy", None, [_P]),
    ("mopcuda_scene_add_draw", C.c_int, [_P, C.POINTER(MopCudaDraw)]),
    ("mopcuda_scene_set_model", C.c_int, [_P, C.c_uint32, _P]),
    ("mopcuda_scene_draw_count", C.c_uint32, [_P]),
    ("mopcuda_scene_triangle_count", C.c_uint64, [_P]),
    ("mopcuda_batch_create", _P, [_P, C.POINTER(MopCudaView), C.c_uint32]),
    ("mopcuda_batch_destroy", None, [_P]),
    ("mopcuda_batch_set_views", C.c_int, [_P, C.POINTER(MopCudaView), C.c_uint32]),
    ("mopcuda_batch_submit", C.c_int, [_P]),
    ("mopcuda_batch_wait", C.c_int, [_P, C.c_int]),
    ("mopcuda_batch_gpu_time_ms", C.c_float, [_P]),
    ("mopcuda_batch_read", C.c_int, [_P, C.c_uint32, C.c_int, _P, C.c_size_t]),
    ("mopcuda_batch_read_views", C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_int,
                                           C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]),
    ("mopcuda_batch_read_views_async", C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_int,
                                                 C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]),
    ("mopcuda_batch_readback_wait", C.c_int, [_P, C.c_int]),
    ("mopcuda_batch_pick", C.c_int, [_P, C.c_uint32, _P, C.c_uint32, _P, _P, _P]),
    ("mopcuda_batch_get_config", C.c_int, [_P, C.POINTER(MopCudaBatchConfig)]),
    ("mopcuda_batch_set_config", C.c_int, [_P, C.POINTER(MopCudaBatchConfig)]),
    ("mopcuda_batch_autotune", C.c_int, [_P, C.c_int, C.c_char_p, C.c_size_t]),
    ("mopcuda_batch_device_bytes", C.c_uint64, [_P]),
    ("mopcuda_server_create", _P, [_P, C.POINTER(MopCudaServerConfig)]),
    ("mopcuda_server_destroy", None, [_P]),
    ("mopcuda_server_add_scene", C.c_int, [_P, _P]),
    ("mopcuda_server_submit", C.c_int, [_P, C.POINTER(MopCudaRequest), C.POINTER(C.c_uint64)]),
    ("mopcuda_server_wait", C.c_int, [_P, C.c_uint64, C.c_int, C.POINTER(C.c_double)]),
    ("mopcuda_server_drain", C.c_int, [_P, C.c_int]),
    ("mopcuda_server_stats", C.c_int, [_P, C.POINTER(MopCudaServerStats)]),
    ("mopcuda_host_alloc", _P, [C.c_size_t]),
    ("mopcuda_host_free", None, [_P]),
    ("mopcuda_mat4_multiply", None, [_P, _P, _P]),
    ("mopcuda_mat4_compose_trs", None, [_P, _P, _P, _P]),
    ("mopcuda_camera_matrices", None, [_P, _P, _P, C.c_float, C.c_float, C.c_float, C.c_int,
                                       C.c_int, _P, _P, _P]),
    ("mopcuda_camera_orbit", None, [_P, _P, _P, _P, _P]),
    ("mopcuda_shadow_light_vp", C.c_int, [_P, C.c_uint32, _P, _P]),
]

_lib = None


def lib():
    """Load libmopcuda.so (built in-tree by __graft_entry__.build / make)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"CUDA backend library missing: {LIB_PATH} (run the build)")
        L = C.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return lib().mopcuda_last_error().decode(errors="replace")


class MopCudaError(RuntimeError):
    def __init__(self, code, what):
        super().__init__(f"{what} failed ({code}): {last_error()}")
        self.code = code


def _check(rc, what):
    if rc != OK:
        raise MopCudaError(rc, what)
    return rc


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


# --------------------------------------------------------------------------
# host matrices (run in libmopcuda.so host code)
# --------------------------------------------------------------------------

def mat4_multiply(a, b):
    a, b = _f32(a), _f32(b)
    out = np.zeros(16, np.float32)
    lib().mopcuda_mat4_multiply(a.ctypes.data, b.ctypes.data, out.ctypes.data)
    return out


def camera_matrices(scene):
    """View, projection and eye of a scene's (or a View's) camera."""
    view = np.zeros(16, np.float32)
    proj = np.zeros(16, np.float32)
    eye = np.zeros(3, np.float32)
    e, t, u = _f32(scene.eye), _f32(scene.target), _f32(scene.up)
    lib().mopcuda_camera_matrices(e.ctypes.data, t.ctypes.data, u.ctypes.data, scene.fov_deg,
                                  scene.near, scene.far, scene.width, scene.height,
                                  view.ctypes.data, proj.ctypes.data, eye.ctypes.data)
    return view, proj, eye


def light_struct(l) -> MopCudaLight:
    s = MopCudaLight()
    s.type = l.type
    s.position[:] = l.position
    s.direction[:] = l.direction
    s.color[:] = l.color
    s.intensity = l.intensity
    s.range = l.range
    s.spot_inner_cos = l.spot_inner_cos
    s.spot_outer_cos = l.spot_outer_cos
    s.active = 1 if l.active else 0
    return s


class Device:
    def __init__(self, ordinal: int = 0):
        self.L = lib()
        self.h = self.L.mopcuda_device_create(ordinal)
        if not self.h:
            raise RuntimeError(f"mopcuda_device_create({ordinal}) failed: {last_error()}")

    @property
    def launches(self) -> int:
        return int(self.L.mopcuda_launch_count(self.h))

    STAGES = ("vertex", "setup_clip", "raster", "resolve", "shade", "post")

    def set_stage_timing(self, on: bool = True):
        self.L.mopcuda_set_stage_timing(self.h, 1 if on else 0)

    def stage_times(self):
        ms = np.zeros(len(self.STAGES), np.float32)
        _check(self.L.mopcuda_stage_times(self.h, ms.ctypes.data, ms.size), "stage_times")
        return dict(zip(self.STAGES, [float(x) for x in ms]))

    def frame_io_bytes(self):
        h, d = C.c_uint64(), C.c_uint64()
        _check(self.L.mopcuda_frame_io_bytes(self.h, C.byref(h), C.byref(d)), "frame_io_bytes")
        return int(h.value), int(d.value)

    def fp32_peak_gops(self) -> float:
        g = C.c_double()
        _check(self.L.mopcuda_measure_fp32_peak(self.h, C.byref(g)), "measure_fp32_peak")
        return float(g.value)

    def ibl_procedural_sky(self, sun_dir, turbidity, ground_albedo, rotation=0.0,
                           intensity=1.0):
        """The procedural sky and its IBL maps computed on the device and
        bound (mop_viewport_set_procedural_sky + set_environment)."""
        sd = (C.c_float * 3)(*sun_dir)
        _check(self.L.mopcuda_ibl_procedural_sky(self.h, sd, turbidity, ground_albedo, rotation,
                                                 intensity), "ibl_procedural_sky")

    def ibl_from_env(self, env, rotation=0.0, intensity=1.0):
        """IBL maps computed on the device from an RGBA32F equirect map
        [h, w, 4] and bound."""
        env = np.ascontiguousarray(env, np.float32)
        _check(self.L.mopcuda_ibl_from_env(self.h, env.ctypes.data, env.shape[1], env.shape[0],
                                           rotation, intensity), "ibl_from_env")

    @property
    def ibl_gpu_ms(self) -> float:
        return float(self.L.mopcuda_ibl_gpu_time_ms(self.h))

    def ibl_maps(self, env_shape=None):
        """The bound maps in the dictionary form of set_ibl's arguments (and
        the environment map when env_shape = (h, w) is given)."""
        irr = np.zeros((32, 64, 4), np.float32)
        n_pf = sum(max(1, 128 >> l) * max(1, 64 >> l) for l in range(5))
        pf = np.zeros(n_pf * 4, np.float32)
        brdf = np.zeros((256, 256, 4), np.float32)
        env = np.zeros(tuple(env_shape) + (4,), np.float32) if env_shape else None
        _check(self.L.mopcuda_ibl_read(self.h, irr.ctypes.data, irr.nbytes, pf.ctypes.data,
                                       pf.nbytes, brdf.ctypes.data, brdf.nbytes,
                                       env.ctypes.data if env is not None else None,
                                       env.nbytes if env is not None else 0), "ibl_read")
        out = {"irr": irr.reshape(-1), "irr_w": 64, "irr_h": 32, "pf": pf, "pf_w": 128,
               "pf_h": 64, "pf_levels": 5, "brdf": brdf.reshape(-1), "brdf_size": 256}
        if env is not None:
            out["env"] = env
        return out

    def close(self):
        if self.h:
            self.L.mopcuda_device_destroy(self.h)
            self.h = None


class _Resident:
    """A scene's meshes, textures, lights and device state uploaded through
    the C ABI (mop_viewport_add_mesh -> buffer_create, create_texture ->
    texture_create, set_exposure / set_post_effects / set_ibl)."""

    def __init__(self, device: Device, scene, ibl=None, preloaded=None):
        """preloaded: the meshes' device buffers already made (one
        scene_file.upload entry per mesh, in mesh order) instead of uploading
        scene.meshes' arrays."""
        self.dev = device
        self.scene = scene
        L = device.L
        d = device.h
        self.L = L
        self._buffers = []
        self.meshes = []
        for k, m in enumerate(scene.meshes):
            if preloaded is not None:
                p = preloaded[k]
                vb, ib, vc, ic = p["vertices"], p["indices"], p["vertex_count"], p["index_count"]
            else:
                v = _f32(m.vertices)
                i = np.ascontiguousarray(m.indices, np.uint32)
                vb = L.mopcuda_buffer_create(d, v.ctypes.data, v.nbytes)
                ib = L.mopcuda_buffer_create(d, i.ctypes.data, i.nbytes)
                if not vb or not ib:
                    raise RuntimeError(f"buffer_create failed: {last_error()}")
                vc, ic = v.shape[0], i.size
            self._buffers += [vb, ib]
            self.meshes.append((m, vb, ib, vc, ic))
        # instanced meshes (mop_viewport_add_instanced_mesh): buffers + transforms
        self.instanced = []
        for im in getattr(scene, "instanced", []):
            v = _f32(im.vertices)
            i = np.ascontiguousarray(im.indices, np.uint32)
            vb = L.mopcuda_buffer_create(d, v.ctypes.data, v.nbytes)
            ib = L.mopcuda_buffer_create(d, i.ctypes.data, i.nbytes)
            if not vb or not ib:
                raise RuntimeError(f"buffer_create failed: {last_error()}")
            self._buffers += [vb, ib]
            tr = np.ascontiguousarray(np.asarray(im.transforms, np.float32).reshape(-1, 16))
            self.instanced.append((im, vb, ib, v.shape[0], i.size, tr))
        self.textures = []
        for t in scene.textures:
            if hasattr(t, "format"):  # block-compressed: texture_create_ex decodes on the device
                b = np.ascontiguousarray(t.data, np.uint8)
                th = L.mopcuda_texture_create_ex(d, t.width, t.height, t.format, 1, b.ctypes.data,
                                                 b.size)
                if not th:
                    raise RuntimeError(f"texture_create_ex failed: {last_error()}")
                self.textures.append(th)
                continue
            t = np.ascontiguousarray(t, np.uint8)
            th = L.mopcuda_texture_create(d, t.shape[1], t.shape[0], t.ctypes.data)
            if not th:
                raise RuntimeError(f"texture_create failed: {last_error()}")
            self.textures.append(th)
        # environment background (mop_viewport_set_environment_background): the
        # environment map as an HDR texture, drawn behind every frame
        self.env_tex = None
        if getattr(scene, "env_background", False) and ibl is not None and "env" in ibl:
            env = _f32(ibl["env"])
            self._env = env
            self.env_tex = L.mopcuda_texture_create_hdr(d, env.shape[1], env.shape[0],
                                                        env.ctypes.data)
            if not self.env_tex:
                raise RuntimeError(f"texture_create_hdr failed: {last_error()}")
            self.textures.append(self.env_tex)
        L.mopcuda_set_exposure(d, scene.exposure)
        L.mopcuda_set_post_effects(d, scene.post_effects)
        # mop_viewport_set_fog; a scene without fog keeps a new viewport's zeros
        fog = getattr(scene, "fog", None)
        fc, fnear, ffar = (fog[0], fog[1], fog[2]) if fog is not None else ((0, 0, 0, 0), 0, 0)
        _check(L.mopcuda_set_fog(d, (C.c_float * 4)(*[float(x) for x in fc]), float(fnear),
                                 float(ffar)), "set_fog")
        if ibl is not None:
            self.set_ibl(ibl)
        else:
            _check(L.mopcuda_set_ibl(d, None, 0, 0, None, 0, 0, 0, None, 0, 0.0, 1.0), "set_ibl")
        self.lights = (MopCudaLight * max(1, len(scene.lights)))()
        for k, l in enumerate(scene.lights):
            self.lights[k] = light_struct(l)
        # the device's shadow binding outlives a scene: start unbound
        _check(L.mopcuda_shadow_clear(d), "shadow_clear")
        self._shadow_bound = False
        self._caster_key, self._caster_arr, self._caster_models = None, None, None

    def set_ibl(self, ibl):
        self._ibl = [_f32(ibl["irr"]), _f32(ibl["pf"]), _f32(ibl["brdf"])]
        irr, pf, brdf = self._ibl
        _check(self.L.mopcuda_set_ibl(self.dev.h, irr.ctypes.data, ibl["irr_w"], ibl["irr_h"],
                                      pf.ctypes.data, ibl["pf_w"], ibl["pf_h"], ibl["pf_levels"],
                                      brdf.ctypes.data, ibl["brdf_size"], ibl["rotation"],
                                      ibl["intensity"]), "set_ibl")

    def draw_struct(self, k, view=None, proj=None, eye=None) -> MopCudaDraw:
        """EMIT_DRAW's draw call for mesh k (mvp = proj * (view * model))."""
        sc = self.scene
        m, vb, ib, vc, ic = self.meshes[k]
        dr = MopCudaDraw()
        dr.vertex_buffer, dr.index_buffer = vb, ib
        dr.vertex_count, dr.index_count = vc, ic
        dr.object_id = m.object_id
        dr.model[:] = [float(x) for x in m.transform]
        if view is not None:
            dr.mvp[:] = [float(x) for x in mat4_multiply(proj, mat4_multiply(view, m.transform))]
            dr.cam_eye[:] = [float(x) for x in eye]
        dr.light_dir[:] = DEFAULT_LIGHT_DIR
        dr.ambient = min(max(sc.ambient, 0.0), 1.0)
        dr.opacity = m.opacity
        dr.metallic = m.metallic if m.has_material else 0.0
        dr.roughness = m.roughness if m.has_material else 0.5
        dr.depth_bias = 0.0
        dr.smooth = 1 if getattr(sc, "smooth", True) else 0
        # MOP_RENDER_WIREFRAME: every mesh but ID 0 (EMIT_DRAW, viewport.c:2056-2057)
        dr.wireframe = 1 if getattr(sc, "wireframe", False) and m.object_id != 0 else 0
        dr.depth_test = dr.depth_write = dr.backface_cull = 1
        dr.blend_mode = getattr(m, "blend_mode", 0) or (1 if m.opacity < 1.0 else 0)
        dr.texture = self.textures[m.texture] if m.texture >= 0 else None
        dr.lights = self.lights
        dr.light_count = len(sc.lights)
        dr.layout = None
        if m.object_id >= 0xFFFD0000:  # chrome (EMIT_DRAW, reference viewport.c:2035-2076)
            dr.depth_test = dr.backface_cull = 0
            dr.lights, dr.light_count = None, 0
            dr.ambient = 1.0
        return dr

    def instanced_struct(self, k) -> MopCudaDraw:
        """pass_instanced's draw call for instanced mesh k (reference
        viewport.c:2613-2641): identity model and mvp (replaced per instance),
        the default material, no texture, culling only for a non-zero ID,
        depth test with the depth write off, cam_eye left at zero."""
        sc = self.scene
        im, vb, ib, vc, ic, _ = self.instanced[k]
        dr = MopCudaDraw()
        dr.vertex_buffer, dr.index_buffer = vb, ib
        dr.vertex_count, dr.index_count = vc, ic
        dr.object_id = im.object_id
        ident = [1.0, 0, 0, 0, 0, 1.0, 0, 0, 0, 0, 1.0, 0, 0, 0, 0, 1.0]
        dr.model[:] = ident
        dr.mvp[:] = ident
        dr.cam_eye[:] = [0.0, 0.0, 0.0]
        dr.light_dir[:] = DEFAULT_LIGHT_DIR
        dr.ambient = min(max(sc.ambient, 0.0), 1.0)
        dr.opacity = 1.0
        dr.metallic, dr.roughness = 0.0, 0.5
        dr.depth_bias = 0.0
        dr.smooth = 1 if getattr(sc, "smooth", True) else 0
        dr.wireframe = 1 if getattr(sc, "wireframe", False) and im.object_id != 0 else 0
        dr.depth_test, dr.depth_write = 1, 0
        dr.backface_cull = 1 if im.object_id != 0 else 0
        dr.blend_mode = 0
        dr.texture = None
        dr.lights = self.lights
        dr.light_count = len(sc.lights)
        dr.layout = None
        return dr

    def close_resident(self):
        L, d = self.L, self.dev.h
        if not d:
            return
        for b in self._buffers:
            L.mopcuda_buffer_destroy(d, b)
        for t in self.textures:
            L.mopcuda_texture_destroy(d, t)
        self._buffers, self.textures = [], []


class SceneRenderer(_Resident):
    """Scene resident on one device; renders frames through the C ABI."""

    def __init__(self, device: Device, scene, ibl=None, preloaded=None):
        super().__init__(device, scene, ibl, preloaded)
        L, d = self.L, device.h
        self.sw, self.sh = scene.width * scene.ssaa, scene.height * scene.ssaa
        self.fb = L.mopcuda_framebuffer_create(d, self.sw, self.sh)
        if not self.fb:
            raise RuntimeError(f"framebuffer_create failed: {last_error()}")
        _check(L.mopcuda_framebuffer_set_ssaa(self.fb, scene.ssaa), "framebuffer_set_ssaa")
        self.update_camera()
        self.clear = (C.c_float * 4)(*scene.clear)

    def set_view(self, v):
        """Re-targets the frame to a viewport of another size / SSAA / camera
        (framebuffer_resize, then new per-draw matrices)."""
        import dataclasses
        self.scene = dataclasses.replace(self.scene, width=v.width, height=v.height, ssaa=v.ssaa,
                                         eye=v.eye, target=v.target, up=v.up, fov_deg=v.fov_deg,
                                         near=v.near, far=v.far, clear=v.clear)
        sc = self.scene
        self.sw, self.sh = sc.width * sc.ssaa, sc.height * sc.ssaa
        _check(self.L.mopcuda_framebuffer_resize(self.dev.h, self.fb, self.sw, self.sh),
               "framebuffer_resize")
        _check(self.L.mopcuda_framebuffer_set_ssaa(self.fb, sc.ssaa), "framebuffer_set_ssaa")
        self.clear = (C.c_float * 4)(*sc.clear)
        self.update_camera()

    def update_camera(self):
        import scenes
        self.view, self.proj, self.eye = camera_matrices(self.scene)
        # the core's pass order: opaque meshes, then blended ones back to front
        self.draws = [self.draw_struct(k, self.view, self.proj, self.eye)
                      for k in scenes.draw_order(self.scene, self.eye)]
        self.draw_array = (MopCudaDraw * max(1, len(self.draws)))(*self.draws)
        self.inst_draws = [self.instanced_struct(k) for k in range(len(self.instanced))]
        sc = self.scene
        self._orbit_eye = np.zeros(3, np.float32)
        self._orbit_up = np.zeros(3, np.float32)
        # the inputs stay referenced until the call returns
        eye_in, target_in, up_in = _f32(sc.eye), _f32(sc.target), _f32(sc.up)
        self.L.mopcuda_camera_orbit(eye_in.ctypes.data, target_in.ctypes.data, up_in.ctypes.data,
                                    self._orbit_eye.ctypes.data, self._orbit_up.ctypes.data)
        self._target = _f32(sc.target)
        self._view_arr = _f32(self.view)
        self._proj_arr = _f32(self.proj)

    def shadow_pass(self) -> bool:
        """pass_shadow through the C ABI (reference viewport.c:2288-2442):
        the light camera from the casters' world transforms, every caster
        rasterised into the map, the map bound for the following frames.
        Without a casting directional light or a caster the map is unbound."""
        import scenes
        L, d, sc = self.L, self.dev.h, self.scene
        light = scenes.shadow_light(sc)
        casters = scenes.shadow_casters(sc) if light is not None else []
        if light is None or not casters:
            if self._shadow_bound:
                _check(L.mopcuda_shadow_clear(d), "shadow_clear")
                self._shadow_bound = False
            return False
        models = np.concatenate([_f32(sc.meshes[k].transform) for k in casters])
        vp = np.zeros(16, np.float32)
        dr = _f32(light.direction)
        L.mopcuda_shadow_light_vp(models.ctypes.data, len(casters), dr.ctypes.data,
                                  vp.ctypes.data)
        key = tuple(casters)
        if self._caster_key != key:  # the caster array is rebuilt when the set changes
            arr = (MopCudaShadowCaster * len(casters))()
            for j, k in enumerate(casters):
                _, vb, ib, vc, ic = self.meshes[k]
                arr[j].vertices, arr[j].indices = vb, ib
                arr[j].vertex_count, arr[j].index_count, arr[j].stride = vc, ic, 48
            self._caster_arr, self._caster_key = arr, key
            self._caster_models = np.frombuffer(arr, _CASTER_MODELS)["model"]
        self._caster_models[:] = models.reshape(-1, 16)
        _check(L.mopcuda_shadow_begin(d, scenes.SHADOW_MAP_SIZE, vp.ctypes.data), "shadow_begin")
        _check(L.mopcuda_shadow_draw_list(d, self._caster_arr, len(casters)), "shadow_draw_list")
        _check(L.mopcuda_shadow_end(d), "shadow_end")
        self._shadow_bound = True
        return True

    @property
    def shadow_gpu_ms(self) -> float:
        """Device time of the last shadow pass."""
        return float(self.L.mopcuda_shadow_gpu_time_ms(self.dev.h))

    def shadow_map(self):
        """The bound shadow map as float32 [size, size]."""
        import scenes
        n = scenes.SHADOW_MAP_SIZE
        out = np.zeros((n, n), np.float32)
        _check(self.L.mopcuda_shadow_read(self.dev.h, out.ctypes.data, out.nbytes), "shadow_read")
        return out

    def submit(self):
        """Record and launch one frame (asynchronous); the shadow pass first
        when a directional light casts shadows."""
        L, d, fb = self.L, self.dev.h, self.fb
        self.shadow_pass()
        _check(L.mopcuda_frame_begin(d, fb, self.clear), "frame_begin")
        if self.env_tex:  # pass_background before the scene passes
            sc = self.scene
            _check(L.mopcuda_draw_background(d, fb, self.env_tex, self._orbit_eye.ctypes.data,
                                             self._target.ctypes.data, self._orbit_up.ctypes.data,
                                             sc.fov_deg, sc.env_rotation, sc.env_intensity),
                   "draw_background")
        _check(L.mopcuda_draw_list(d, fb, self.draw_array, len(self.draws)), "draw_list")
        # pass_instanced after the transparent pass: one draw per instance
        for dr, (_, _, _, _, _, tr) in zip(self.inst_draws, self.instanced):
            _check(L.mopcuda_draw_instanced(d, fb, C.byref(dr), self._view_arr.ctypes.data,
                                            self._proj_arr.ctypes.data, tr.ctypes.data,
                                            tr.shape[0]), "draw_instanced")
        _check(L.mopcuda_frame_end(d, fb), "frame_end")

    def wait(self, timeout_ms: int = 20000):
        _check(self.L.mopcuda_frame_wait(self.dev.h, timeout_ms), "frame_wait")

    def render(self):
        self.submit()
        self.wait()
        return self

    @property
    def gpu_ms(self) -> float:
        return float(self.L.mopcuda_frame_gpu_time_ms(self.dev.h))

    def _view(self, p, dtype, shape):
        if not p:
            raise RuntimeError(f"readback failed: {last_error()}")
        n = int(np.prod(shape))
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(dtype)), shape=(n,)).reshape(shape).copy()

    def color_full(self):
        return self._view(self.L.mopcuda_read_color(self.dev.h, self.fb, None, None), C.c_uint8,
                          (self.sh, self.sw, 4))

    def depth(self):
        return self._view(self.L.mopcuda_read_depth(self.dev.h, self.fb, None, None), C.c_float,
                          (self.sh, self.sw))

    def object_id(self):
        return self._view(self.L.mopcuda_read_object_id(self.dev.h, self.fb, None, None),
                          C.c_uint32, (self.sh, self.sw))

    def color(self, out=None):
        sc = self.scene
        if out is None:
            out = np.zeros((sc.height, sc.width, 4), np.uint8)
        _check(self.L.mopcuda_read_color_resolved(self.dev.h, self.fb, sc.ssaa, out.ctypes.data,
                                                  out.nbytes), "read_color_resolved")
        return out

    def color_async(self, out):
        """Requests the presented image into `out` (a page-locked uint8
        [height, width, 4] array for a true overlap); it is copied on the
        copy stream once the frame completes, overlapping the next frame."""
        sc = self.scene
        _check(self.L.mopcuda_read_color_resolved_async(self.dev.h, self.fb, sc.ssaa,
                                                        out.ctypes.data, out.nbytes),
               "read_color_resolved_async")

    def wait_readback(self, timeout_ms: int = 20000):
        _check(self.L.mopcuda_readback_wait(self.dev.h, self.fb, timeout_ms), "readback_wait")

    def pick(self, xy):
        xy = np.ascontiguousarray(xy, np.int32)
        n = xy.shape[0]
        ids = np.zeros(n, np.uint32)
        dep = np.zeros(n, np.float32)
        hits = np.zeros(n, np.int32)
        _check(self.L.mopcuda_pick_batch(self.dev.h, self.fb, self.scene.ssaa, xy.ctypes.data, n,
                                         ids.ctypes.data, dep.ctypes.data, hits.ctypes.data),
               "pick_batch")
        return ids, dep, hits

    def close(self):
        L, d = self.L, self.dev.h
        if not d:
            return
        if self.fb:
            L.mopcuda_framebuffer_destroy(d, self.fb)
        self.fb = None
        self.close_resident()


def view_struct(v) -> MopCudaView:
    """MopCudaView of a scenes.View (camera derived as for a frame)."""
    s = MopCudaView()
    view, proj, eye = camera_matrices(v)
    s.view[:] = [float(x) for x in view]
    s.proj[:] = [float(x) for x in proj]
    s.eye[:] = [float(x) for x in eye]
    s.width, s.height, s.ssaa = v.width, v.height, v.ssaa
    s.clear[:] = [float(x) for x in v.clear]
    return s


class ResidentScene(_Resident):
    """A scene uploaded once and recorded as a MopCudaScene (one draw per
    mesh, in mesh order) for batches and servers."""

    def __init__(self, device: Device, scene, ibl=None):
        super().__init__(device, scene, ibl)
        L = self.L
        self.sh_scene = L.mopcuda_scene_create(device.h)
        if not self.sh_scene:
            raise RuntimeError(f"scene_create failed: {last_error()}")
        self._draws = [self.draw_struct(k) for k in range(len(self.meshes))]
        for dr in self._draws:
            rc = L.mopcuda_scene_add_draw(self.sh_scene, C.byref(dr))
            if rc < 0:
                raise MopCudaError(rc, "scene_add_draw")
        # pass_shadow: the first active directional light with cast_shadows
        import scenes as _sc
        light = _sc.shadow_light(scene)
        if light is not None:
            dr_ = _f32(light.direction)
            _check(L.mopcuda_scene_set_shadow(self.sh_scene, _sc.SHADOW_MAP_SIZE,
                                              dr_.ctypes.data), "scene_set_shadow")

    def set_model(self, k: int, model):
        m = _f32(model)
        _check(self.L.mopcuda_scene_set_model(self.sh_scene, k, m.ctypes.data), "scene_set_model")

    @property
    def triangles(self) -> int:
        return int(self.L.mopcuda_scene_triangle_count(self.sh_scene))

    def close(self):
        if getattr(self, "sh_scene", None):
            self.L.mopcuda_scene_destroy(self.sh_scene)
            self.sh_scene = None
        self.close_resident()


class BatchRenderer(ResidentScene):
    """A resident scene rendered into many viewports per graph launch
    (mopcuda_scene_* / mopcuda_batch_*)."""

    def __init__(self, device: Device, scene, views, ibl=None):
        super().__init__(device, scene, ibl)
        L = self.L
        self.views = list(views)
        arr = (MopCudaView * len(self.views))(*[view_struct(v) for v in self.views])
        self.h = L.mopcuda_batch_create(self.sh_scene, arr, len(self.views))
        if not self.h:
            raise RuntimeError(f"batch_create failed: {last_error()}")

    @property
    def samples(self) -> int:
        return sum(v.samples for v in self.views)

    @property
    def pixels(self) -> int:
        return sum(v.pixels for v in self.views)

    def set_views(self, views):
        views = list(views)
        arr = (MopCudaView * len(views))(*[view_struct(v) for v in views])
        _check(self.L.mopcuda_batch_set_views(self.h, arr, len(views)), "batch_set_views")
        self.views = views

    def submit(self):
        _check(self.L.mopcuda_batch_submit(self.h), "batch_submit")

    def wait(self, timeout_ms: int = 20000):
        _check(self.L.mopcuda_batch_wait(self.h, timeout_ms), "batch_wait")

    def render(self):
        self.submit()
        self.wait()
        return self

    @property
    def gpu_ms(self) -> float:
        return float(self.L.mopcuda_batch_gpu_time_ms(self.h))

    def read(self, i: int, what: int, out=None):
        v = self.views[i]
        sw, sh = v.width * v.ssaa, v.height * v.ssaa
        shape, dt = {BATCH_COLOR: ((sh, sw, 4), np.uint8),
                     BATCH_PRESENTED: ((v.height, v.width, 4), np.uint8),
                     BATCH_DEPTH: ((sh, sw), np.float32),
                     BATCH_IDS: ((sh, sw), np.uint32)}[what]
        if out is None:
            out = np.empty(shape, dt)
        _check(self.L.mopcuda_batch_read(self.h, i, what, out.ctypes.data, out.nbytes), "batch_read")
        return out

    def read_all(self, what: int, outs):
        """Buffer `what` of every viewport into outs[i] (arrays of the sizes
        read() gives), in one call."""
        n = len(self.views)
        ptrs = (C.c_void_p * n)(*[o.ctypes.data for o in outs])
        sizes = (C.c_size_t * n)(*[o.nbytes for o in outs])
        _check(self.L.mopcuda_batch_read_views(self.h, 0, n, what, ptrs, sizes), "batch_read_views")
        return outs

    def read_all_async(self, what: int, outs):
        """Colour buffer `what` of every viewport of the last submitted
        launch into outs[i] (page-locked arrays), copied while the next
        submitted launch renders; complete after wait_readback()."""
        n = len(self.views)
        ptrs = (C.c_void_p * n)(*[o.ctypes.data for o in outs])
        sizes = (C.c_size_t * n)(*[o.nbytes for o in outs])
        _check(self.L.mopcuda_batch_read_views_async(self.h, 0, n, what, ptrs, sizes),
               "batch_read_views_async")
        return outs

    def wait_readback(self, timeout_ms: int = 20000):
        _check(self.L.mopcuda_batch_readback_wait(self.h, timeout_ms), "batch_readback_wait")

    def pick(self, i: int, xy):
        xy = np.ascontiguousarray(xy, np.int32)
        n = xy.shape[0]
        ids = np.zeros(n, np.uint32)
        dep = np.zeros(n, np.float32)
        hits = np.zeros(n, np.int32)
        _check(self.L.mopcuda_batch_pick(self.h, i, xy.ctypes.data, n, ids.ctypes.data,
                                         dep.ctypes.data, hits.ctypes.data), "batch_pick")
        return ids, dep, hits

    def config(self) -> dict:
        c = MopCudaBatchConfig()
        _check(self.L.mopcuda_batch_get_config(self.h, C.byref(c)), "batch_get_config")
        return {f: getattr(c, f) for f, _ in MopCudaBatchConfig._fields_}

    def set_config(self, **kw):
        cur = self.config()
        cur.update(kw)
        c = MopCudaBatchConfig(**cur)
        _check(self.L.mopcuda_batch_set_config(self.h, C.byref(c)), "batch_set_config")

    def autotune(self, reps: int = 5) -> dict:
        import json
        buf = C.create_string_buffer(8192)
        _check(self.L.mopcuda_batch_autotune(self.h, reps, buf, len(buf)), "batch_autotune")
        return json.loads(buf.value.decode())

    @property
    def device_bytes(self) -> int:
        return int(self.L.mopcuda_batch_device_bytes(self.h))

    def close(self):
        if self.h:
            self.L.mopcuda_batch_destroy(self.h)
            self.h = None
        super().close()


class HostArray:
    """A numpy array over page-locked host memory (mopcuda_host_alloc)."""

    def __init__(self, shape, dtype):
        self.L = lib()
        n = int(np.prod(shape)) * np.dtype(dtype).itemsize
        self.p = self.L.mopcuda_host_alloc(n)
        if not self.p:
            raise RuntimeError(f"host_alloc failed: {last_error()}")
        buf = (C.c_uint8 * n).from_address(self.p)
        self.a = np.frombuffer(buf, dtype=dtype).reshape(shape)
        self.a.fill(0)

    def close(self):
        if self.p:
            self.a = None
            self.L.mopcuda_host_free(self.p)
            self.p = None


class Ticket:
    """An in-flight server request and the host buffers it fills."""

    def __init__(self, req, kind, view, color=None, ids=None, depth=None, xy=None):
        self.req, self.kind, self.view = req, kind, view
        self.color, self.ids, self.depth, self.xy = color, ids, depth, xy
        self.pick = None
        self.id = 0
        self.latency_ms = None


class Server:
    """Continuous-batching request server over resident scenes
    (mopcuda_server_*)."""

    def __init__(self, device: Device, hbm_budget: int, max_views: int = 64,
                 max_inflight: int = 3, batch_window_us: int = 0, max_launch_samples: int = 0):
        self.dev = device
        self.L = device.L
        cfg = MopCudaServerConfig(hbm_budget, max_views, max_inflight, batch_window_us,
                                  max_launch_samples)
        self.h = self.L.mopcuda_server_create(device.h, C.byref(cfg))
        if not self.h:
            raise RuntimeError(f"server_create failed: {last_error()}")
        self.scenes = []

    def add_scene(self, rs: ResidentScene) -> int:
        rc = self.L.mopcuda_server_add_scene(self.h, rs.sh_scene)
        if rc < 0:
            raise MopCudaError(rc, "server_add_scene")
        self.scenes.append(rs)
        return rc

    def _submit(self, t: Ticket) -> Ticket:
        tid = C.c_uint64()
        _check(self.L.mopcuda_server_submit(self.h, C.byref(t.req), C.byref(tid)), "server_submit")
        t.id = tid.value
        return t

    def submit_render(self, scene_id: int, view, want_ids=False, want_depth=False,
                      out=None) -> Ticket:
        """out: optional (h, w, 4) uint8 destination (page-locked memory
        receives the device copy directly)."""
        r = MopCudaRequest()
        r.kind, r.scene, r.view = REQ_RENDER, scene_id, view_struct(view)
        sw, sh = view.width * view.ssaa, view.height * view.ssaa
        color = out if out is not None else np.empty((view.height, view.width, 4), np.uint8)
        ids = np.empty((sh, sw), np.uint32) if want_ids else None
        dep = np.empty((sh, sw), np.float32) if want_depth else None
        r.color = color.ctypes.data
        r.ids = ids.ctypes.data if ids is not None else None
        r.depth = dep.ctypes.data if dep is not None else None
        return self._submit(Ticket(r, REQ_RENDER, view, color, ids, dep))

    def submit_pick(self, scene_id: int, view, xy) -> Ticket:
        xy = np.ascontiguousarray(xy, np.int32)
        n = xy.shape[0]
        r = MopCudaRequest()
        r.kind, r.scene, r.view = REQ_PICK, scene_id, view_struct(view)
        t = Ticket(r, REQ_PICK, view, xy=xy)
        t.pick = (np.zeros(n, np.uint32), np.zeros(n, np.float32), np.zeros(n, np.int32))
        r.pick_xy, r.pick_n = xy.ctypes.data, n
        r.pick_ids, r.pick_depths, r.pick_hits = [a.ctypes.data for a in t.pick]
        return self._submit(t)

    def wait(self, t: Ticket, timeout_ms: int = 20000) -> float:
        lat = C.c_double()
        _check(self.L.mopcuda_server_wait(self.h, t.id, timeout_ms, C.byref(lat)), "server_wait")
        t.latency_ms = float(lat.value)
        return t.latency_ms

    def drain(self, timeout_ms: int = 60000):
        _check(self.L.mopcuda_server_drain(self.h, timeout_ms), "server_drain")

    def stats(self) -> dict:
        st = MopCudaServerStats()
        _check(self.L.mopcuda_server_stats(self.h, C.byref(st)), "server_stats")
        return {f: getattr(st, f) for f, _ in MopCudaServerStats._fields_ if f != "pad"}

    def close(self):
        if self.h:
            self.L.mopcuda_server_destroy(self.h)
            self.h = None


def deform(dev: Device, bind_bytes, vertex_count: int, layout, bones=None, targets=None,
           weights=None) -> np.ndarray:
    """Skinning (bones) or morph (targets + weights) of a vertex buffer on the
    device through the C ABI; returns the deformed bytes (the host shadow
    mopcuda_buffer_read gives after the call)."""
    L, d = dev.L, dev.h
    b = np.ascontiguousarray(bind_bytes, np.uint8)
    bind = L.mopcuda_buffer_create(d, b.ctypes.data, b.nbytes)
    dst = L.mopcuda_buffer_create(d, b.ctypes.data, b.nbytes)
    tb = None
    try:
        lay = MopCudaDeformLayout(*layout)
        if bones is not None:
            m = _f32(bones).reshape(-1)
            _check(L.mopcuda_skin_apply(d, dst, bind, vertex_count, C.byref(lay), m.ctypes.data,
                                        m.size // 16), "skin_apply")
        else:
            t = _f32(targets).reshape(-1)
            w = _f32(weights)
            tb = L.mopcuda_buffer_create(d, t.ctypes.data, t.nbytes)
            _check(L.mopcuda_morph_apply(d, dst, bind, vertex_count, C.byref(lay), tb,
                                         w.ctypes.data, w.size), "morph_apply")
        p = L.mopcuda_buffer_read(dst)
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), shape=(b.nbytes,)).copy()
    finally:
        for h in (bind, dst, tb):
            if h:
                L.mopcuda_buffer_destroy(d, h)
