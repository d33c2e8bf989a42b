"""ctypes driver for the plain-C oracle (oracle/liboracle.so).

Test infrastructure only: builds the per-draw records a viewport would emit
for a scene (EMIT_DRAW, reference src/core/viewport.c:2015-2088) and runs the
serial restatement of the CPU frame path on them.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

import scenes

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"

DEFAULT_LIGHT_DIR = (0.3, 1.0, 0.5)  # viewport default, reference viewport.c:641


class OrLight(C.Structure):
    _fields_ = [("type", C.c_int32), ("position", C.c_float * 3),
                ("direction", C.c_float * 3), ("color", C.c_float * 4),
                ("intensity", C.c_float), ("range", C.c_float),
                ("spot_inner_cos", C.c_float), ("spot_outer_cos", C.c_float),
                ("active", C.c_int32)]


class OrDraw(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("vertex_count", C.c_uint32),
                ("indices", C.c_void_p), ("index_count", C.c_uint32),
                ("object_id", C.c_uint32), ("model", C.c_float * 16),
                ("mvp", C.c_float * 16), ("light_dir", C.c_float * 3),
                ("ambient", C.c_float), ("opacity", C.c_float),
                ("metallic", C.c_float), ("roughness", C.c_float),
                ("depth_bias", C.c_float), ("cam_eye", C.c_float * 3),
                ("smooth", C.c_int32), ("depth_test", C.c_int32),
                ("backface_cull", C.c_int32), ("blend_mode", C.c_int32),
                ("lights", C.POINTER(OrLight)), ("light_count", C.c_uint32),
                ("texture", C.c_void_p), ("tex_w", C.c_int32), ("tex_h", C.c_int32),
                ("depth_write", C.c_int32), ("wireframe", C.c_int32)]


class OrIBL(C.Structure):
    _fields_ = [("irr", C.c_void_p), ("irr_w", C.c_int32), ("irr_h", C.c_int32),
                ("pf", C.c_void_p), ("pf_w", C.c_int32), ("pf_h", C.c_int32),
                ("pf_levels", C.c_int32), ("brdf", C.c_void_p), ("brdf_size", C.c_int32),
                ("rotation", C.c_float), ("intensity", C.c_float)]


class OrShadow(C.Structure):
    _fields_ = [("depth", C.c_void_p), ("w", C.c_int32), ("h", C.c_int32),
                ("vp", C.c_float * 16)]


class OrShadowMesh(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("vertex_count", C.c_uint32),
                ("indices", C.c_void_p), ("index_count", C.c_uint32),
                ("model", C.c_float * 16)]


class OrSky(C.Structure):
    _fields_ = [("env", C.c_void_p), ("w", C.c_int32), ("h", C.c_int32),
                ("rotation", C.c_float), ("intensity", C.c_float), ("eye", C.c_float * 3),
                ("target", C.c_float * 3), ("up", C.c_float * 3), ("fov_deg", C.c_float)]


class OrFrame(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("ssaa", C.c_int32),
                ("clear", C.c_float * 4), ("exposure", C.c_float),
                ("post_effects", C.c_uint32), ("ibl", C.POINTER(OrIBL)),
                ("color_full", C.c_void_p), ("depth", C.c_void_p),
                ("object_id", C.c_void_p), ("color_presented", C.c_void_p),
                ("hdr", C.c_void_p), ("shadow", C.POINTER(OrShadow)),
                ("fog_on", C.c_int32), ("fog_color", C.c_float * 4),
                ("fog_near", C.c_float), ("fog_far", C.c_float), ("sky", C.POINTER(OrSky))]


_lib = None


class OrDeformLayout(C.Structure):
    _fields_ = [("stride", C.c_uint32), ("position_offset", C.c_int32),
                ("normal_offset", C.c_int32), ("joints_offset", C.c_int32),
                ("weights_offset", C.c_int32)]


def skin(layout, bind: np.ndarray, vertex_count: int, bones: np.ndarray) -> np.ndarray:
    """mop_skin_apply restated (bytes in, bytes out)."""
    L = OrDeformLayout(*layout)
    b = np.ascontiguousarray(bind, np.uint8)
    m = np.ascontiguousarray(bones, np.float32).reshape(-1)
    out = np.empty_like(b)
    lib().oracle_skin_apply(C.byref(L), b.ctypes.data, vertex_count, m.ctypes.data,
                            m.size // 16, out.ctypes.data)
    return out


def morph(layout, bind: np.ndarray, vertex_count: int, targets: np.ndarray,
          weights: np.ndarray) -> np.ndarray:
    """mop_morph_apply restated (bytes in, bytes out)."""
    L = OrDeformLayout(*layout)
    b = np.ascontiguousarray(bind, np.uint8)
    t = np.ascontiguousarray(targets, np.float32).reshape(-1)
    w = np.ascontiguousarray(weights, np.float32)
    out = np.empty_like(b)
    lib().oracle_morph_apply(C.byref(L), b.ctypes.data, vertex_count, t.ctypes.data,
                             w.ctypes.data, w.size, out.ctypes.data)
    return out


def lib():
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            raise FileNotFoundError(f"oracle not built: {ORACLE_SO} (run make -C oracle oracle)")
        _lib = C.CDLL(str(ORACLE_SO))
        _lib.oracle_render.argtypes = [C.POINTER(OrFrame), C.POINTER(OrDraw), C.c_uint32]
        _lib.oracle_camera.argtypes = [C.c_void_p] * 3 + [C.c_float] * 3 + [C.c_int] * 2 + [C.c_void_p] * 3
        _lib.oracle_mat4_multiply.argtypes = [C.c_void_p] * 3
        _lib.oracle_pick.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.oracle_gamma_lut.argtypes = [C.c_void_p]
        _lib.oracle_skin_apply.argtypes = [C.POINTER(OrDeformLayout), C.c_void_p, C.c_uint32,
                                           C.c_void_p, C.c_uint32, C.c_void_p]
        _lib.oracle_morph_apply.argtypes = [C.POINTER(OrDeformLayout), C.c_void_p, C.c_uint32,
                                            C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
        _lib.oracle_mop_decode_mesh.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
        _lib.oracle_bc_decode.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        _lib.oracle_shadow_matrix.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
        _lib.oracle_shadow_render.argtypes = [C.POINTER(OrShadowMesh), C.c_uint32, C.c_int,
                                              C.c_void_p, C.c_void_p]
    return _lib


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def camera(scene):
    """(view, proj, eye) of the frame, as mop_viewport_render derives them."""
    view = np.zeros(16, np.float32)
    proj = np.zeros(16, np.float32)
    eye = np.zeros(3, np.float32)
    e, t, u = _f32(scene.eye), _f32(scene.target), _f32(scene.up)
    lib().oracle_camera(e.ctypes.data, t.ctypes.data, u.ctypes.data, scene.fov_deg, scene.near,
                        scene.far, scene.width, scene.height, view.ctypes.data, proj.ctypes.data,
                        eye.ctypes.data)
    return view, proj, eye


def mat4_multiply(a, b):
    a, b = _f32(a), _f32(b)
    c = np.zeros(16, np.float32)
    lib().oracle_mat4_multiply(a.ctypes.data, b.ctypes.data, c.ctypes.data)
    return c


def gamma_lut():
    lut = np.zeros(256, np.uint8)
    lib().oracle_gamma_lut(lut.ctypes.data)
    return lut


def _light(l):
    s = OrLight()
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


def shadow_map(scene):
    """pass_shadow restated (reference viewport.c:2288-2442): None when no
    active directional light casts or no mesh casts, else the bound map
    {"depth": float32 [size, size], "vp": float32 [16], "size": size}."""
    light = scenes.shadow_light(scene)
    casters = scenes.shadow_casters(scene)
    if light is None or not casters:
        return None
    models = np.concatenate([_f32(scene.meshes[k].transform) for k in casters])
    vp = np.zeros(16, np.float32)
    d = _f32(light.direction)
    lib().oracle_shadow_matrix(models.ctypes.data, len(casters), d.ctypes.data, vp.ctypes.data)
    keep = []
    ms = (OrShadowMesh * len(casters))()
    for j, k in enumerate(casters):
        m = scene.meshes[k]
        v = _f32(m.vertices)
        i = np.ascontiguousarray(m.indices, np.uint32)
        keep += [v, i]
        ms[j].vertices, ms[j].vertex_count = v.ctypes.data, v.shape[0]
        ms[j].indices, ms[j].index_count = i.ctypes.data, i.size
        ms[j].model[:] = [float(x) for x in m.transform]
    n = scenes.SHADOW_MAP_SIZE
    depth = np.zeros((n, n), np.float32)
    lib().oracle_shadow_render(ms, len(casters), n, vp.ctypes.data, depth.ctypes.data)
    return {"depth": depth, "vp": vp, "size": n}


def render(scene, ibl=None, want_hdr=False):
    """Render `scene` with the oracle.  `ibl` is the dict returned by
    refdrive.Reference.env_maps() (or None for no IBL)."""
    L = lib()
    view, proj, eye = camera(scene)
    keep = []
    lights = (OrLight * max(1, len(scene.lights)))()
    for k, l in enumerate(scene.lights):
        lights[k] = _light(l)
    texs = [bc_decode(t) if isinstance(t, scenes.CompressedTexture)
            else np.ascontiguousarray(t, np.uint8) for t in scene.textures]
    inst = getattr(scene, "instanced", [])
    n_inst = sum(int(im.transforms.shape[0]) for im in inst)
    order = scenes.draw_order(scene, eye)
    n_draws = len(order) + n_inst
    draws = (OrDraw * max(1, n_draws))()
    amb = min(max(scene.ambient, 0.0), 1.0)
    for k, mi in enumerate(order):
        m = scene.meshes[mi]
        v = _f32(m.vertices)
        i = np.ascontiguousarray(m.indices, np.uint32)
        keep += [v, i]
        d = draws[k]
        d.vertices, d.vertex_count = v.ctypes.data, v.shape[0]
        d.indices, d.index_count = i.ctypes.data, i.size
        d.object_id = m.object_id
        d.model[:] = [float(x) for x in m.transform]
        d.mvp[:] = [float(x) for x in mat4_multiply(proj, mat4_multiply(view, m.transform))]
        d.light_dir[:] = DEFAULT_LIGHT_DIR
        d.ambient = amb
        d.opacity = m.opacity
        d.metallic = m.metallic if m.has_material else 0.0
        d.roughness = m.roughness if m.has_material else 0.5
        d.depth_bias = 0.0
        d.cam_eye[:] = [float(x) for x in eye]
        d.smooth = 1 if getattr(scene, "smooth", True) else 0
        d.depth_test, d.backface_cull = 1, 1
        d.blend_mode = scenes.effective_blend(m)
        d.lights = lights
        d.light_count = len(scene.lights)
        d.depth_write = 1
        # MOP_RENDER_WIREFRAME: every mesh but ID 0 as lines (viewport.c:2056-2057)
        d.wireframe = 1 if getattr(scene, "wireframe", False) and m.object_id != 0 else 0
        if scenes.is_chrome(m.object_id):  # EMIT_DRAW, viewport.c:2035-2076
            d.depth_test, d.backface_cull = 0, 0
            d.lights, d.light_count = None, 0
            d.ambient = 1.0
        if m.texture >= 0:
            t = texs[m.texture]
            d.texture, d.tex_h, d.tex_w = t.ctypes.data, t.shape[0], t.shape[1]
    # pass_instanced (reference viewport.c:2602-2646), after the transparent pass: one draw
    # per instance (cpu_draw_instanced, cpu_backend.c:638-657) with model = the instance,
    # mvp = P * (V * instance), the default material, no texture, culling only for
    # non-zero IDs, depth test with the depth write off, and cam_eye left at zero
    k = len(order)
    for im in inst:
        v = _f32(im.vertices)
        i = np.ascontiguousarray(im.indices, np.uint32)
        keep += [v, i]
        for t in np.asarray(im.transforms, np.float32).reshape(-1, 16):
            d = draws[k]
            k += 1
            d.vertices, d.vertex_count = v.ctypes.data, v.shape[0]
            d.indices, d.index_count = i.ctypes.data, i.size
            d.object_id = im.object_id
            d.model[:] = [float(x) for x in t]
            d.mvp[:] = [float(x) for x in mat4_multiply(proj, mat4_multiply(view, t))]
            d.light_dir[:] = DEFAULT_LIGHT_DIR
            d.ambient = amb
            d.opacity = 1.0
            d.metallic, d.roughness = 0.0, 0.5
            d.cam_eye[:] = [0.0, 0.0, 0.0]
            d.smooth = 1 if getattr(scene, "smooth", True) else 0
            d.depth_test, d.depth_write = 1, 0
            d.backface_cull = 1 if im.object_id != 0 else 0
            d.blend_mode = 0
            d.lights = lights
            d.light_count = len(scene.lights)
            d.wireframe = 1 if getattr(scene, "wireframe", False) and im.object_id != 0 else 0
    sw, sh = scene.width * scene.ssaa, scene.height * scene.ssaa
    out = {
        "color": np.zeros((scene.height, scene.width, 4), np.uint8),
        "color_full": np.zeros((sh, sw, 4), np.uint8),
        "depth": np.zeros((sh, sw), np.float32),
        "object_id": np.zeros((sh, sw), np.uint32),
        "view": view, "proj": proj, "eye": eye,
    }
    f = OrFrame()
    f.width, f.height, f.ssaa = sw, sh, scene.ssaa
    f.clear[:] = scene.clear
    f.exposure = scene.exposure
    f.post_effects = scene.post_effects
    fog = getattr(scene, "fog", None)
    if fog is not None:
        f.fog_on = 1
        f.fog_color[:] = fog[0]
        f.fog_near, f.fog_far = fog[1], fog[2]
    if ibl is not None:
        arrs = [_f32(ibl["irr"]), _f32(ibl["pf"]), _f32(ibl["brdf"])]
        keep += arrs
        ib = OrIBL()
        ib.irr, ib.irr_w, ib.irr_h = arrs[0].ctypes.data, ibl["irr_w"], ibl["irr_h"]
        ib.pf, ib.pf_w, ib.pf_h, ib.pf_levels = arrs[1].ctypes.data, ibl["pf_w"], ibl["pf_h"], ibl["pf_levels"]
        ib.brdf, ib.brdf_size = arrs[2].ctypes.data, ibl["brdf_size"]
        ib.rotation, ib.intensity = ibl["rotation"], ibl["intensity"]
        keep.append(ib)
        f.ibl = C.pointer(ib)
    f.color_full = out["color_full"].ctypes.data
    f.depth = out["depth"].ctypes.data
    f.object_id = out["object_id"].ctypes.data
    f.color_presented = out["color"].ctypes.data
    if want_hdr:
        out["hdr"] = np.zeros((sh, sw, 4), np.float32)
        f.hdr = out["hdr"].ctypes.data
    if getattr(scene, "env_background", False) and ibl is not None and "env" in ibl:
        env = _f32(ibl["env"])
        sk = OrSky()
        sk.env, sk.h, sk.w = env.ctypes.data, env.shape[0], env.shape[1]
        sk.rotation, sk.intensity = scene.env_rotation, scene.env_intensity
        sk.eye[:], sk.target[:], sk.up[:] = scene.eye, scene.target, scene.up
        sk.fov_deg = scene.fov_deg
        keep += [env, sk]
        f.sky = C.pointer(sk)
    shadow = shadow_map(scene)
    if shadow is not None:
        so = OrShadow()
        so.depth, so.w, so.h = shadow["depth"].ctypes.data, shadow["size"], shadow["size"]
        so.vp[:] = [float(x) for x in shadow["vp"]]
        keep += [shadow, so]
        f.shadow = C.pointer(so)
        out["shadow"] = shadow
    rc = L.oracle_render(C.byref(f), draws, n_draws)
    if rc != 0:
        raise RuntimeError(f"oracle_render failed: {rc}")
    return out


def bc_decode(t):
    """The RGBA8 texels [h, w, 4] of a scenes.CompressedTexture
    (bc_decompress_to_rgba8)."""
    out = np.zeros((t.height, t.width, 4), np.uint8)
    d = np.ascontiguousarray(t.data, np.uint8)
    if lib().oracle_bc_decode(t.format, t.width, t.height, d.ctypes.data, out.ctypes.data):
        raise ValueError(f"format {t.format} is not decoded")
    return out


def pick(scene, frame, xy):
    xy = np.ascontiguousarray(xy, np.int32)
    n = xy.shape[0]
    ids = np.zeros(n, np.uint32)
    dep = np.zeros(n, np.float32)
    hits = np.zeros(n, np.int32)
    oid = np.ascontiguousarray(frame["object_id"], np.uint32)
    d = np.ascontiguousarray(frame["depth"], np.float32)
    lib().oracle_pick(oid.ctypes.data, d.ctypes.data, scene.width, scene.height, scene.ssaa, n,
                      xy.ctypes.data, ids.ctypes.data, dep.ctypes.data, hits.ctypes.data)
    return ids, dep, hits


def scene_file_meshes(path):
    """Every mesh section of a .mop v2 file decoded as mop_scene_get_mesh
    does: a list of (vertices float32 [V, 12], indices uint32, bbox [6])."""
    import struct
    data = open(path, "rb").read()
    magic, version, nsec, _ = struct.unpack_from("<IIII", data, 0)
    if magic != 0x4D4F5002 or version != 2 or nsec > 256:
        raise ValueError("not a .mop v2 file")
    buf = np.frombuffer(data, np.uint8)
    out = []
    for k in range(nsec):
        kind, _, off, size = struct.unpack_from("<IIQQ", data, 64 + 24 * k)
        if kind != 1:
            continue
        vc, ic = struct.unpack_from("<II", data, off)
        bbox = np.frombuffer(data, np.float32, 6, off + 16).copy()
        v = np.zeros((vc, 12), np.float32)
        i = np.zeros(ic, np.uint32)
        sec = np.ascontiguousarray(buf[off:off + size])
        if lib().oracle_mop_decode_mesh(sec.ctypes.data, size, v.ctypes.data, i.ctypes.data):
            raise ValueError(f"mesh section {k} shorter than its counts")
        out.append((v, i, bbox))
    return out
