"""CUDA frame path vs the oracle (plain-C restatement of the reference CPU
backend) on seeded scenes, through the C ABI of libmopcuda.so.

IDs and depth must match bit for bit; colour within the contract tolerance
(tests/parity.py).  Scenes cover: multi-light smooth GGX (directional,
point, spot, ranged, inactive lights), textures, SSAA 2, IBL, flat shading
(lit and unlit), near-plane clipping (the config-1 ground plane passes
behind the camera), coplanar draw-order ties, the clipping/depth stress scene
(near-plane straddlers, coplanar pairs, host-skinned meshes), blended meshes
(alpha, additive, multiply) in the core's transparent-pass order, unlit
smooth draws (the legacy path's silhouette edge AA), directional
lights shadowed through the shadow pass (the shadow map itself compared
texel for texel), and picks.
"""
import dataclasses

import numpy as np
import pytest

import cpu_oracle
import mopcuda
import refdrive
import scenes
from parity import assert_frame_parity, color_stats, COLOR_MAX_LSB, COLOR_1LSB_FRACTION

pytestmark = pytest.mark.gpu


def _ibl_for(scene):
    if not scene.env:
        return None
    r = refdrive.Reference(scene)
    maps = r.env_maps()
    if scene.env_background:
        maps["env"] = r.env_hdr()
    r.close()
    return maps


def _render_cuda(dev, scene, ibl):
    r = mopcuda.SceneRenderer(dev, scene, ibl)
    try:
        r.render()
        return {"object_id": r.object_id(), "depth": r.depth(), "color_full": r.color_full(),
                "color": r.color(), "renderer": r}
    finally:
        pass


CASES = {
    "config1": lambda: scenes.config1(),
    "small_mixed_a": lambda: scenes.small_scene(seed=0),
    "small_mixed_b": lambda: scenes.small_scene(seed=1, width=203, height=117),
    "small_ssaa2": lambda: scenes.small_scene(seed=5, ssaa=2),
    "small_ssaa3": lambda: scenes.small_scene(seed=6, width=90, height=70, ssaa=3),
    "small_ibl": lambda: scenes.small_scene(seed=9, env=1),
    "small_flat_lit": lambda: dataclasses.replace(scenes.small_scene(seed=6), smooth=False),
    "small_flat_unlit": lambda: dataclasses.replace(scenes.small_scene(seed=8, lights="none"),
                                                    smooth=False),
    "coplanar_ties": lambda: scenes.coplanar_scene(),
    "config2_reduced": lambda: scenes.config2(width=320, height=180, ssaa=2, instances=24,
                                              tex_size=64),
    # clipping / depth stress: near-plane straddlers, out-of-frustum triangles, coplanar pairs
    # in separate meshes, host-skinned tubes, 0.1-8 px triangles
    "config3_reduced": lambda: scenes.config3(n_tris=80_000, width=480, height=270),
    "config3_medium": lambda: scenes.config3(seed=4, n_tris=400_000, width=960, height=540),
    # the benchmark workloads at full size: 1920x1080 SSAA 2 with 1.47 M triangles, 7 lights,
    # 1024^2 textures and IBL; 1920x1080 with 2 M clipping / coplanar / skinned triangles
    "config2_full": lambda: scenes.config2(),
    "config3_full": lambda: scenes.config3(),
    # blended meshes (alpha / additive / multiply), composited in submission order
    "transparent": lambda: scenes.transparent_scene(seed=21),
    "transparent_ssaa2_ibl": lambda: scenes.transparent_scene(seed=22, ssaa=2, env=1),
    "transparent_config2": lambda: _transparent_config2(),
    # 64 stacked blended quads: samples with more than 48 fragments (scratch heapsort)
    "transparent_deep": lambda: scenes.deep_transparent_scene(seed=65),
    "transparent_deep_ssaa2": lambda: scenes.deep_transparent_scene(seed=66, ssaa=2,
                                                                    layers=80),
    # blended flat draws (colour only, no depth or ID writes) in the transparent pass
    "transparent_flat": lambda: dataclasses.replace(scenes.transparent_scene(seed=60),
                                                    smooth=False),
    # no lights: the legacy smooth path with silhouette edge AA (order-dependent)
    "unlit_smooth": lambda: scenes.small_scene(seed=56, lights="none"),
    "unlit_smooth_ssaa2": lambda: scenes.small_scene(seed=57, lights="none", ssaa=2),
    "unlit_transparent": lambda: dataclasses.replace(scenes.transparent_scene(seed=58),
                                                     lights=[]),
    # shadow pass + 3x3 PCF on every directional light (one casting, one not)
    "shadow": lambda: scenes.shadow_scene(seed=51),
    "shadow_flat": lambda: dataclasses.replace(scenes.shadow_scene(seed=52), smooth=False),
    "shadow_ssaa2_ibl": lambda: scenes.shadow_scene(seed=53, ssaa=2, env=1),
    "shadow_transparent": lambda: scenes.shadow_scene(seed=54, transparent=True),
    "shadow_config2": lambda: _with_shadow(scenes.config2(width=320, height=180, ssaa=2,
                                                          instances=24, tex_size=64)),
    "shadow_config3": lambda: _with_shadow(scenes.config3(seed=5, n_tris=80_000, width=480,
                                                          height=270)),
    # MOP_POST_FOG with mop_viewport_set_fog: each sample's colour moved towards the fog colour
    # by its depth value, ahead of tonemap / gamma / vignette
    "fog": lambda: _fog(scenes.small_scene(seed=41), ((0.6, 0.65, 0.7, 1.0), 0.85, 0.99)),
    "fog_ssaa2": lambda: _fog(scenes.small_scene(seed=44, ssaa=2),
                              ((0.55, 0.6, 0.7, 1.0), 0.8, 0.99)),
    "fog_all_effects_ssaa2": lambda: _fog(
        scenes.small_scene(seed=42, ssaa=2), ((0.2, 0.3, 0.5, 1.0), 0.9, 0.995),
        scenes.POST_GAMMA | scenes.POST_TONEMAP | scenes.POST_VIGNETTE | scenes.POST_FXAA),
    "fog_tonemap_no_gamma": lambda: _fog(scenes.small_scene(seed=45),
                                         ((0.9, 0.8, 0.7, 1.0), 0.7, 0.999),
                                         scenes.POST_TONEMAP | scenes.POST_FXAA),
    "fog_zero_range": lambda: _fog(scenes.small_scene(seed=43), ((1.0, 0.0, 0.0, 1.0), 0.95, 0.95)),
    "fog_bright_colour_ssaa3": lambda: _fog(scenes.small_scene(seed=46, width=90, height=60, ssaa=3),
                                            ((1.6, -0.2, 0.4, 1.0), 0.5, 0.98)),
    "fog_transparent": lambda: _fog(scenes.transparent_scene(seed=47),
                                    ((0.5, 0.5, 0.55, 1.0), 0.9, 0.999)),
    "fog_config2_ibl": lambda: _fog(scenes.config2(width=320, height=180, ssaa=2, instances=24,
                                                   tex_size=64), ((0.7, 0.75, 0.8, 1.0), 0.95, 1.0)),
    # mop_viewport_add_instanced_mesh through mopcuda_draw_instanced: 96 instances with one
    # ID after the transparent pass, depth write off (each instance's depth undone after it)
    "instanced": lambda: scenes.instanced_scene(seed=71),
    "instanced_zero_id_ssaa2": lambda: scenes.instanced_scene(seed=72, ssaa=2, zero_id=True),
    "instanced_transparent": lambda: scenes.instanced_scene(seed=73, transparent=True),
    "instanced_flat": lambda: dataclasses.replace(scenes.instanced_scene(seed=74), smooth=False),
    "instanced_unlit": lambda: dataclasses.replace(scenes.instanced_scene(seed=75), lights=[]),
    "instanced_shadow_ibl_ssaa2": lambda: _with_shadow(scenes.instanced_scene(seed=76, ssaa=2,
                                                                              env=1)),
    # mop_viewport_set_environment_background: the procedural sky behind the scene
    "env_background": lambda: dataclasses.replace(scenes.small_scene(seed=97, env=1),
                                                  env_background=True),
    "env_background_ssaa2_transparent": lambda: dataclasses.replace(
        scenes.transparent_scene(seed=98, ssaa=2, env=1), env_background=True,
        env_rotation=0.7, env_intensity=1.3),
    # MOP_RENDER_WIREFRAME: each triangle's edges as Xiaolin Wu lines in its flat colour,
    # blended over what is there in submission order (ID 0 stays filled)
    "wireframe": lambda: scenes.wireframe_scene(seed=121),
    "wireframe_unlit_ssaa2": lambda: scenes.wireframe_scene(seed=122, ssaa=2, lights="none"),
    "wireframe_flat_ssaa3": lambda: dataclasses.replace(
        scenes.wireframe_scene(seed=123, width=96, height=64, ssaa=3), smooth=False),
    "wireframe_transparent": lambda: dataclasses.replace(scenes.transparent_scene(seed=124),
                                                         wireframe=True),
    "wireframe_chrome": lambda: dataclasses.replace(scenes.chrome_scene(seed=125),
                                                    wireframe=True),
    "wireframe_instanced": lambda: dataclasses.replace(scenes.instanced_scene(seed=126),
                                                       wireframe=True),
    # editor-chrome IDs among the opaque meshes: depth test and culling off, unlit
    "chrome": lambda: scenes.chrome_scene(seed=81),
    "chrome_ssaa2_flat": lambda: dataclasses.replace(scenes.chrome_scene(seed=82, ssaa=2),
                                                     smooth=False),
}

# fog cases whose colour is bit-exact: no IBL lookups (CUDA's atan2f/asinf) and no
# vignette (the one place the sRGB value itself, not its byte, is needed)
FOG_EXACT = ["fog", "fog_ssaa2", "fog_tonemap_no_gamma", "fog_zero_range",
             "fog_bright_colour_ssaa3", "fog_transparent"]


def _fog(sc, fog, post=None):
    """The scene with the FOG bit added to its post effects (or to `post`) and
    the given MopFogParams ((r, g, b, a), near, far)."""
    fx = (sc.post_effects if post is None else post) | scenes.POST_FOG
    return dataclasses.replace(sc, post_effects=fx, fog=fog)


def _with_shadow(sc):
    """The scene with its first directional light casting shadows (one is
    added when the scene has none)."""
    for k, l in enumerate(sc.lights):
        if l.type == scenes.LIGHT_DIRECTIONAL and l.active:
            sc.lights[k] = dataclasses.replace(l, cast_shadows=True)
            return sc
    sc.lights.insert(0, scenes.Light(scenes.LIGHT_DIRECTIONAL, direction=(-0.3, -0.9, -0.2),
                                     intensity=1.5, cast_shadows=True))
    return sc


def _transparent_config2():
    sc = scenes.config2(width=320, height=180, ssaa=2, instances=32, tex_size=64)
    for k in range(0, len(sc.meshes), 3):  # every third instance blended
        sc.meshes[k] = dataclasses.replace(sc.meshes[k], opacity=0.35 + 0.1 * (k % 5),
                                           blend_mode=(1, 2, 3, 1)[k % 4])
    return sc


@pytest.mark.parametrize("name", list(CASES))
def test_frame_parity(cuda_device, name):
    sc = CASES[name]()
    ibl = _ibl_for(sc)
    ref = cpu_oracle.render(sc, ibl)
    got = _render_cuda(cuda_device, sc, ibl)
    try:
        assert_frame_parity(got, ref, name)
        xy = scenes.pick_points(sc, 1000)
        i1, d1, h1 = got["renderer"].pick(xy)
        i2, d2, h2 = cpu_oracle.pick(sc, ref, xy)
        assert (i1 == i2).all() and (h1 == h2).all()
        assert (d1.view(np.uint32) == d2.view(np.uint32)).all()
    finally:
        got["renderer"].close()


@pytest.mark.parametrize("name", FOG_EXACT)
def test_fog_colour_bit_exact(cuda_device, name):
    """The fog term, Reinhard and the sRGB step through the threshold table
    give the reference's bytes exactly where no IBL lookup is involved."""
    sc = CASES[name]()
    ref = cpu_oracle.render(sc, None)
    got = _render_cuda(cuda_device, sc, None)
    try:
        for key in ("color_full", "color"):
            s = color_stats(got[key], ref[key])
            assert s["exact"] == 1.0, (name, key, s)
    finally:
        got["renderer"].close()


def test_fog_follows_set_fog(cuda_device):
    """Fog parameters changed between frames take effect on the next frame;
    the FOG bit with a new device's zero parameters leaves colours as they are."""
    sc = CASES["fog"]()
    plain = dataclasses.replace(sc, fog=None)
    r = mopcuda.SceneRenderer(cuda_device, plain)
    try:
        r.render()
        zero = r.color_full().copy()
        ref0 = cpu_oracle.render(dataclasses.replace(sc, post_effects=scenes.DEFAULT_POST,
                                                     fog=None), None)
        assert (zero == ref0["color_full"]).all()
        fc = (mopcuda.C.c_float * 4)(*sc.fog[0])
        assert cuda_device.L.mopcuda_set_fog(cuda_device.h, fc, sc.fog[1], sc.fog[2]) == 0
        r.render()
        ref1 = cpu_oracle.render(sc, None)
        assert (r.color_full() == ref1["color_full"]).all()
        assert cuda_device.L.mopcuda_set_fog(cuda_device.h, None, 0.0, 1.0) != 0
    finally:
        r.close()


def test_repeat_frames_identical(cuda_device):
    """Deterministic replay: two frames of one scene are byte-identical
    (reference tests/test_torture_picking.c:432-456 replays with bit-equal
    depth)."""
    sc = scenes.small_scene(seed=2)
    r = mopcuda.SceneRenderer(cuda_device, sc)
    try:
        a = (r.render().color_full(), r.depth(), r.object_id())
        b = (r.render().color_full(), r.depth(), r.object_id())
        for x, y in zip(a, b):
            assert x.tobytes() == y.tobytes()
    finally:
        r.close()


@pytest.mark.parametrize("name", ["shadow", "shadow_config3"])
def test_shadow_map_matches_oracle(cuda_device, name):
    """The device shadow pass (depth-only raster of the casters from the
    light) equals pass_shadow's map texel for texel (-0 and +0 count as one
    value: the lookup compares after adding the bias)."""
    sc = CASES[name]()
    want = cpu_oracle.shadow_map(sc)
    r = mopcuda.SceneRenderer(cuda_device, sc)
    try:
        assert r.shadow_pass()
        got = r.shadow_map()
        assert ((got + 0.0).view(np.uint32) == (want["depth"] + 0.0).view(np.uint32)).all(), \
            int(((got + 0.0).view(np.uint32) != (want["depth"] + 0.0).view(np.uint32)).sum())
        assert (want["depth"] < 1.0).mean() > 0.05  # the casters cover part of the map
    finally:
        r.close()


def test_shadow_draw_list_equals_single_draws(cuda_device):
    """mopcuda_shadow_draw_list (the renderer's path) builds the same map as
    one mopcuda_shadow_draw call per caster, and rejects a caster whose
    counts exceed its buffers as the single call does."""
    sc = scenes.shadow_scene(seed=57)
    r = mopcuda.SceneRenderer(cuda_device, sc)
    L, d = mopcuda.lib(), cuda_device.h
    try:
        assert r.shadow_pass()
        by_list = r.shadow_map()
        casters = scenes.shadow_casters(sc)
        vp = np.zeros(16, np.float32)
        models = np.concatenate([mopcuda._f32(sc.meshes[k].transform) for k in casters])
        dr = mopcuda._f32(scenes.shadow_light(sc).direction)
        L.mopcuda_shadow_light_vp(models.ctypes.data, len(casters), dr.ctypes.data, vp.ctypes.data)
        assert L.mopcuda_shadow_begin(d, scenes.SHADOW_MAP_SIZE, vp.ctypes.data) == 0
        for j, k in enumerate(casters):
            _, vb, ib, vc, ic = r.meshes[k]
            assert L.mopcuda_shadow_draw(d, vb, vc, 48, ib, ic, models[16 * j:].ctypes.data) == 0
        assert L.mopcuda_shadow_end(d) == 0
        one_by_one = r.shadow_map()
        assert (by_list.view(np.uint32) == one_by_one.view(np.uint32)).all()
        bad = (mopcuda.MopCudaShadowCaster * 1)()
        _, vb, ib, vc, ic = r.meshes[casters[0]]
        bad[0].vertices, bad[0].indices, bad[0].stride = vb, ib, 48
        bad[0].vertex_count, bad[0].index_count = vc + 1000000, ic
        assert L.mopcuda_shadow_begin(d, scenes.SHADOW_MAP_SIZE, vp.ctypes.data) == 0
        assert L.mopcuda_shadow_draw_list(d, bad, 1) != 0
        assert "exceed the buffers" in mopcuda.last_error()
        assert L.mopcuda_shadow_end(d) == 0
    finally:
        r.close()


def test_shadow_pipelined_frames_match_sync(cuda_device):
    """Shadowed frames submitted back to back (each shadow pass recorded
    while the previous frame runs, into the map that frame does not read)
    with a caster moving every frame and the images read asynchronously
    equal the same frames rendered one at a time."""
    sc = scenes.shadow_scene(seed=61)
    r = mopcuda.SceneRenderer(cuda_device, sc)
    casters = scenes.shadow_casters(sc)
    mover = sc.meshes[casters[-1]]
    base = mover.transform.copy()
    steps = [(0.0, 0.0), (0.35, 0.0), (0.35, 0.3), (-0.3, 0.1), (0.0, -0.25)]
    bufs = [mopcuda.HostArray((sc.height, sc.width, 4), np.uint8) for _ in steps]

    def place(dx, dz):
        mover.transform[:] = base
        mover.transform[12] += dx
        mover.transform[14] += dz
        r.update_camera()

    try:
        want, maps = [], []
        for dx, dz in steps:
            place(dx, dz)
            r.render()
            want.append(r.color())
            maps.append(r.shadow_map())
        assert all((maps[k] != maps[k + 1]).any() for k in range(len(steps) - 1))
        for k, (dx, dz) in enumerate(steps):
            place(dx, dz)
            r.submit()
            r.color_async(bufs[k].a)
        r.wait_readback()
        for k in range(len(steps)):
            assert (bufs[k].a == want[k]).all(), f"frame {k}"
        assert (r.shadow_map().view(np.uint32) == maps[-1].view(np.uint32)).all()
    finally:
        for b in bufs:
            b.close()
        r.close()


def test_shadow_clear_unbinds(cuda_device):
    """Once the casting light is switched off, frames render as without a
    shadow map (mop_sw_shadow_clear)."""
    sc = scenes.shadow_scene(seed=55)
    r = mopcuda.SceneRenderer(cuda_device, sc)
    try:
        shadowed = r.render().color_full()
        sc.lights[0] = dataclasses.replace(sc.lights[0], cast_shadows=False)
        plain = r.render().color_full()
        ref = cpu_oracle.render(sc)
        assert "shadow" not in ref
        st = color_stats(plain, ref["color_full"])
        assert st["max"] <= COLOR_MAX_LSB and st["within1"] >= COLOR_1LSB_FRACTION, st
        assert (plain != shadowed).any()
    finally:
        r.close()


@pytest.mark.parametrize("ssaa,width,height", [(1, 160, 120), (2, 160, 120),
                                               (2, 1920, 1080)])
def test_async_readback_matches_sync(cuda_device, ssaa, width, height):
    """mopcuda_read_color_resolved_async: frames submitted back to back with
    their images requested asynchronously (each copy issued inside the next
    frame's launch and overlapping it) equal the synchronous reads of the
    same frames.  At 1920x1080 an image copy outlasts the next frame's work
    up to its post pass, which must wait for it."""
    sc = scenes.small_scene(seed=59, ssaa=ssaa, width=width, height=height)
    eyes = [(4.0, 3.0, 7.0), (-5.0, 2.0, 5.0), (2.0, 6.0, -6.0), (6.0, 1.5, 1.0),
            (-3.0, 4.0, -5.0), (5.0, 5.0, 3.0)]
    r = mopcuda.SceneRenderer(cuda_device, sc)
    bufs = [mopcuda.HostArray((sc.height, sc.width, 4), np.uint8) for _ in eyes]
    try:
        want = []
        for e in eyes:
            sc.eye = e
            r.update_camera()
            r.render()
            want.append(r.color())
        for k, e in enumerate(eyes):
            sc.eye = e
            r.update_camera()
            r.submit()
            r.color_async(bufs[k].a)
        r.wait_readback()
        for k in range(len(eyes)):
            assert (bufs[k].a == want[k]).all(), f"frame {k}"
    finally:
        for b in bufs:
            b.close()
        r.close()
