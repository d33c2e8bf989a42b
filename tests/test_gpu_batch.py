"""Batched viewports (mopcuda_scene_* / mopcuda_batch_*): every viewport of a
batch equals the single-viewport frame of the same draws and camera, byte
for byte (colour at sample and presented resolution, depth bits, object IDs,
picks), under any launch configuration, after the autotuner, after TRS
updates, and when the pools must grow.  One batch is also checked against
the oracle directly.
"""
import dataclasses

import numpy as np
import pytest

import cpu_oracle
import mopcuda
import scenes
from parity import assert_frame_parity

pytestmark = pytest.mark.gpu


def _plain(dev, sc, ibl):
    r = mopcuda.SceneRenderer(dev, sc, ibl)
    try:
        r.render()
        return {"color_full": r.color_full(), "color": r.color(), "depth": r.depth(),
                "object_id": r.object_id(), "pick": r.pick(scenes.pick_points(sc, 64, seed=3))}
    finally:
        r.close()


def _batch_view(b, i):
    v = b.views[i]
    sc_pts = scenes.pick_points(dataclasses.replace(b.scene, width=v.width, height=v.height), 64,
                                seed=3)
    return {"color_full": b.read(i, mopcuda.BATCH_COLOR),
            "color": b.read(i, mopcuda.BATCH_PRESENTED),
            "depth": b.read(i, mopcuda.BATCH_DEPTH),
            "object_id": b.read(i, mopcuda.BATCH_IDS),
            "pick": b.pick(i, sc_pts)}


def _assert_same(got, want, label):
    for k in ("color_full", "color", "object_id"):
        assert got[k].shape == want[k].shape, f"{label}: {k} shape"
        n = int((got[k] != want[k]).sum())
        assert n == 0, f"{label}: {k} differs in {n} entries"
    nd = int((got["depth"].view(np.uint32) != want["depth"].view(np.uint32)).sum())
    assert nd == 0, f"{label}: depth differs in {nd} samples"
    for a, b in zip(got["pick"], want["pick"]):
        assert (np.asarray(a).view(np.uint32) == np.asarray(b).view(np.uint32)).all(), label


def _scene(instances=24, tex=64):
    return scenes.config2(width=320, height=180, ssaa=2, instances=instances, tex_size=tex)


def _views(sc, n, seed, max_px=320 * 240):
    vs = scenes.batch_views(sc, n=n, seed=seed, min_px=24 * 24, max_px=max_px)
    vs[0] = dataclasses.replace(vs[0], ssaa=3)  # all SSAA templates
    return vs


def _check_batch(dev, b, sc, ibl, label):
    for i, v in enumerate(b.views):
        want = _plain(dev, scenes.scene_for_view(sc, v), ibl)
        _assert_same(_batch_view(b, i), want, f"{label} view {i} ({v.width}x{v.height}x{v.ssaa})")


@pytest.fixture(scope="module")
def ibl():
    return scenes.procedural_ibl((0.4, 0.8, 0.35), irr_size=(32, 16), pf_size=(64, 32),
                                 levels=4, brdf_size=64)


def test_batch_equals_single_viewport_frames(cuda_device, ibl):
    sc = _scene()
    b = mopcuda.BatchRenderer(cuda_device, sc, _views(sc, 10, seed=1), ibl)
    try:
        b.render()
        _check_batch(cuda_device, b, sc, ibl, "batch")
        # a second launch of the captured graph gives the same bytes
        first = [_batch_view(b, i) for i in range(len(b.views))]
        b.render()
        for i in range(len(b.views)):
            _assert_same(_batch_view(b, i), first[i], f"replay view {i}")
    finally:
        b.close()


def test_batch_fog_equals_single_viewport_frames(cuda_device, ibl):
    """A batch made while the device has the FOG bit and fog parameters set
    applies them to every viewport as the plain frame does."""
    sc = dataclasses.replace(_scene(), fog=((0.6, 0.65, 0.7, 1.0), 0.9, 0.999),
                             post_effects=scenes.DEFAULT_POST | scenes.POST_FOG)
    b = mopcuda.BatchRenderer(cuda_device, sc, _views(sc, 6, seed=9), ibl)
    try:
        b.render()
        _check_batch(cuda_device, b, sc, ibl, "fog batch")
    finally:
        b.close()


def _shadowed(sc):
    """The scene with its first directional light casting shadows."""
    for k, l in enumerate(sc.lights):
        if l.type == scenes.LIGHT_DIRECTIONAL and l.active:
            sc.lights[k] = dataclasses.replace(l, cast_shadows=True)
            break
    return sc


def test_batch_shadow_equals_single_viewport_frames(cuda_device, ibl):
    """A scene whose sun casts shadows: every viewport of the batch equals
    the plain frame rendered after the plain path's shadow pass, and a TRS
    update between launches moves the shadows as it moves them there."""
    sc = _shadowed(_scene(instances=16))
    b = mopcuda.BatchRenderer(cuda_device, sc, _views(sc, 6, seed=11), ibl)
    try:
        b.render()
        _check_batch(cuda_device, b, sc, ibl, "shadow batch")
        m = sc.meshes[3].transform.copy()
        m[12:15] += np.float32(2.0)
        b.set_model(3, m)
        b.render()
        moved = dataclasses.replace(sc, meshes=[dataclasses.replace(x, transform=m) if k == 3
                                                else x for k, x in enumerate(sc.meshes)])
        _check_batch(cuda_device, b, moved, ibl, "shadow batch after TRS")
    finally:
        b.close()


def _blended(sc):
    """Every third instance blended (alpha / additive / multiply, opacity
    0.35-0.75): each viewport sorts them back to front for its own eye."""
    for k in range(0, len(sc.meshes), 3):
        sc.meshes[k] = dataclasses.replace(sc.meshes[k], opacity=0.35 + 0.1 * (k % 5),
                                           blend_mode=(1, 2, 3, 1)[k % 4])
    return sc


def test_batch_blended_equals_single_viewport_frames(cuda_device, ibl):
    """Blended instances: every viewport composites its ordered suffix in the
    core's back-to-front order for its own camera, as the plain frame does;
    a TRS update that changes a blended instance's distance reorders it."""
    sc = _blended(_scene(instances=24))
    b = mopcuda.BatchRenderer(cuda_device, sc, _views(sc, 8, seed=21), ibl)
    try:
        b.render()
        _check_batch(cuda_device, b, sc, ibl, "blended batch")
        m = sc.meshes[3].transform.copy()
        m[12:15] *= np.float32(-1.5)
        b.set_model(3, m)
        b.render()
        moved = dataclasses.replace(sc, meshes=[dataclasses.replace(x, transform=m) if k == 3
                                                else x for k, x in enumerate(sc.meshes)])
        _check_batch(cuda_device, b, moved, ibl, "blended batch after TRS")
    finally:
        b.close()


def test_batch_blended_shadow_and_unlit(cuda_device, ibl):
    """Blended instances with the sun casting shadows (blended meshes cast
    none), and a scene without lights (the unlit smooth path, order-dependent
    for every draw): each viewport equals its plain frame."""
    sc = _shadowed(_blended(_scene(instances=12)))
    b = mopcuda.BatchRenderer(cuda_device, sc, _views(sc, 4, seed=22), ibl)
    try:
        b.render()
        _check_batch(cuda_device, b, sc, ibl, "blended shadow batch")
    finally:
        b.close()
    unlit = dataclasses.replace(_scene(instances=8), lights=[])
    b = mopcuda.BatchRenderer(cuda_device, unlit, _views(unlit, 4, seed=23), None)
    try:
        b.render()
        _check_batch(cuda_device, b, unlit, None, "unlit batch")
    finally:
        b.close()


def test_batch_wireframe_equals_single_viewport_frames(cuda_device, ibl):
    """MOP_RENDER_WIREFRAME in a batch (with blended instances, and with the
    sun casting shadows): every viewport's line plots composite in its own
    suffix as in its plain frame; and against the oracle directly."""
    sc = dataclasses.replace(_blended(_scene(instances=10)), wireframe=True)
    b = mopcuda.BatchRenderer(cuda_device, sc, _views(sc, 5, seed=25), ibl)
    try:
        b.render()
        _check_batch(cuda_device, b, sc, ibl, "wireframe batch")
    finally:
        b.close()
    small = dataclasses.replace(scenes.wireframe_scene(seed=26, width=96, height=72),
                                lights=[])
    views = [scenes.View(96, 72, 1, small.eye, small.target, fov_deg=small.fov_deg,
                         near=small.near, far=small.far, clear=small.clear),
             scenes.View(64, 48, 2, (-4.0, 3.0, 5.0), (0.0, 0.4, 0.0), fov_deg=55.0, near=0.1,
                         far=50.0, clear=small.clear)]
    b = mopcuda.BatchRenderer(cuda_device, small, views)
    try:
        b.render()
        for i, v in enumerate(views):
            ref = cpu_oracle.render(scenes.scene_for_view(small, v), None)
            assert_frame_parity(_batch_view(b, i), ref, f"wireframe oracle view {i}")
    finally:
        b.close()


def test_batch_blended_matches_oracle(cuda_device):
    """Blended meshes in a batch against the oracle directly (two cameras,
    different back-to-front orders)."""
    sc = scenes.transparent_scene(seed=24, width=96, height=72)
    views = [scenes.View(96, 72, 1, sc.eye, sc.target, fov_deg=sc.fov_deg, near=sc.near,
                         far=sc.far, clear=sc.clear),
             scenes.View(80, 48, 2, (-5.0, 2.0, -4.0), (0.0, 0.5, 0.0), fov_deg=45.0, near=0.1,
                         far=50.0, clear=sc.clear)]
    b = mopcuda.BatchRenderer(cuda_device, sc, views)
    try:
        b.render()
        for i, v in enumerate(views):
            ref = cpu_oracle.render(scenes.scene_for_view(sc, v), None)
            assert_frame_parity(_batch_view(b, i), ref, f"blended oracle view {i}")
    finally:
        b.close()


def test_batch_read_views_equals_single_reads(cuda_device, ibl):
    """mopcuda_batch_read_views (every view's buffer in one call) returns the
    bytes of one mopcuda_batch_read per view, for each buffer, and rejects a
    wrong size or range before copying anything."""
    import ctypes as C
    sc = _scene()
    b = mopcuda.BatchRenderer(cuda_device, sc, _views(sc, 6, seed=5), ibl)
    try:
        b.render()
        for what in (mopcuda.BATCH_COLOR, mopcuda.BATCH_PRESENTED, mopcuda.BATCH_DEPTH,
                     mopcuda.BATCH_IDS):
            one = [b.read(i, what) for i in range(len(b.views))]
            every = b.read_all(what, [np.zeros_like(x) for x in one])
            for i, (x, y) in enumerate(zip(one, every)):
                assert x.tobytes() == y.tobytes(), f"buffer {what} view {i}"
        outs = [np.full_like(b.read(i, mopcuda.BATCH_IDS), 7) for i in range(len(b.views))]
        ptrs = (C.c_void_p * len(outs))(*[o.ctypes.data for o in outs])
        sizes = (C.c_size_t * len(outs))(*[o.nbytes for o in outs])
        sizes[-1] -= 4
        L = mopcuda.lib()
        assert L.mopcuda_batch_read_views(b.h, 0, len(outs), mopcuda.BATCH_IDS, ptrs, sizes) != 0
        assert all((o == 7).all() for o in outs)  # nothing copied
        sizes[-1] += 4
        assert L.mopcuda_batch_read_views(b.h, 1, len(outs), mopcuda.BATCH_IDS, ptrs, sizes) != 0
    finally:
        b.close()


def test_batch_async_readback_matches_sync(cuda_device, ibl):
    """mopcuda_batch_read_views_async: launches submitted back to back with
    new cameras, each launch's images copied while the next one renders (its
    post passes wait for the copies), equal the synchronous reads of the same
    launches; with no next submit, readback_wait issues the copies.  Depth
    and IDs are refused (they are rewritten before the post passes)."""
    sc = _scene()
    views0 = _views(sc, 8, seed=7)
    steps = [scenes.batch_views(sc, n=8, seed=7 + k, min_px=24 * 24, max_px=320 * 240)
             for k in range(4)]
    # same sizes and SSAA as the batch, new cameras
    steps = [[dataclasses.replace(v0, eye=v.eye, target=v.target) for v0, v in zip(views0, vs)]
             for vs in steps]
    b = mopcuda.BatchRenderer(cuda_device, sc, views0, ibl)
    host = []
    try:
        want = []
        for vs in steps:
            b.set_views(vs)
            b.render()
            want.append([b.read(i, w) for w in (mopcuda.BATCH_PRESENTED, mopcuda.BATCH_COLOR)
                         for i in range(len(vs))])
        assert any((want[0][i] != want[1][i]).any() for i in range(len(views0)))
        for k, vs in enumerate(steps):
            bufs = [mopcuda.HostArray(x.shape, x.dtype) for x in want[k]]
            host.append(bufs)
            b.set_views(vs)
            b.submit()
            n = len(vs)
            b.read_all_async(mopcuda.BATCH_PRESENTED, [h.a for h in bufs[:n]])
            b.read_all_async(mopcuda.BATCH_COLOR, [h.a for h in bufs[n:]])
        b.wait_readback()
        for k in range(len(steps)):
            for i, (h, x) in enumerate(zip(host[k], want[k])):
                assert h.a.tobytes() == x.tobytes(), f"launch {k} buffer {i}"
        ids = [np.zeros_like(b.read(i, mopcuda.BATCH_IDS)) for i in range(len(views0))]
        with pytest.raises(RuntimeError):
            b.read_all_async(mopcuda.BATCH_IDS, ids)
    finally:
        for bufs in host:
            for h in bufs:
                h.close()
        b.close()


def test_batch_matches_oracle(cuda_device):
    sc = scenes.small_scene(seed=4, width=96, height=72)
    views = [scenes.View(96, 72, 1, sc.eye, sc.target, fov_deg=sc.fov_deg, near=sc.near,
                         far=sc.far, clear=sc.clear),
             scenes.View(64, 40, 2, (3.0, 4.0, 6.0), (0.0, 0.3, 0.0), fov_deg=40.0, near=0.1,
                         far=50.0, clear=sc.clear)]
    b = mopcuda.BatchRenderer(cuda_device, sc, views)
    try:
        b.render()
        for i, v in enumerate(views):
            ref = cpu_oracle.render(scenes.scene_for_view(sc, v), None)
            got = _batch_view(b, i)
            assert_frame_parity(got, ref, f"oracle view {i}")
    finally:
        b.close()


def test_batch_launch_configs_and_autotune_do_not_change_results(cuda_device, ibl):
    sc = _scene(instances=16)
    b = mopcuda.BatchRenderer(cuda_device, sc, _views(sc, 6, seed=2), ibl)
    try:
        b.render()
        base = [_batch_view(b, i) for i in range(len(b.views))]
        for cfg in ({"small_side": 8, "small_area": 16, "raster_block": 64},
                    {"small_side": 64, "small_area": 4096, "shade_block": 128, "grid_mul": 2},
                    {"setup_block": 128, "vertex_block": 128, "large_block": 128}):
            b.set_config(**cfg)
            b.render()
            for i in range(len(b.views)):
                _assert_same(_batch_view(b, i), base[i], f"config {cfg} view {i}")
        rep = b.autotune(reps=2)
        assert rep["best_ms"] > 0 and len(rep["trials"]) >= 5
        b.render()
        for i in range(len(b.views)):
            _assert_same(_batch_view(b, i), base[i], f"autotuned view {i}")
    finally:
        b.close()


def test_batch_trs_update_and_camera_change(cuda_device, ibl):
    sc = _scene(instances=12)
    views = _views(sc, 4, seed=3)
    b = mopcuda.BatchRenderer(cuda_device, sc, views, ibl)
    try:
        b.render()
        rng = np.random.default_rng(0)
        for k in (1, 5):
            t = sc.meshes[k].transform.copy()
            t[12:15] += rng.uniform(-2, 2, 3).astype(np.float32)
            sc.meshes[k] = dataclasses.replace(sc.meshes[k], transform=t)
            b.set_model(k, t)
        moved = [dataclasses.replace(v, eye=tuple(np.array(v.eye) * 1.1)) for v in views]
        b.set_views(moved)
        b.render()
        _check_batch(cuda_device, b, sc, ibl, "after update")
    finally:
        b.close()


def test_batch_pool_growth(cuda_device, ibl):
    """Views that all see the whole scene need more than the first pools:
    the batch grows them, re-runs, and still equals the single frames."""
    sc = _scene(instances=10)
    v = scenes.View(200, 120, 1, (0.0, 10.0, 60.0), (0.0, 0.0, 0.0), clear=sc.clear)
    views = [dataclasses.replace(v, eye=(float(x), 10.0, 60.0)) for x in (-6, -2, 2, 6)]
    b = mopcuda.BatchRenderer(cuda_device, sc, views, ibl)
    try:
        b.render()
        _check_batch(cuda_device, b, sc, ibl, "growth")
    finally:
        b.close()
