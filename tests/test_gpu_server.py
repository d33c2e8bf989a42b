"""Request server (mopcuda_server_*): continuous batching over resident
scenes.  A request's result is the same alone and in a mix of other scenes,
sizes, SSAA factors and pick requests, and equals the single-viewport frame
of the same draws and camera; admission respects the HBM budget (a budget
too small for two requests runs them one launch at a time, same results)
and the per-launch sample cap.
"""
import dataclasses

import numpy as np
import pytest

import mopcuda
import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def world(cuda_device):
    ibl = scenes.procedural_ibl((0.4, 0.8, 0.35), irr_size=(32, 16), pf_size=(64, 32),
                                levels=4, brdf_size=64)
    scs = [scenes.config2(seed=s, width=160, height=90, ssaa=1, instances=n, tex_size=64)
           for s, n in ((11, 10), (12, 16), (13, 6))]
    rss = [mopcuda.ResidentScene(cuda_device, sc, ibl) for sc in scs]
    yield scs, rss, ibl
    for rs in rss:
        rs.close()


def _views(sc, n, seed):
    return scenes.batch_views(sc, n=n, seed=seed, min_px=32 * 32, max_px=240 * 160)


def _plain(dev, sc, v, ibl, xy=None):
    r = mopcuda.SceneRenderer(dev, scenes.scene_for_view(sc, v), ibl)
    try:
        r.render()
        out = {"color": r.color(), "ids": r.object_id(), "depth": r.depth()}
        if xy is not None:
            out["pick"] = r.pick(xy)
        return out
    finally:
        r.close()


def _same_render(t, want, label):
    assert (t.color == want["color"]).all(), f"{label}: colour differs"
    assert (t.ids == want["ids"]).all(), f"{label}: IDs differ"
    assert (t.depth.view(np.uint32) == want["depth"].view(np.uint32)).all(), f"{label}: depth"


def _same_pick(got, want, label):
    for a, b in zip(got, want):
        assert (np.asarray(a).view(np.uint32) == np.asarray(b).view(np.uint32)).all(), label


def test_server_alone_equals_mix_equals_frame(cuda_device, world):
    scs, rss, ibl = world
    srv = mopcuda.Server(cuda_device, hbm_budget=8 << 30, max_views=16, max_inflight=2)
    try:
        sid = [srv.add_scene(rs) for rs in rss]
        probe_v = dataclasses.replace(_views(scs[1], 1, seed=5)[0], ssaa=2)
        pick_v = _views(scs[2], 1, seed=6)[0]
        xy = scenes.pick_points(dataclasses.replace(scs[2], width=pick_v.width,
                                                    height=pick_v.height), 48, seed=2)
        # alone
        a = srv.submit_render(sid[1], probe_v, want_ids=True, want_depth=True)
        srv.wait(a)
        ap = srv.submit_pick(sid[2], pick_v, xy)
        srv.wait(ap)
        # in a mix: 40 requests over all scenes, the probes in the middle
        rng = np.random.default_rng(9)
        mix = []
        for k in range(40):
            s = int(rng.integers(0, 3))
            v = _views(scs[s], 1, seed=100 + k)[0]
            if k % 7 == 3:
                pts = scenes.pick_points(dataclasses.replace(scs[s], width=v.width,
                                                             height=v.height), 16, seed=k)
                mix.append(srv.submit_pick(sid[s], v, pts))
            else:
                mix.append(srv.submit_render(sid[s], v))
            if k == 20:
                b = srv.submit_render(sid[1], probe_v, want_ids=True, want_depth=True)
                bp = srv.submit_pick(sid[2], pick_v, xy)
        for t in mix + [b, bp]:
            srv.wait(t)
        assert (a.color == b.color).all() and (a.ids == b.ids).all()
        assert (a.depth.view(np.uint32) == b.depth.view(np.uint32)).all()
        _same_pick(ap.pick, bp.pick, "pick alone vs mix")
        st = srv.stats()
        assert st["completed"] == 44 and st["failed"] == 0
        assert st["launches"] < st["completed"] and st["max_views_in_launch"] > 1, st
        # and both equal the request's own frame
        want = _plain(cuda_device, scs[1], probe_v, ibl)
        _same_render(b, want, "probe vs frame")
        wantp = _plain(cuda_device, scs[2], pick_v, ibl, xy)
        _same_pick(bp.pick, wantp["pick"], "pick vs frame")
        for t in mix[:12]:
            if t.kind == mopcuda.REQ_RENDER:
                w = _plain(cuda_device, scs[sid.index(t.req.scene)], t.view, ibl)
                assert (t.color == w["color"]).all(), "mix render vs frame"
    finally:
        srv.close()


def test_server_budget_admission(cuda_device, world):
    scs, rss, ibl = world
    srv = mopcuda.Server(cuda_device, hbm_budget=1, max_views=16, max_inflight=2)
    try:
        sid = srv.add_scene(rss[0])
        views = _views(scs[0], 6, seed=7)
        ts = [srv.submit_render(sid, v, want_ids=True, want_depth=True) for v in views]
        for t in ts:
            srv.wait(t)
        st = srv.stats()
        assert st["max_views_in_launch"] == 1 and st["launches"] == 6, st
        for t, v in zip(ts, views):
            _same_render(t, _plain(cuda_device, scs[0], v, ibl), "budget-limited")
    finally:
        srv.close()


def test_server_launch_sample_cap(cuda_device, world):
    """max_launch_samples: a launch takes requests only while their samples
    fit the cap (three 64x64 views here), a request larger than the cap
    still runs, alone, and every result equals the request's own frame."""
    scs, rss, ibl = world
    side = 64
    cap = 3 * side * side
    srv = mopcuda.Server(cuda_device, hbm_budget=8 << 30, max_views=16, max_inflight=2,
                         max_launch_samples=cap)
    try:
        sid = srv.add_scene(rss[1])
        views = [dataclasses.replace(v, width=side, height=side, ssaa=1)
                 for v in _views(scs[1], 12, seed=21)]
        big = dataclasses.replace(views[0], width=2 * side, height=2 * side, ssaa=1)
        ts = [srv.submit_render(sid, v, want_ids=True, want_depth=True) for v in views]
        tb = srv.submit_render(sid, big, want_ids=True, want_depth=True)
        for t in ts + [tb]:
            srv.wait(t)
        st = srv.stats()
        assert st["completed"] == 13 and st["failed"] == 0, st
        assert st["max_views_in_launch"] <= 3 and st["launches"] >= 5, st
        for t, v in zip(ts + [tb], views + [big]):
            _same_render(t, _plain(cuda_device, scs[1], v, ibl), f"capped {v.width}x{v.height}")
    finally:
        srv.close()


def test_served_requests_match_oracle(cuda_device):
    """Served requests of a config-2-style scene (1024^2 textures, IBL, the
    config-2 lights) checked directly against the CPU oracle: IDs and depth
    bit-exact, the presented colour within the contract, for renders at two
    sizes and SSAA factors sharing launches with each other."""
    import cpu_oracle
    from parity import color_stats, COLOR_MAX_LSB, COLOR_1LSB_FRACTION
    ibl = scenes.procedural_ibl((0.4, 0.8, 0.35), irr_size=(32, 16), pf_size=(64, 32),
                                levels=4, brdf_size=64)
    sc = scenes.served_scene(5, 60_000, tex_size=1024, width=320, height=180)
    rs = mopcuda.ResidentScene(cuda_device, sc, ibl)
    srv = mopcuda.Server(cuda_device, hbm_budget=8 << 30, max_views=8, max_inflight=2)
    try:
        sid = srv.add_scene(rs)
        views = scenes.batch_views(sc, n=4, seed=13, min_px=160 * 90, max_px=320 * 180)
        views[1] = dataclasses.replace(views[1], ssaa=2)
        ts = [srv.submit_render(sid, v, want_ids=True, want_depth=True) for v in views]
        for t in ts:
            srv.wait(t)
        for k, (t, v) in enumerate(zip(ts, views)):
            ref = cpu_oracle.render(scenes.scene_for_view(sc, v), ibl)
            assert (t.ids == ref["object_id"]).all(), f"request {k}: IDs"
            assert (t.depth.view(np.uint32) == ref["depth"].view(np.uint32)).all(), \
                f"request {k}: depth"
            st = color_stats(t.color, ref["color"])
            assert st["max"] <= COLOR_MAX_LSB and st["within1"] >= COLOR_1LSB_FRACTION, (k, st)
            assert (t.ids != 0).any()
    finally:
        srv.close()
        rs.close()


def test_server_shadowed_scene_in_a_mix(cuda_device, world):
    """A scene whose sun casts shadows served beside unshadowed ones: each
    request equals its own plain frame (shadow pass included), and a request
    submitted after a TRS update sees the moved caster's shadow while the
    earlier one keeps the old."""
    scs, rss, ibl = world
    sc = scenes.config2(seed=14, width=160, height=90, ssaa=1, instances=12, tex_size=64)
    for k, l in enumerate(sc.lights):
        if l.type == scenes.LIGHT_DIRECTIONAL:
            sc.lights[k] = dataclasses.replace(l, cast_shadows=True)
            break
    rs = mopcuda.ResidentScene(cuda_device, sc, ibl)
    srv = mopcuda.Server(cuda_device, hbm_budget=8 << 30, max_views=16, max_inflight=2)
    try:
        sid = [srv.add_scene(r) for r in rss] + [srv.add_scene(rs)]
        v = _views(sc, 1, seed=31)[0]
        first = srv.submit_render(sid[3], v, want_ids=True, want_depth=True)
        others = [srv.submit_render(sid[k % 3], _views(scs[k % 3], 1, seed=40 + k)[0])
                  for k in range(5)]
        m = sc.meshes[2].transform.copy()
        m[12:15] += np.float32(1.5)
        rs.set_model(2, m)
        second = srv.submit_render(sid[3], v, want_ids=True, want_depth=True)
        for t in [first, second] + others:
            srv.wait(t)
        _same_render(first, _plain(cuda_device, sc, v, ibl), "shadowed before TRS")
        moved = dataclasses.replace(sc, meshes=[dataclasses.replace(x, transform=m) if k == 2
                                                else x for k, x in enumerate(sc.meshes)])
        _same_render(second, _plain(cuda_device, moved, v, ibl), "shadowed after TRS")
        for t in others:
            s_ = scs[sid.index(t.req.scene)]
            assert (t.color == _plain(cuda_device, s_, t.view, ibl)["color"]).all()
    finally:
        srv.close()
        rs.close()


def test_server_blended_scene_in_a_mix(cuda_device, world):
    """A scene with blended instances served beside opaque ones in the same
    launches: each request (its own camera, so its own back-to-front order)
    equals its plain frame, and the opaque requests are unchanged."""
    scs, rss, ibl = world
    sc = scenes.config2(seed=15, width=160, height=90, ssaa=1, instances=15, tex_size=64)
    for k in range(0, len(sc.meshes), 3):
        sc.meshes[k] = dataclasses.replace(sc.meshes[k], opacity=0.4 + 0.1 * (k % 4),
                                           blend_mode=(1, 2, 3)[k % 3])
    rs = mopcuda.ResidentScene(cuda_device, sc, ibl)
    srv = mopcuda.Server(cuda_device, hbm_budget=8 << 30, max_views=16, max_inflight=2)
    try:
        sid = [srv.add_scene(r) for r in rss] + [srv.add_scene(rs)]
        vs = _views(sc, 3, seed=51)
        mine = [srv.submit_render(sid[3], v, want_ids=True, want_depth=True) for v in vs]
        others = [srv.submit_render(sid[k % 3], _views(scs[k % 3], 1, seed=60 + k)[0])
                  for k in range(4)]
        for t in mine + others:
            srv.wait(t)
        for k, (t, v) in enumerate(zip(mine, vs)):
            _same_render(t, _plain(cuda_device, sc, v, ibl), f"blended request {k}")
        for t in others:
            s_ = scs[sid.index(t.req.scene)]
            assert (t.color == _plain(cuda_device, s_, t.view, ibl)["color"]).all()
    finally:
        srv.close()
        rs.close()


def test_server_trs_update_between_requests(cuda_device, world):
    scs, rss, ibl = world
    srv = mopcuda.Server(cuda_device, hbm_budget=8 << 30, max_views=8, max_inflight=2)
    try:
        sid = srv.add_scene(rss[2])
        v = _views(scs[2], 1, seed=8)[0]
        sc = scs[2]
        m = sc.meshes[0].transform.copy()
        m[12:15] += np.float32(0.75)
        rss[2].set_model(0, m)
        t = srv.submit_render(sid, v, want_ids=True, want_depth=True)
        srv.wait(t)
        moved = dataclasses.replace(sc, meshes=[dataclasses.replace(sc.meshes[0], transform=m)]
                                    + sc.meshes[1:])
        _same_render(t, _plain(cuda_device, moved, v, ibl), "after TRS update")
        rss[2].set_model(0, sc.meshes[0].transform)
    finally:
        srv.close()
