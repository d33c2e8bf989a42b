"""Bounded waits that run out.  Every host wait of the library is bounded and
returns MOPCUDA_ETIMEOUT (the analogue of the reference's
MOP_RENDER_DEVICE_LOST) instead of blocking; these tests make the limit run
out on real, finite work — a waited frame or request that is still running —
so no kernel is made to hang.  The wait then resumes and the result equals
an unhurried render of the same input.
"""
import dataclasses

import numpy as np
import pytest

import mopcuda
import scenes

pytestmark = pytest.mark.gpu


def test_frame_wait_times_out_then_resumes(cuda_device):
    sc = scenes.config2()  # 1920x1080 SSAA 2, 1.47 M triangles: ~0.6 ms on the device
    r = mopcuda.SceneRenderer(cuda_device, sc)
    try:
        r.render()
        want = {"color": r.color(), "ids": r.object_id(), "depth": r.depth()}
        L, d = r.L, r.dev.h
        r.submit()
        rc = L.mopcuda_frame_wait(d, 0)  # the frame was enqueued microseconds ago
        assert rc == mopcuda.ETIMEOUT, (rc, mopcuda.last_error())
        assert "did not complete within 0 ms" in mopcuda.last_error()
        assert L.mopcuda_frame_wait(d, 20000) == mopcuda.OK, mopcuda.last_error()
        assert (r.color() == want["color"]).all()
        assert (r.object_id() == want["ids"]).all()
        assert (r.depth().view(np.uint32) == want["depth"].view(np.uint32)).all()
    finally:
        r.close()


def test_server_wait_times_out_then_resumes(cuda_device):
    ibl = scenes.procedural_ibl((0.4, 0.8, 0.35), irr_size=(32, 16), pf_size=(64, 32),
                                levels=4, brdf_size=64)
    sc = scenes.config2(seed=7, width=1920, height=1080, ssaa=1, instances=96, tex_size=256)
    rs = mopcuda.ResidentScene(cuda_device, sc, ibl)
    srv = mopcuda.Server(cuda_device, hbm_budget=16 << 30, max_views=32, max_inflight=1)
    try:
        sid = srv.add_scene(rs)
        views = scenes.batch_views(sc, n=32, seed=3, min_px=1280 * 720, max_px=1920 * 1080)
        tickets = [srv.submit_render(sid, v, want_ids=True, want_depth=True) for v in views]
        last = tickets[-1]
        rc = srv.L.mopcuda_server_wait(srv.h, last.id, 0, None)
        assert rc == mopcuda.ETIMEOUT, (rc, mopcuda.last_error())
        assert "not done" in mopcuda.last_error()
        for t in tickets:
            srv.wait(t)
        drain = srv.L.mopcuda_server_drain(srv.h, 20000)
        assert drain == mopcuda.OK
        # the timed-out request's result equals its own plain frame
        v = last.view
        pr = mopcuda.SceneRenderer(cuda_device, scenes.scene_for_view(sc, v), ibl)
        try:
            pr.render()
            assert (last.color == pr.color()).all()
            assert (last.ids == pr.object_id()).all()
            assert (last.depth.view(np.uint32) == pr.depth().view(np.uint32)).all()
        finally:
            pr.close()
    finally:
        srv.close()
        rs.close()
