"""The allocation-free batched pick (mopcuda_pick_batch_noalloc) must return
exactly what mopcuda_pick_batch returns — object IDs, depths and hit flags
are bit-exact in this project — on two calls in a row with different
queries.  Those callers (fixed-budget hosts, threads that must not call
cudaMalloc/cudaFree, embedders that forbid allocation after start-up) get
their query staging from a file-scope device array instead of allocations.

Collected last (file name) so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

import mopcuda
import scenes

pytestmark = pytest.mark.gpu


def _noalloc(r, xy):
    xy = np.ascontiguousarray(xy, np.int32)
    n = xy.shape[0]
    ids = np.zeros(n, np.uint32)
    dep = np.zeros(n, np.float32)
    hits = np.zeros(n, np.int32)
    rc = r.L.mopcuda_pick_batch_noalloc(r.dev.h, r.fb, r.scene.ssaa, xy.ctypes.data, n,
                                        ids.ctypes.data, dep.ctypes.data, hits.ctypes.data)
    assert rc == mopcuda.OK, mopcuda.last_error()
    return ids, dep, hits


def test_noalloc_pick_matches_pick_batch():
    dev = mopcuda.Device(0)
    sc = scenes.small_scene(seed=31, width=200, height=150, ssaa=2)
    r = mopcuda.SceneRenderer(dev, sc)
    try:
        r.render()
        queries = []
        for seed in (1, 2):
            xy = scenes.pick_points(sc, 3000 if seed == 1 else 1200, seed=seed)
            xy[:7] = [(-1, 0), (0, -1), (sc.width, 0), (0, sc.height), (0, 0),
                      (sc.width - 1, sc.height - 1), (sc.width // 2, sc.height // 2)]
            queries.append((xy, r.pick(xy)))
        # two calls of the allocation-free entry point in a row
        got = [_noalloc(r, xy) for xy, _ in queries]
        for (xy, want), have in zip(queries, got):
            for a, b in zip(want, have):
                assert (a.view(np.uint32) == b.view(np.uint32)).all()
            assert want[2].sum() > 0  # some queries hit geometry
        too_many = np.zeros((65537, 2), np.int32)
        out = np.zeros(65537, np.uint32)
        rc = r.L.mopcuda_pick_batch_noalloc(r.dev.h, r.fb, 1, too_many.ctypes.data, 65537,
                                            out.ctypes.data, out.ctypes.data, out.ctypes.data)
        assert rc == mopcuda.EINVAL
        assert "limit" in mopcuda.last_error()
        # no queries: nothing to do, nothing touched
        rc = r.L.mopcuda_pick_batch_noalloc(r.dev.h, r.fb, sc.ssaa, None, 0, None, None, None)
        assert rc == mopcuda.OK
    finally:
        r.close()
        dev.close()


def test_noalloc_pick_refuses_pending_frame():
    """With the framebuffer's frame still in flight the call returns EINVAL
    (completing the frame could reallocate); after mopcuda_frame_wait it
    answers as mopcuda_pick_batch does."""
    dev = mopcuda.Device(0)
    sc = scenes.small_scene(seed=32, width=160, height=120)
    r = mopcuda.SceneRenderer(dev, sc)
    try:
        r.render()
        xy = np.ascontiguousarray(scenes.pick_points(sc, 500, seed=4), np.int32)
        n = xy.shape[0]
        out = [np.zeros(n, np.uint32), np.zeros(n, np.float32), np.zeros(n, np.int32)]
        r.submit()  # launched, not waited for
        rc = r.L.mopcuda_pick_batch_noalloc(r.dev.h, r.fb, sc.ssaa, xy.ctypes.data, n,
                                            *[o.ctypes.data for o in out])
        # pending is host state (set by frame_end, cleared by frame_wait), so this holds
        # however far the device has got
        assert rc == mopcuda.EINVAL and "pending" in mopcuda.last_error()
        r.wait()
        got = _noalloc(r, xy)
        for a, b in zip(r.pick(xy), got):
            assert (a.view(np.uint32) == b.view(np.uint32)).all()
    finally:
        r.close()
        dev.close()
