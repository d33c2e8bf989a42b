"""The served workload and its two drivers.

Workload: resident config-2-style scenes of log-normal size, requests
arriving as a Poisson process; 85% renders at 256x256, 1280x720, 1920x1080
or 2560x1440, 15% batches of 1-64 picks; before each request 1% of its
scene's instances (at least one) get a new TRS.  Latency is measured from a
request's arrival time to its result in host memory.

Drivers:
  * run_server — the continuous-batching server (mopcuda_server_*);
  * run_plain  — the plain per-viewport path: one frame per request
    (frame_begin / draw_list / frame_end / read), first come first served
    on one thread, the same arrival times.
Both render the same requests through libmopcuda.so; neither has a CPU
fallback.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import threading
import time
from typing import List, Optional

import numpy as np

import mopcuda
import scenes

RESOLUTIONS = ((256, 256), (1280, 720), (1920, 1080), (2560, 1440))


@dataclasses.dataclass
class Request:
    t: float                 # arrival, seconds from the start of the trace
    kind: int                # mopcuda.REQ_RENDER / REQ_PICK
    scene: int
    view: scenes.View
    xy: Optional[np.ndarray]
    moves: list              # [(draw index, model)] applied just before submission

    @property
    def pixels(self) -> int:
        return self.view.pixels


def make_trace(scs: List[scenes.Scene], rate: float, duration: float, seed: int = 1,
               trs_frac: float = 0.01) -> List[Request]:
    """Poisson arrivals at `rate` per second for `duration` seconds."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    models = [[m.transform.copy() for m in sc.meshes] for sc in scs]
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration:
            break
        s = int(rng.integers(0, len(scs)))
        sc = scs[s]
        w, h = RESOLUTIONS[int(rng.integers(0, len(RESOLUTIONS)))]
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        eye = tuple(float(x) for x in d * rng.uniform(15.0, 40.0))
        tgt = tuple(float(x) for x in
                    sc.meshes[int(rng.integers(0, len(sc.meshes)))].transform[12:15])
        view = scenes.View(w, h, 1, eye, tgt, clear=sc.clear)
        moves = []
        for k in rng.choice(len(sc.meshes), max(1, int(round(trs_frac * len(sc.meshes)))),
                            replace=False):
            m = models[s][int(k)]
            m[12:15] += rng.uniform(-0.05, 0.05, 3).astype(np.float32)
            moves.append((int(k), m.copy()))
        if rng.random() < 0.15:
            n = int(rng.integers(1, 65))
            xy = np.stack([rng.integers(0, w, n), rng.integers(0, h, n)], 1).astype(np.int32)
            out.append(Request(t, mopcuda.REQ_PICK, s, view, xy, moves))
        else:
            out.append(Request(t, mopcuda.REQ_RENDER, s, view, None, moves))
    return out


def _summary(lat_ms, pixels, wall_s, extra=None):
    lat = np.asarray(lat_ms, np.float64)
    d = {"requests": int(lat.size), "p50_ms": float(np.percentile(lat, 50)),
         "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
         "wall_s": wall_s, "mpix_s": pixels / wall_s / 1e6}
    if extra:
        d.update(extra)
    return d


def _sleep_until(t_abs):
    while True:
        dt = t_abs - time.perf_counter()
        if dt <= 0:
            return
        time.sleep(min(dt, 0.0005) if dt > 0.0002 else 0)


def reset_models(rss, scs):
    """Back to the scenes' initial instance transforms."""
    for rs, sc in zip(rss, scs):
        for k, m in enumerate(sc.meshes):
            rs.set_model(k, m.transform)


class _Ring:
    """Reusable page-locked result buffers of one shape; take() waits while
    the next one still belongs to an unfinished request."""

    def __init__(self, shape, n):
        self.bufs = [mopcuda.HostArray(shape, np.uint8) for _ in range(n)]
        self.free = [threading.Event() for _ in range(n)]
        for e in self.free:
            e.set()
        self.i = 0

    def take(self):
        k = self.i
        self.i = (self.i + 1) % len(self.bufs)
        self.free[k].wait()
        self.free[k].clear()
        return k, self.bufs[k].a

    def close(self):
        for b in self.bufs:
            b.close()


def run_server(dev, rss, trace: List[Request], hbm_budget: int, max_views: int = 64,
               max_inflight: int = 3, batch_window_us: int = 0, keep_every: int = 0,
               ring: int = 64, warmup: Optional[List[Request]] = None,
               max_launch_samples: int = 0) -> dict:
    """Serve the trace (after serving `warmup`, untimed, on the same server).
    Render results land in rings of page-locked buffers per resolution
    (reused once their request completed); keep_every > 0 also keeps every
    k-th render's IDs and depth (for the exactness check) under "kept"."""
    srv = mopcuda.Server(dev, hbm_budget, max_views, max_inflight, batch_window_us,
                         max_launch_samples)
    rings = {(w, h): _Ring((h, w, 4), ring) for w, h in RESOLUTIONS}
    try:
        ids = [srv.add_scene(rs) for rs in rss]

        def serve(tr, keep_every):
            tickets = [None] * len(tr)
            slots = [None] * len(tr)
            lat = [0.0] * len(tr)

            def collector():
                for i in range(len(tr)):
                    while tickets[i] is None:
                        time.sleep(0.0001)
                    lat[i] = srv.wait(tickets[i], 60000)
                    if slots[i] is not None:
                        rg, k = slots[i]
                        rg.free[k].set()

            th = threading.Thread(target=collector, daemon=True)
            t0 = time.perf_counter()
            th.start()
            for i, r in enumerate(tr):
                _sleep_until(t0 + r.t)
                for k, m in r.moves:
                    rss[r.scene].set_model(k, m)
                keep = keep_every and i % keep_every == 0 and r.kind == mopcuda.REQ_RENDER
                if r.kind == mopcuda.REQ_RENDER:
                    out = None
                    if not keep:
                        rg = rings[(r.view.width, r.view.height)]
                        k, out = rg.take()
                        slots[i] = (rg, k)
                    tickets[i] = srv.submit_render(ids[r.scene], r.view, want_ids=bool(keep),
                                                   want_depth=bool(keep), out=out)
                else:
                    tickets[i] = srv.submit_pick(ids[r.scene], r.view, r.xy)
            th.join()
            wall = time.perf_counter() - t0
            kept = {i: tickets[i] for i in range(len(tr))
                    if keep_every and i % keep_every == 0 and tr[i].kind == mopcuda.REQ_RENDER}
            return lat, wall, kept

        if warmup:
            serve(warmup, 0)
        s0 = srv.stats()
        lat, wall, kept = serve(trace, keep_every)
        st = srv.stats()
        for k in ("submitted", "completed", "failed", "launches", "launched_views", "reruns"):
            st[k] -= s0[k]
        pixels = sum(r.pixels for r in trace)
        return _summary(lat, pixels, wall, {"stats": st, "kept": kept})
    finally:
        srv.close()
        for rg in rings.values():
            rg.close()


# ---------------------------------------------------------------------------
# plain per-viewport path
# ---------------------------------------------------------------------------

def _mat_mul_rows(a, b):
    """mop_mat4_multiply for stacks: a (16,) or (n, 16), b (n, 16), float32,
    running sum from 0 in the reference's order (numpy float32 elementwise
    operations round once each, so this equals the C loop)."""
    a = np.broadcast_to(a, b.shape) if a.ndim == 1 else a
    out = np.empty_like(b)
    for c in range(4):
        for r in range(4):
            s = np.zeros(b.shape[0], np.float32)
            for k in range(4):
                s = s + a[:, k * 4 + r] * b[:, c * 4 + k]
            out[:, c * 4 + r] = s
    return out


class PlainScene:
    """One resident scene driven through the per-viewport frame API: its
    draw calls in one array, matrices written per request."""

    def __init__(self, rs):
        self.rs = rs
        n = len(rs._draws)
        self.arr = (mopcuda.MopCudaDraw * n)(*rs._draws)
        size = C.sizeof(mopcuda.MopCudaDraw)
        self.mvp = np.ndarray((n, 16), np.float32, buffer=self.arr,
                              offset=mopcuda.MopCudaDraw.mvp.offset, strides=(size, 4))
        self.model = np.ndarray((n, 16), np.float32, buffer=self.arr,
                                offset=mopcuda.MopCudaDraw.model.offset, strides=(size, 4))
        self.eye = np.ndarray((n, 3), np.float32, buffer=self.arr,
                              offset=mopcuda.MopCudaDraw.cam_eye.offset, strides=(size, 4))

    def set_camera(self, view):
        v, p, e = mopcuda.camera_matrices(view)
        self.mvp[:] = _mat_mul_rows(p, _mat_mul_rows(v, np.ascontiguousarray(self.model)))
        self.eye[:] = e

    def submit(self, dev, fb, view):
        """Records and launches the frame (asynchronous)."""
        L, d = dev.L, dev.h
        clear = (C.c_float * 4)(*view.clear)
        mopcuda._check(L.mopcuda_frame_begin(d, fb, clear), "frame_begin")
        mopcuda._check(L.mopcuda_draw_list(d, fb, C.addressof(self.arr), len(self.arr)),
                       "draw_list")
        mopcuda._check(L.mopcuda_frame_end(d, fb), "frame_end")

    def frame(self, dev, fb, view):
        self.submit(dev, fb, view)
        mopcuda._check(dev.L.mopcuda_frame_wait(dev.h, 20000), "frame_wait")


def check_kept(dev, rss, trace: List[Request], kept: dict) -> dict:
    """Re-renders each kept server request as its own frame (its scene's
    models as of that request) and compares object IDs and depth bits."""
    L, d = dev.L, dev.h
    bad_ids = bad_depth = samples = 0
    for i in sorted(kept):
        r, t = trace[i], kept[i]
        ps = PlainScene(rss[r.scene])
        for j in range(i + 1):
            if trace[j].scene == r.scene:
                for k, m in trace[j].moves:
                    ps.model[k] = m
        ps.set_camera(r.view)
        fb = L.mopcuda_framebuffer_create(d, r.view.width, r.view.height)
        try:
            ps.frame(dev, fb, r.view)
            n = r.view.width * r.view.height
            ids = np.ctypeslib.as_array(C.cast(L.mopcuda_read_object_id(d, fb, None, None),
                                               C.POINTER(C.c_uint32)), shape=(n,)).copy()
            dep = np.ctypeslib.as_array(C.cast(L.mopcuda_read_depth(d, fb, None, None),
                                               C.POINTER(C.c_float)), shape=(n,)).copy()
        finally:
            L.mopcuda_framebuffer_destroy(d, fb)
        bad_ids += int((ids != t.ids.reshape(-1)).sum())
        bad_depth += int((dep.view(np.uint32) != t.depth.reshape(-1).view(np.uint32)).sum())
        samples += n
    return {"checked_requests": len(kept), "checked_samples": samples,
            "id_mismatches": bad_ids, "depth_mismatches": bad_depth}


def run_plain(dev, rss, trace: List[Request], warmup: Optional[List[Request]] = None) -> dict:
    L, d = dev.L, dev.h
    plains = [PlainScene(rs) for rs in rss]
    fbs = {}
    for w, h in RESOLUTIONS:
        fb = L.mopcuda_framebuffer_create(d, w, h)
        L.mopcuda_framebuffer_set_ssaa(fb, 1)
        fbs[(w, h)] = fb
    # page-locked destinations: the image copies are direct DMA, as the server's are
    pinned = {k: mopcuda.HostArray((k[1], k[0], 4), np.uint8) for k in fbs}
    outs = {k: v.a for k, v in pinned.items()}
    lat = []
    try:
        for r in warmup or []:  # untimed: first-use allocations of every frame size
            ps = plains[r.scene]
            ps.set_camera(r.view)
            ps.frame(dev, fbs[(r.view.width, r.view.height)], r.view)
        t0 = time.perf_counter()
        for r in trace:
            _sleep_until(t0 + r.t)
            ps = plains[r.scene]
            for k, m in r.moves:
                ps.model[k] = m
            ps.set_camera(r.view)
            key = (r.view.width, r.view.height)
            ps.frame(dev, fbs[key], r.view)
            if r.kind == mopcuda.REQ_RENDER:
                o = outs[key]
                mopcuda._check(L.mopcuda_read_color_resolved(d, fbs[key], 1, o.ctypes.data,
                                                             o.nbytes), "read_color")
            else:
                n = r.xy.shape[0]
                a, b, c = np.zeros(n, np.uint32), np.zeros(n, np.float32), np.zeros(n, np.int32)
                mopcuda._check(L.mopcuda_pick_batch(d, fbs[key], 1, r.xy.ctypes.data, n,
                                                    a.ctypes.data, b.ctypes.data,
                                                    c.ctypes.data), "pick")
            lat.append((time.perf_counter() - (t0 + r.t)) * 1e3)
        wall = time.perf_counter() - t0
    finally:
        for fb in fbs.values():
            L.mopcuda_framebuffer_destroy(d, fb)
        for v in pinned.values():
            v.close()
    return _summary(lat, sum(r.pixels for r in trace), wall)
