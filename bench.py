#!/usr/bin/env python
"""Frame-path benchmark: Mpix/s (and Mtri/s) of the CUDA backend on one B200.

Workload (default): the large static scene — 1920x1080 presented, SSAA 2
(3840x2160 = 8.29 M samples), 256 mesh instances (1,470,464 triangles:
icospheres subdiv 4-6 and 64x128 tori) with random TRS, 1 directional +
4 point + 2 spot lights, 1024^2 value-noise base-colour textures, IBL maps
of the reference's sizes, ACES resolve, FXAA + gamma, SSAA box.  A "step" is
one frame of that scene: the draw table is uploaded, then vertex transform,
setup/clip, binning, tile visibility + shading + resolve and post run on the
device; the scene's buffers and textures are resident in HBM.

Value:  presented pixels of all ranks' frames / max-over-ranks device time
        (CUDA events recorded by libmopcuda.so on its own stream around each
        frame; an L2-sized buffer is rewritten between timed frames).
e2e:    the same metric through the public C ABI with host buffers: every
        step records the frame on the host (draw table H2D from pinned
        staging) and reads the resolved RGBA8 image back into pinned host
        memory; wall clock, max over ranks.
Multi-GPU: replicas only — every rank renders its own frames of its own copy
        of the scene (weak scaling); no collective on the data path.
--impl reference: the reference library's own CPU backend (built from the
        reference sources into oracle/_ref) renders the same workload on the
        host cores, rank 0 only.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "master-of-puppets_b200"))

HBM_FALLBACK_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["cuda", "reference"], default="cuda")
    ap.add_argument("--config", choices=["config2", "config1"], default="config2")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--flush-mb", type=int, default=256)
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the batched (64 viewports) and served (32 scenes) forms")
    ap.add_argument("--forms-only", action="store_true",
                    help="run only the batched and served forms (one JSON line)")
    ap.add_argument("--form", choices=["all", "batched", "served", "shadowed", "ibl",
                                           "scene_load", "config3", "config1", "transparent"],
                    default="all",
                    help="with --forms-only: which form to run")
    return ap.parse_args()


L2_NOTE = ("frame working set (~170 MB of geometry, samples and images) is larger than the "
           "126 MB L2; the GPU arm also rewrites a 256 MiB buffer between timed frames")


def config_dict(desc, world, sc):
    """The `config` object both arms print (identical keys and values for one
    workload and rank count)."""
    return {"workload": desc, "parallelism": f"replicas x{world}", "l2": L2_NOTE,
            "samples": sc.samples, "pixels": sc.pixels, "triangles": sc.triangle_count}


def workload(name):
    import scenes
    if name == "config1":
        sc = scenes.config1()
        desc = ("config1: 800x600 ssaa1, UV sphere 64x32 + ground plane, 1 directional light, "
                "untextured GGX")
    else:
        sc = scenes.config2()
        desc = ("config2: 1920x1080 ssaa2 (3840x2160 samples), 256 instances / 1,470,464 tris "
                "(icosphere s4-s6 + torus 64x128), 1 dir + 4 point + 2 spot lights, 1024^2 "
                "textures, IBL maps 64x32 / 128x64x5 / 256^2, ACES, FXAA+gamma, SSAA box")
    return sc, desc


def read_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """Samples SM clock and clock-event reasons through NVML while running."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, cuda_index):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self.ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            idx = cuda_index
            if vis:
                parts = [p.strip() for p in vis.split(",") if p.strip()]
                if cuda_index < len(parts) and parts[cuda_index].isdigit():
                    idx = int(parts[cuda_index])
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(idx)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.ok = False
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        nv = self.nv
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            getattr(nv, "nvmlDeviceGetCurrentClocksThrottleReasons")
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                r = get_reasons(self.h)
                for bit, name in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            self._stop.wait(0.01)

    def start(self):
        if self.ok:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()

    def stop(self):
        if self._t:
            self._stop.set()
            self._t.join()
        s = sorted(self.samples)
        return {"sm_mhz": s[len(s) // 2] if s else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(s)}


def pair_traffic():
    """DRAM bytes (read + write) of one k_resolve + k_shade frame from the
    committed ncu capture summary, or None."""
    try:
        t = json.loads((ROOT / "profiles" / "traffic_config2.json").read_text())["per_launch"]
        mb = sum(t[k]["dram_read_mb"] + t[k]["dram_write_mb"] for k in ("k_resolve", "k_shade"))
        return round(mb * 1e6)
    except Exception:
        return None


def dist_setup(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def cpu_reference_time(config, budget_s=60.0, warm=2, frames=10):
    """The reference CPU backend (oracle/_ref, built from the reference
    sources) timed on the host cores, each attempt in a subprocess under a
    timeout.  The reference sizes its tile pool from the online CPU count and
    stalls when that oversubscribes the host, so the pool is tried with half
    the usable cores, then the reference's serial path; the faster completed
    attempt is reported with the thread count it used."""
    ncpu = len(os.sched_getaffinity(0))
    attempts = [max(1, ncpu // 2 - 1), 0]
    best, modes = None, {}
    for workers in attempts:
        cmd = [sys.executable, str(ROOT / "oracle" / "time_reference.py"), "--config", config,
               "--workers", str(workers), "--warm", str(warm), "--frames", str(frames),
               "--budget-s", str(budget_s)]
        try:
            p = subprocess.run(cmd, capture_output=True, text=True, timeout=budget_s + 60)
            if p.returncode != 0:
                continue
            t = json.loads(p.stdout.strip().splitlines()[-1])
        except (subprocess.TimeoutExpired, ValueError, IndexError):
            continue
        modes[t["mode"]] = {"ms": round(t["ms"], 3), "threads": t["threads"]}
        if best is None or t["ms"] < best["ms"]:
            best = t
    if best is None:
        raise RuntimeError("reference CPU backend did not complete a frame in time")
    return {"ms": best["ms"], "frames": best["frames"], "cores": best["threads"],
            "kind": "reference", "mode": best["mode"], "modes": modes, "warm": warm}


def emit(line):
    print(json.dumps(line), flush=True)


def max_over_ranks(x, dist=None, device="cpu"):
    """Max of a per-rank float over the process group (identity when alone)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate(local_ms, steps, world, pixels, triangles, dist=None, device="cpu"):
    """Replica aggregation: every rank rendered `steps` frames of `pixels`
    presented pixels; the job's time is the slowest rank's.  Returns
    (max_ms, Mpix/s, Mtri/s) for the whole job."""
    total = max_over_ranks(local_ms, dist, device)
    return (total, world * steps * pixels / (total * 1e3),
            world * steps * triangles / (total * 1e3))


def run_reference(args):
    rank, world, local = dist_setup(args)
    if rank != 0:
        return 0
    sc, desc = workload(args.config)
    warm = max(0, args.warmup)
    steps = max(1, args.steps)
    # every warm-up and timed frame of the driver's counts, each mode bounded in time
    t = cpu_reference_time(args.config, budget_s=150.0, warm=warm, frames=steps)
    mpix = sc.pixels / (t["ms"] * 1e3)
    line = {"impl": "reference", "metric": "Mpix/s", "value": round(mpix, 4), "unit": "Mpix/s",
            "n_gpus": args.gpus, "steps": t["frames"], "warmup": warm,
            "ms_per_step": round(t["ms"], 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
            "config": config_dict(desc, 1, sc),
            "backend": f"reference CPU backend ({t['mode']})",
            "mtri_per_s": round(sc.triangle_count / (t["ms"] * 1e3), 5),
            "cpu_baseline": {"value": round(mpix, 4), "unit": "Mpix/s", "cores": t["cores"],
                             "kind": t["kind"],
                             "sample": f"{t['frames']} full frame(s) ({t['mode']}), median wall "
                                       "time of mop_viewport_render + mop_viewport_read_color",
                             "modes": t["modes"]},
            "e2e": {"value": round(mpix, 4), "unit": "Mpix/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    emit(line)
    return 0


def run_cuda(args):
    rank, world, local = dist_setup(args)
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    import mopcuda
    import scenes
    sc, desc = workload(args.config)
    ibl = scenes.procedural_ibl(sc.sun_dir) if sc.env else None
    dev = mopcuda.Device(local)
    r = mopcuda.SceneRenderer(dev, sc, ibl)
    flush = torch.empty(args.flush_mb * (1 << 20) // 4, dtype=torch.float32, device="cuda")
    warm = max(3, args.warmup)
    steps = max(1, args.steps)

    # ---- device-timed frames (no stage events inside the timed frames) ----
    dev.set_stage_timing(False)
    for _ in range(warm):
        r.render()
    ids = r.object_id()
    covered = int((ids != 0).sum())
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    frame_ms = []
    l0 = dev.launches
    for _ in range(steps):
        flush.add_(1.0)  # rewrite > L2 (126 MB) between frames
        torch.cuda.synchronize()
        r.render()
        frame_ms.append(r.gpu_ms)
    launches = dev.launches - l0
    barrier()
    clocks = sampler.stop()
    # ---- per-stage times: the same frames again with events between the stages ----
    dev.set_stage_timing(True)
    stage = {k: 0.0 for k in mopcuda.Device.STAGES}
    for _ in range(steps):
        flush.add_(1.0)
        torch.cuda.synchronize()
        r.render()
        for k, v in dev.stage_times().items():
            stage[k] += v
    total_ms, value, mtri = aggregate(sum(frame_ms), steps, world, sc.pixels,
                                      sc.triangle_count, dist, "cuda")

    # ---- end to end through the C ABI with host buffers ----
    # Each step uploads its draw table and lights (pinned, inside frame_end)
    # and reads its presented image back into page-locked host memory; the
    # readback of frame k runs on the copy stream while frame k+1 renders
    # (mopcuda_read_color_resolved_async), into two alternating buffers.
    dev.set_stage_timing(False)
    outs = [torch.empty((sc.height, sc.width, 4), dtype=torch.uint8, pin_memory=True).numpy()
            for _ in range(2)]
    for k in range(warm):
        r.submit()
        r.color_async(outs[k % 2])
    r.wait_readback()
    barrier()
    t0 = time.perf_counter()
    for k in range(steps):
        r.submit()
        r.color_async(outs[k % 2])
    r.wait_readback()
    t1 = time.perf_counter()
    barrier()
    e2e_ms = max_over_ranks((t1 - t0) * 1e3, dist, "cuda")
    e2e = world * steps * sc.pixels / (e2e_ms * 1e3)
    # the same steps with the synchronous readback (no overlap), for reference
    t0 = time.perf_counter()
    for _ in range(steps):
        r.submit()
        r.color(outs[0])
    t1 = time.perf_counter()
    barrier()
    sync_ms = max_over_ranks((t1 - t0) * 1e3, dist, "cuda")
    h2d, d2h = dev.frame_io_bytes()
    d2h += outs[0].nbytes

    # ---- roofline of the dominant kernel (tile visibility + shading) ----
    hbm_peak, peak_kind = read_peaks()
    tile_ms = (stage["resolve"] + stage["shade"]) / steps
    tile_bytes = 12 * sc.samples  # colour RGBA8 + depth f32 + id u32 written per sample
    achieved = tile_bytes / (tile_ms * 1e-3) / 1e9
    fp32_peak = dev.fp32_peak_gops()
    L = sum(1 for l in sc.lights if l.active)
    ops_per_sample = 80 + 120 * L + (150 if sc.env else 0)
    alu_achieved = covered * ops_per_sample / (tile_ms * 1e-3) / 1e9
    frame_bytes = frame_bytes_of(sc)

    line = {"metric": "Mpix/s", "value": round(value, 3), "unit": "Mpix/s", "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": round(total_ms / steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene generator, procedural IBL maps)",
            "config": config_dict(desc, world, sc),
            "l2_flush": f"{args.flush_mb} MiB buffer rewritten between timed frames",
            "mtri_per_s": round(mtri, 3),
            "stage_ms": {k: round(v / steps, 4) for k, v in stage.items()},
            "frame_algorithmic_bytes": frame_bytes,
            "roofline": {"bound": "hbm", "kernel": "k_resolve + k_shade (deferred shading + ACES)",
                         "achieved": round(achieved, 1), "peak": hbm_peak,
                         "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
                         "peak_source": peak_kind, "traffic": pair_traffic(),
                         "alu": {"achieved": round(alu_achieved, 1), "peak": round(fp32_peak, 1),
                                 "unit": "Gop/s (fp32 add/mul, no FMA)",
                                 "frac": round(alu_achieved / fp32_peak, 4) if fp32_peak else None,
                                 "ops_per_covered_sample": ops_per_sample,
                                 "covered_samples": covered}},
            "e2e": {"value": round(e2e, 3), "unit": "Mpix/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": round(e2e_ms / steps, 4),
                    "readback": "async, overlapping the next frame",
                    "sync_readback_mpix_s": round(world * steps * sc.pixels / (sync_ms * 1e3), 3)},
            "gpu_launches": launches,
            "clocks": clocks}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            t = cpu_reference_time(args.config)
            line["cpu_baseline"] = {
                "value": round(sc.pixels / (t["ms"] * 1e3), 4), "unit": "Mpix/s",
                "cores": t["cores"], "kind": t["kind"],
                "sample": f"{t['frames']} full frame(s) of the same scene after {t['warm']} "
                          f"warm-up frame(s) ({t['mode']}, median of mop_viewport_render + "
                          "read_color)",
                "modes": t["modes"]}  # the tile pool and the serial path (the parity reference)
        except Exception as e:  # report, do not fail the GPU measurement
            line["cpu_baseline"] = {"value": None, "unit": "Mpix/s", "error": str(e)[:200]}
    r.close()
    dev.close()
    if rank == 0 and world == 1 and not args.no_forms:
        line.update(forms_subprocess())
    if rank == 0:
        emit(line)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def run_batched(dev, steps=10, warm=3, n_views=64):
    """64 viewports of uneven size, camera and SSAA over the large static
    scene in one CUDA-graph launch, against the plain per-viewport frames of
    the same viewports (both read every presented image back to host)."""
    import ctypes as C
    import numpy as np
    import mopcuda
    import scenes
    import serving
    sc = scenes.config2()
    ibl = scenes.procedural_ibl(sc.sun_dir)
    views = scenes.batch_views(sc, n=n_views, seed=4)
    pixels = sum(v.pixels for v in views)
    b = mopcuda.BatchRenderer(dev, sc, views, ibl)
    outs = [mopcuda.HostArray((v.height, v.width, 4), np.uint8) for v in views]
    try:
        default_cfg = b.config()
        tuned = b.autotune(5)  # block shapes and raster limits picked on this batch
        for _ in range(warm):
            b.render()
        gms, t0 = [], time.perf_counter()
        for _ in range(steps):
            b.render()
            gms.append(b.gpu_ms)
            b.read_all(mopcuda.BATCH_PRESENTED, [o.a for o in outs])
        wall_b = (time.perf_counter() - t0) / steps
        # back to back: each launch's images copied while the next one renders
        second = [mopcuda.HostArray((v.height, v.width, 4), np.uint8) for v in views]
        sets = [outs, second]
        try:
            for k in range(warm):
                b.submit()
                b.read_all_async(mopcuda.BATCH_PRESENTED, [o.a for o in sets[k % 2]])
            b.wait_readback()
            t0 = time.perf_counter()
            for k in range(steps):
                b.submit()
                b.read_all_async(mopcuda.BATCH_PRESENTED, [o.a for o in sets[k % 2]])
            b.wait_readback()
            wall_pipe = (time.perf_counter() - t0) / steps
        finally:
            for o in second:
                o.close()
        cfg = b.config()
        # plain: one frame per viewport through the per-viewport C ABI
        L, d = dev.L, dev.h
        ps = serving.PlainScene(b)
        fbs = []
        for v in views:
            fb = L.mopcuda_framebuffer_create(d, v.width * v.ssaa, v.height * v.ssaa)
            L.mopcuda_framebuffer_set_ssaa(fb, v.ssaa)
            fbs.append(fb)

        def plain_gpu_pass():
            """Device time of every viewport's frame (each waited for)."""
            g = 0.0
            for v, fb in zip(views, fbs):
                ps.set_camera(v)
                ps.frame(dev, fb, v)
                g += L.mopcuda_frame_gpu_time_ms(d)
            return g

        def plain_pass():
            """The plain path's best mode: each viewport's frame recorded while
            the previous one renders, its image read asynchronously into
            page-locked memory (copied while the next frame renders), one wait
            per framebuffer at the end."""
            for v, fb, o in zip(views, fbs, outs):
                ps.set_camera(v)
                ps.submit(dev, fb, v)
                mopcuda._check(L.mopcuda_read_color_resolved_async(d, fb, v.ssaa, C.c_void_p(o.p),
                                                                   o.a.nbytes), "read_async")
            for fb in fbs:
                mopcuda._check(L.mopcuda_readback_wait(d, fb, 20000), "readback_wait")
        plain_gpu_pass()
        g_plain = sum(plain_gpu_pass() for _ in range(2)) / 2
        plain_pass()
        t0 = time.perf_counter()
        for _ in range(3):
            plain_pass()
        wall_p = (time.perf_counter() - t0) / 3
        for fb in fbs:
            L.mopcuda_framebuffer_destroy(d, fb)
    finally:
        for o in outs:
            o.close()
        b.close()
    gmed = float(np.median(gms))
    return {"workload": f"{n_views} viewports (log-uniform 128^2..1920x1080, aspect 0.5-2, "
                        "ssaa 1|2, cameras r=15-40) over the 1,470,464-tri scene, one CUDA graph",
            "pixels": pixels, "samples": sum(v.samples for v in views),
            "batch_ms": round(wall_b * 1e3, 3), "batch_gpu_ms": round(gmed, 3),
            "batch_mpix_s": round(pixels / (wall_b * 1e6), 1),
            "pipelined_ms": round(wall_pipe * 1e3, 3),
            "pipelined_mpix_s": round(pixels / (wall_pipe * 1e6), 1),
            "plain_ms": round(wall_p * 1e3, 3), "plain_gpu_ms": round(g_plain, 3),
            "plain_mpix_s": round(pixels / (wall_p * 1e6), 1),
            "speedup_vs_plain": {"wall": round(wall_p / wall_b, 2),
                                 "wall_pipelined": round(wall_p / wall_pipe, 2),
                                 "device": round(g_plain / gmed, 2)},
            "launch_config": cfg, "default_launch_config": default_cfg,
            "autotune": {"start_ms": tuned.get("start_ms"), "best_ms": tuned.get("best_ms"),
                         "passes": tuned.get("passes"), "trials": len(tuned.get("trials", []))},
            "note": ("wall time per pass including every presented image read to host; the "
                     "plain arm records each frame while the previous renders and reads its "
                     "image asynchronously into page-locked memory; device = summed per-frame "
                     "device time over the batch's device time")}


CAP_SAMPLES = 24 << 20  # samples per server launch (about two 1080p SSAA-2 views)


def run_served(dev, rates=(2000.0, 4000.0, 6000.0), duration=2.0, n_scenes=32):
    """Served mix: resident scenes of log-normal size, Poisson render/pick
    requests; p50/p99 arrival-to-result latency and Mpix/s of the
    continuous-batching server (and with launches capped at CAP_SAMPLES
    samples) and of the plain per-viewport path on the same trace; IDs/depth
    of a 1% sample checked bit-exact against the request's own frame in a
    separate, untimed run of the same trace."""
    import mopcuda
    import scenes
    import serving
    counts = scenes.served_triangle_counts(n_scenes)
    scs = [scenes.served_scene(100 + i, c, tex_size=1024) for i, c in enumerate(counts)]
    ibl = scenes.procedural_ibl(scs[0].sun_dir)
    rss = [mopcuda.ResidentScene(dev, sc, ibl) for sc in scs]
    out = {"workload": f"{n_scenes} resident scenes ({sum(counts):,} tris, 50k-2M log-normal), "
                       "Poisson arrivals, 85% renders at 256^2/720p/1080p/1440p, 15% pick "
                       "batches of 1-64, 1% of a scene's instances moved per request",
           "server_config": {"max_views": 32, "max_inflight": 3, "hbm_budget_gib": 100},
           "plain_arm": "one frame per request through the per-viewport C ABI, image read "
                        "into page-locked memory",
           "textures": "4 x 1024^2 RGBA8 per scene, as in config 2",
           "capped_config": {"max_launch_samples": CAP_SAMPLES},
           "rates": []}
    keys = ("p50_ms", "p99_ms", "mpix_s")
    try:
        for rate in rates:
            warm = serving.make_trace(scs, rate, 0.5, seed=7 + int(rate))
            for r in warm:
                r.moves = []
            trace = serving.make_trace(scs, rate, duration, seed=int(rate))
            # timed runs keep no results for checking: copying a kept request's
            # sample-resolution IDs and depth into pageable memory stalls the
            # server's worker and would dominate the tail
            runs = {}
            for name, cap in (("server", 0), ("server_capped", CAP_SAMPLES)):
                serving.reset_models(rss, scs)
                r_ = serving.run_server(dev, rss, trace, hbm_budget=100 << 30, max_views=32,
                                        max_inflight=3, warmup=warm, max_launch_samples=cap)
                r_.pop("kept", None)
                st = r_.pop("stats")
                runs[name] = dict({k: round(r_[k], 3) for k in keys}, launches=st["launches"],
                                  reruns=st["reruns"],
                                  max_views_in_launch=st["max_views_in_launch"])
            # exactness: the same trace again, every 100th render's IDs and depth kept
            serving.reset_models(rss, scs)
            k_ = serving.run_server(dev, rss, trace, hbm_budget=100 << 30, max_views=32,
                                    max_inflight=3, keep_every=100, warmup=warm)
            chk = serving.check_kept(dev, rss, trace, k_.pop("kept"))
            serving.reset_models(rss, scs)
            p = serving.run_plain(dev, rss, trace, warmup=warm[:40])
            out["rates"].append({
                "req_per_s": rate, "requests": len(trace), **runs,
                "plain": {k: round(p[k], 3) for k in keys},
                "speedup_vs_plain": {
                    "mpix_s": round(runs["server"]["mpix_s"] / p["mpix_s"], 2),
                    "p99": round(p["p99_ms"] / runs["server"]["p99_ms"], 2)},
                "exact_check": dict(chk, against="each kept request's own plain frame (the "
                                    "plain path is pinned to the CPU oracle by the GPU parity "
                                    "tests; served requests are checked against the oracle "
                                    "in tests/test_gpu_server.py)")})
    finally:
        for rs in rss:
            rs.close()
    return out


def frame_bytes_of(sc):
    """Algorithmic bytes of one frame: every mesh's indices and vertices read
    once, 64 B of draw state per draw, colour + depth + ID per sample and the
    presented image when SSAA is on."""
    return (sum(4 * m.indices.size + 48 * m.vertices.shape[0] for m in sc.meshes)
            + 64 * len(sc.meshes) + 12 * sc.samples + (4 * sc.pixels if sc.ssaa > 1 else 0))


def run_frames_form(dev, name, steps=20, warm=3):
    """Device-timed frames of another workload (an L2-sized buffer rewritten
    between frames): frame ms, Mpix/s, Mtri/s, per-stage ms and the frame's
    algorithmic bytes against the HBM peak."""
    import numpy as np
    import torch
    import mopcuda
    import scenes
    if name == "transparent":
        import dataclasses
        sc = scenes.config2()
        for k in range(0, len(sc.meshes), 3):  # every third instance blended, the core's order
            sc.meshes[k] = dataclasses.replace(sc.meshes[k], opacity=0.35 + 0.1 * (k % 5),
                                               blend_mode=(1, 2, 3, 1)[k % 4])
        desc = ("config2 with every third of its 256 instances blended (alpha / additive / "
                "multiply, opacity 0.35-0.75): the transparent pass composited per sample in "
                "submission order")
    elif name == "config3":
        sc = scenes.config3()
        desc = ("config3: 1920x1080 ssaa1, 2,000,000 tris (0.1-8 px edges; 10% straddle the near "
                "plane, 5% outside, 20% coplanar pairs in separate meshes, 5% skinned tubes), "
                "1 dir + 1 point light")
    else:
        sc = scenes.config1()
        desc = "config1: 800x600 ssaa1, UV sphere 64x32 + ground plane, 1 directional light"
    ibl = scenes.procedural_ibl(sc.sun_dir) if sc.env else None
    r = mopcuda.SceneRenderer(dev, sc, ibl)
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    try:
        dev.set_stage_timing(True)
        for _ in range(warm):
            r.render()
        ms, stage = [], {k: 0.0 for k in mopcuda.Device.STAGES}
        for _ in range(steps):
            flush.add_(1.0)
            torch.cuda.synchronize()
            r.render()
            ms.append(r.gpu_ms)
            for k, v in dev.stage_times().items():
                stage[k] += v
        dev.set_stage_timing(False)
        fm = float(np.median(ms))
        peak, kind = read_peaks()
        b = frame_bytes_of(sc)
        return {"workload": desc, "steps": steps, "frame_ms": round(fm, 4),
                "mpix_s": round(sc.pixels / (fm * 1e3), 1),
                "mtri_s": round(sc.triangle_count / (fm * 1e3), 1),
                "triangles": sc.triangle_count, "samples": sc.samples,
                "stage_ms": {k: round(v / steps, 4) for k, v in stage.items()},
                "roofline": {"bound": "hbm", "kernel": "whole frame",
                             "algorithmic_bytes": b,
                             "achieved": round(b / (fm * 1e-3) / 1e9, 1), "peak": peak,
                             "unit": "GB/s", "frac": round(b / (fm * 1e-3) / 1e9 / peak, 4),
                             "peak_source": kind}}
    finally:
        r.close()


def run_shadowed(dev, steps=20, warm=3):
    """The config-2 frame with its directional light casting shadows: the
    shadow pass (1024^2 map, every opaque mesh a caster) runs before each
    frame and every directional light takes the 3x3 PCF factor."""
    import dataclasses
    import numpy as np
    import mopcuda
    import scenes
    sc, _ = workload("config2")
    k = next(i for i, l in enumerate(sc.lights) if l.type == scenes.LIGHT_DIRECTIONAL)
    sc.lights[k] = dataclasses.replace(sc.lights[k], cast_shadows=True)
    ibl = scenes.procedural_ibl(sc.sun_dir) if sc.env else None
    r = mopcuda.SceneRenderer(dev, sc, ibl)
    try:
        for _ in range(warm):
            r.render()
        frame, shadow, wall = [], [], []
        for _ in range(steps):
            t0 = time.perf_counter()
            r.render()
            wall.append((time.perf_counter() - t0) * 1e3)
            frame.append(r.gpu_ms)
            shadow.append(r.shadow_gpu_ms)
        ids = r.object_id()
        # back to back through the public API, as the e2e loop: each frame's
        # shadow pass and draws recorded while the previous frame runs, its
        # image read asynchronously into page-locked memory
        outs = [mopcuda.HostArray((sc.height, sc.width, 4), np.uint8) for _ in range(2)]
        try:
            for k in range(warm):
                r.submit()
                r.color_async(outs[k % 2].a)
            r.wait_readback()
            t0 = time.perf_counter()
            for k in range(steps):
                r.submit()
                r.color_async(outs[k % 2].a)
            r.wait_readback()
            piped = (time.perf_counter() - t0) * 1e3 / steps
        finally:
            for o in outs:
                o.close()
        fm, sm = float(np.median(frame)), float(np.median(shadow))
        return {"scene": "config2 with its directional light casting shadows",
                "casters": len(scenes.shadow_casters(sc)),
                "caster_triangles": int(sum(sc.meshes[i].indices.size // 3
                                            for i in scenes.shadow_casters(sc))),
                "shadow_map": scenes.SHADOW_MAP_SIZE, "steps": steps,
                "frame_ms": round(fm, 4), "shadow_pass_ms": round(sm, 4),
                "mpix_s": round(sc.pixels / ((fm + sm) * 1e3), 1),
                "wall_ms_per_frame": round(float(np.median(wall)), 4),
                "pipelined_ms_per_frame": round(piped, 4),
                "pipelined_mpix_s": round(sc.pixels / (piped * 1e3), 1),
                "covered_samples": int((ids != 0).sum())}
    finally:
        r.close()


def run_ibl(dev, steps=20, warm=3):
    """Environment admission: the config-2 procedural sky and its IBL maps
    (sky 512x256, irradiance 64x32, prefiltered 128x64x5, BRDF LUT 256^2)
    computed on the device; the reference core's own serial
    mop_viewport_set_environment for the same sky timed on the host beside
    it (oracle/_ref, in a subprocess)."""
    import numpy as np
    sc, _ = workload("config2")
    args = (sc.sun_dir, sc.turbidity, sc.ground_albedo, sc.env_rotation, sc.env_intensity)
    for _ in range(warm):
        dev.ibl_procedural_sky(*args)
    gpu, wall = [], []
    for _ in range(steps):
        t0 = time.perf_counter()
        dev.ibl_procedural_sky(*args)
        wall.append((time.perf_counter() - t0) * 1e3)
        gpu.append(dev.ibl_gpu_ms)
    out = {"scene": "config2 procedural sky (sun %s, turbidity %g)" % (tuple(sc.sun_dir),
                                                                      sc.turbidity),
           "steps": steps, "gpu_ms": round(float(np.median(gpu)), 4),
           "wall_ms": round(float(np.median(wall)), 4)}
    cmd = [sys.executable, str(ROOT / "oracle" / "time_reference.py"), "--config", "config2",
           "--environment", "--frames", "3"]
    try:
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
        t = json.loads(p.stdout.strip().splitlines()[-1])
        out["cpu_baseline"] = {"value": round(t["ms"], 3), "unit": "ms", "cores": t["threads"],
                               "kind": "reference",
                               "sample": f"{t['reps']} x mop_viewport_set_environment"}
    except Exception as e:  # report, do not fail the device measurement
        out["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    return out


def run_scene_load(dev, steps=5):
    """Scene admission from a .mop v2 file: the config-2 scene with 240 of
    its 256 instances (the format holds at most 256 sections: meshes, lights
    and the camera) written with quantized vertices, every mesh read
    straight into device buffers (stored bytes over PCIe, decoded on the
    device); the reference's own mop_scene_load + mop_scene_get_mesh host
    decode of the same file timed beside it (oracle/_ref, in a subprocess)."""
    import tempfile
    import numpy as np
    import scene_file
    import scenes
    sc = scenes.config2(instances=240)
    tmp = tempfile.mkdtemp()
    path = os.path.join(tmp, "config2_quantized.mop")
    scene_file.save(sc, path, True)
    raw_bytes = sum(48 * m.vertices.shape[0] + 4 * m.indices.size for m in sc.meshes)
    out = {"scene": "config2 (240 instances), quantized .mop v2",
           "triangles": int(sum(m.indices.size // 3 for m in sc.meshes)),
           "file_bytes": os.path.getsize(path),
           "decoded_bytes": raw_bytes, "meshes": len(sc.meshes), "steps": steps}
    for key, fn in (("device_load_ms", scene_file.upload_all),
                    ("device_load_per_mesh_ms", scene_file.upload)):
        wall = []
        for s in range(steps + 1):
            t0 = time.perf_counter()
            bufs = fn(dev, path)
            t1 = time.perf_counter()
            for b in bufs:
                dev.L.mopcuda_buffer_destroy(dev.h, b["vertices"])
                dev.L.mopcuda_buffer_destroy(dev.h, b["indices"])
            if s:  # the first pass warms the page cache and the staging buffers
                wall.append((t1 - t0) * 1e3)
        out[key] = round(float(np.median(wall)), 3)
    cmd = [sys.executable, str(ROOT / "oracle" / "time_reference.py"), "--scene-file", path,
           "--frames", "3"]
    try:
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
        t = json.loads(p.stdout.strip().splitlines()[-1])
        out["cpu_baseline"] = {"value": round(t["ms"], 3), "unit": "ms", "cores": t["threads"],
                               "kind": "reference",
                               "sample": f"{t['reps']} x mop_scene_load + every get_mesh"}
    except Exception as e:
        out["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    os.remove(path)
    os.rmdir(tmp)
    return out


def forms_subprocess(timeout_s=900):
    """The batched and served forms in a fresh process on the same GPU, so
    their device and host state starts clean."""
    try:
        p = subprocess.run([sys.executable, str(Path(__file__).resolve()), "--forms-only"],
                           capture_output=True, text=True, timeout=timeout_s)
        for ln in reversed(p.stdout.strip().splitlines()):
            if ln.startswith("{"):
                return json.loads(ln)
        return {"batched": {"error": (p.stderr or "no output")[-300:]}}
    except Exception as e:
        return {"batched": {"error": str(e)[:300]}}


def run_forms(which="all"):
    import mopcuda
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dev = mopcuda.Device(local)
    out = {}
    for key, fn in (("batched", run_batched), ("served", run_served),
                    ("shadowed", run_shadowed), ("ibl", run_ibl),
                    ("scene_load", run_scene_load),
                    ("config3", lambda d: run_frames_form(d, "config3")),
                    ("transparent", lambda d: run_frames_form(d, "transparent")),
                    ("config1", lambda d: run_frames_form(d, "config1"))):
        if which not in ("all", key):
            continue
        try:
            out[key] = fn(dev)
        except Exception as e:  # report, do not lose the other form
            out[key] = {"error": str(e)[:300]}
    dev.close()
    emit(out)
    return 0


def main():
    args = parse()
    if args.forms_only:
        return run_forms(args.form)
    if args.impl == "reference":
        return run_reference(args)
    return run_cuda(args)


if __name__ == "__main__":
    sys.exit(main())
