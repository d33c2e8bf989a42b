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
    return ap.parse_args()


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


def dist_setup(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def cpu_reference_time(config, budget_s=45.0, warm=1, frames=3):
    """The reference CPU backend (oracle/_ref, built from the reference
    sources) timed on the host cores, each attempt in a subprocess under a
    timeout.  The reference sizes its tile pool from the online CPU count and
    stalls when that oversubscribes the host, so the pool is tried with half
    the usable cores, then the reference's serial path; the faster completed
    attempt is reported with the thread count it used."""
    ncpu = len(os.sched_getaffinity(0))
    attempts = [max(1, ncpu // 2 - 1), 0]
    best = None
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
        if best is None or t["ms"] < best["ms"]:
            best = t
    if best is None:
        raise RuntimeError("reference CPU backend did not complete a frame in time")
    return {"ms": best["ms"], "frames": best["frames"], "cores": best["threads"],
            "kind": "reference", "mode": best["mode"]}


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
    t = cpu_reference_time(args.config, budget_s=90.0, warm=min(args.warmup, 1),
                           frames=max(1, args.steps))
    mpix = sc.pixels / (t["ms"] * 1e3)
    line = {"impl": "reference", "metric": "Mpix/s", "value": round(mpix, 4), "unit": "Mpix/s",
            "n_gpus": args.gpus, "steps": t["frames"], "warmup": min(args.warmup, 1),
            "ms_per_step": round(t["ms"], 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
            "config": {"workload": desc, "backend": f"reference CPU backend ({t['mode']})"},
            "mtri_per_s": round(sc.triangle_count / (t["ms"] * 1e3), 5),
            "cpu_baseline": {"value": round(mpix, 4), "unit": "Mpix/s", "cores": t["cores"],
                             "kind": t["kind"],
                             "sample": f"{t['frames']} full frame(s) ({t['mode']}), median wall "
                                       "time of mop_viewport_render + mop_viewport_read_color"},
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

    # ---- device-timed frames ----
    dev.set_stage_timing(True)
    for _ in range(warm):
        r.render()
    ids = r.object_id()
    covered = int((ids != 0).sum())
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    frame_ms, stage = [], {k: 0.0 for k in mopcuda.Device.STAGES}
    l0 = dev.launches
    for _ in range(steps):
        flush.add_(1.0)  # rewrite > L2 (126 MB) between frames
        torch.cuda.synchronize()
        r.render()
        frame_ms.append(r.gpu_ms)
        for k, v in dev.stage_times().items():
            stage[k] += v
    launches = dev.launches - l0
    barrier()
    clocks = sampler.stop()
    total_ms, value, mtri = aggregate(sum(frame_ms), steps, world, sc.pixels,
                                      sc.triangle_count, dist, "cuda")

    # ---- end to end through the C ABI with host buffers ----
    dev.set_stage_timing(False)
    out = torch.empty((sc.height, sc.width, 4), dtype=torch.uint8, pin_memory=True)
    out_np = out.numpy()
    for _ in range(warm):
        r.submit()
        r.color(out_np)
    barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        r.submit()
        r.color(out_np)
    t1 = time.perf_counter()
    barrier()
    e2e_ms = max_over_ranks((t1 - t0) * 1e3, dist, "cuda")
    e2e = world * steps * sc.pixels / (e2e_ms * 1e3)
    h2d, d2h = dev.frame_io_bytes()
    d2h += out_np.nbytes

    # ---- roofline of the dominant kernel (tile visibility + shading) ----
    hbm_peak, peak_kind = read_peaks()
    tile_ms = (stage["resolve"] + stage["shade"]) / steps
    tile_bytes = 12 * sc.samples  # colour RGBA8 + depth f32 + id u32 written per sample
    achieved = tile_bytes / (tile_ms * 1e-3) / 1e9
    fp32_peak = dev.fp32_peak_gops()
    L = sum(1 for l in sc.lights if l.active)
    ops_per_sample = 80 + 120 * L + (150 if sc.env else 0)
    alu_achieved = covered * ops_per_sample / (tile_ms * 1e-3) / 1e9
    frame_bytes = (sum(4 * m.indices.size + 48 * m.vertices.shape[0] for m in sc.meshes)
                   + 64 * len(sc.meshes) + 12 * sc.samples + (4 * sc.pixels if sc.ssaa > 1 else 0))

    line = {"metric": "Mpix/s", "value": round(value, 3), "unit": "Mpix/s", "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": round(total_ms / steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene generator, procedural IBL maps)",
            "config": {"workload": desc, "parallelism": f"replicas x{world}",
                       "l2": f"{args.flush_mb} MiB buffer rewritten between timed frames",
                       "samples": sc.samples, "pixels": sc.pixels,
                       "triangles": sc.triangle_count},
            "mtri_per_s": round(mtri, 3),
            "stage_ms": {k: round(v / steps, 4) for k, v in stage.items()},
            "frame_algorithmic_bytes": frame_bytes,
            "roofline": {"bound": "hbm", "kernel": "k_resolve + k_shade (deferred shading + ACES)",
                         "achieved": round(achieved, 1), "peak": hbm_peak,
                         "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
                         "peak_source": peak_kind, "traffic": None,
                         "alu": {"achieved": round(alu_achieved, 1), "peak": round(fp32_peak, 1),
                                 "unit": "Gop/s (fp32 add/mul, no FMA)",
                                 "frac": round(alu_achieved / fp32_peak, 4) if fp32_peak else None,
                                 "ops_per_covered_sample": ops_per_sample,
                                 "covered_samples": covered}},
            "e2e": {"value": round(e2e, 3), "unit": "Mpix/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": round(e2e_ms / steps, 4)},
            "gpu_launches": launches,
            "clocks": clocks}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            t = cpu_reference_time(args.config)
            line["cpu_baseline"] = {
                "value": round(sc.pixels / (t["ms"] * 1e3), 4), "unit": "Mpix/s",
                "cores": t["cores"], "kind": t["kind"],
                "sample": f"{t['frames']} full frame(s) of the same scene ({t['mode']}, "
                          "median of mop_viewport_render + read_color)"}
        except Exception as e:  # report, do not fail the GPU measurement
            line["cpu_baseline"] = {"value": None, "unit": "Mpix/s", "error": str(e)[:200]}
    r.close()
    dev.close()
    if rank == 0:
        emit(line)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_cuda(args)


if __name__ == "__main__":
    sys.exit(main())
