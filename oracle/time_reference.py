"""Time the reference CPU backend (oracle/_ref/libmopref.so) on a workload.

Run as a subprocess by bench.py's CPU-baseline leg (so a stalled reference
thread pool can be killed by a timeout):

    python oracle/time_reference.py --config config2 --workers 7 --warm 1 --frames 2

--workers 0 selects the reference's serial path (tile pool removed);
--workers N replaces the tile pool with N worker threads (+ the caller).
Prints one JSON object: median ms of mop_viewport_render + read_color
(--environment: of mop_viewport_set_environment with the workload's sky).
"""
import argparse
import json
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent / "master-of-puppets_b200"))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="config2")
    ap.add_argument("--workers", type=int, default=0)
    ap.add_argument("--warm", type=int, default=1)
    ap.add_argument("--frames", type=int, default=2)
    ap.add_argument("--budget-s", type=float, default=60.0)
    ap.add_argument("--scene-file", default=None,
                    help="time mop_scene_load + mop_scene_get_mesh of every mesh of this "
                         ".mop v2 file instead of frames")
    ap.add_argument("--environment", action="store_true",
                    help="time mop_viewport_set_environment (procedural sky + IBL "
                         "precompute) instead of frames")
    a = ap.parse_args()
    import dataclasses
    import refdrive
    import scenes
    sc = scenes.config1() if a.config == "config1" else scenes.config2()
    if a.scene_file:
        ms = refdrive.time_scene_file(a.scene_file, max(1, a.frames))
        print(json.dumps({"ms": ms, "reps": max(1, a.frames), "threads": 1,
                          "mode": "serial (the loader runs on the caller)"}))
        return
    if a.environment:  # the environment only: no meshes, a small viewport
        sc = dataclasses.replace(sc, width=64, height=36, ssaa=1, meshes=[], textures=[])
        r = refdrive.Reference(sc, serial=True)
        print(json.dumps({"ms": r.time_environment(max(1, a.frames)), "reps": max(1, a.frames),
                          "threads": 1, "mode": "serial (the core runs it on the caller)"}))
        r.close()
        return
    r = refdrive.Reference(sc, serial=(a.workers == 0), workers=max(0, a.workers))
    t0 = time.perf_counter()
    first = r.time_frames(a.warm, 1)
    spent = time.perf_counter() - t0
    per = max(first * 1e-3, 1e-3)
    more = max(0, min(a.frames - 1, int((a.budget_s - spent) / per)))
    ms = r.time_frames(0, more) if more > 0 else first
    print(json.dumps({"ms": ms, "frames": 1 + more, "threads": r.threads,
                      "mode": "serial" if a.workers == 0 else f"tile pool x{a.workers}"}))
    r.close()


if __name__ == "__main__":
    main()
