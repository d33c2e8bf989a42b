"""Generate the golden fixtures in this directory from the reference itself.

Renders small seeded scenes with the reference library's CPU backend (serial
path; oracle/_ref/libmopref.so, compiled from the reference sources by
oracle/Makefile) and stores, per scene, the presented colour, sample-res
colour, depth and object-ID buffers and 200 pick results.  The oracle's
tests compare against these files, so the oracle stays pinned even where
the reference library is not available.

    python tests/golden/make_golden.py [name ...]
    python tests/golden/make_golden.py scene_files
"""
import dataclasses
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "master-of-puppets_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

import refdrive  # noqa: E402
import scenes  # noqa: E402

GOLDEN = {
    "small_mixed": lambda: scenes.small_scene(seed=0, width=96, height=72),
    "small_ssaa2": lambda: scenes.small_scene(seed=5, width=64, height=48, ssaa=2),
    "small_ibl": lambda: scenes.small_scene(seed=9, width=96, height=72, env=1),
    "small_flat": lambda: dataclasses.replace(scenes.small_scene(seed=6, width=96, height=72),
                                              smooth=False),
    "small_unlit_flat": lambda: dataclasses.replace(
        scenes.small_scene(seed=8, width=96, height=72, lights="none"), smooth=False),
    "small_unlit_smooth": lambda: scenes.small_scene(seed=4, width=96, height=72, lights="none"),
    "coplanar": lambda: scenes.coplanar_scene(width=96, height=72),
    # the core's transparent pass: alpha / additive / multiply meshes back to front
    "transparent": lambda: scenes.transparent_scene(seed=41, width=96, height=72),
    # a directional light casting shadows: pass_shadow + 3x3 PCF on the CPU backend
    "shadow": lambda: scenes.shadow_scene(seed=42, width=96, height=72),
}


# .mop v2 scene files written by the reference's mop_scene_save, with the
# reference's mop_scene_get_mesh decode of every mesh
SCENE_FILES = {
    "scene_small_quant": (lambda: scenes.small_scene(seed=3), True),
    "scene_coplanar_raw": (lambda: scenes.coplanar_scene(), False),
}


def make_scene_files():
    for name, (make, quant) in SCENE_FILES.items():
        sc = make()
        path = HERE / f"{name}.mop"
        r = refdrive.Reference(sc, serial=True)
        r.save_scene(path, quant)
        r.close()
        n = sum(1 for m in sc.meshes if m.object_id != 0)
        arrays = {}
        for k in range(n):
            v, i, bb = refdrive.scene_file_mesh(path, k)
            arrays[f"v{k}"], arrays[f"i{k}"], arrays[f"b{k}"] = v, i, bb
        np.savez_compressed(HERE / f"{name}_decoded.npz", **arrays)
        print(name, path.stat().st_size, "bytes")


def main(names=None):
    if names and "scene_files" in names:
        return make_scene_files()
    for name, make in GOLDEN.items():
        if names and name not in names:
            continue
        sc = make()
        r = refdrive.Reference(sc, serial=True)
        out = r.render()
        xy = scenes.pick_points(sc, 200, seed=5)
        ids, dep, hits = r.pick(xy)
        if sc.env:
            maps = r.env_maps()
            np.savez_compressed(HERE / f"{name}_maps.npz",
                                **{k: np.asarray(v) for k, v in maps.items()})
        r.close()
        np.savez_compressed(HERE / f"{name}.npz", color=out["color"], color_full=out["color_full"],
                            depth=out["depth"], object_id=out["object_id"], view=out["view"],
                            proj=out["proj"], eye=out["eye"], pick_xy=xy, pick_ids=ids,
                            pick_depth=dep, pick_hits=hits)
        print(name, (HERE / f"{name}.npz").stat().st_size, "bytes")


if __name__ == "__main__":
    main(sys.argv[1:])
