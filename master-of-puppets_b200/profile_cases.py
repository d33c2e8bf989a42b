"""Fixed workloads for a kernel profiler: each case builds one scene, renders
`--frames` frames (or batch launches) through the public API and exits, so a
profiler run (`ncu -k <kernel> -s <skip> -c <count> ...`) captures a known
launch of a known kernel with nothing else on the device.

    python master-of-puppets_b200/profile_cases.py frame --frames 3

cases
  frame        the 1920x1080 SSAA-2 frame of 1,470,464 triangles, 7 lights,
               IBL (k_vertex .. k_post<2>)
  transparent  the same frame with every third instance blended
               (k_ocount, k_oscan, k_oraster, k_ofold)
  shadow       the same frame with the directional light casting shadows
               (k_shadow_tri, k_shadow_scan, k_shadow_large, 1024^2 map)
  batch        16 viewports of the same scene in one batched launch
               (k_batch_prepare, k_b_items, k_b_shade, k_b_post)
  small        the 800x600 sphere-and-plane frame
"""
import argparse
import dataclasses
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import mopcuda  # noqa: E402
import scenes  # noqa: E402


def _frame_scene(case):
    if case == "small":
        return scenes.config1()
    sc = scenes.config2()
    if case == "transparent":
        for k in range(0, len(sc.meshes), 3):
            sc.meshes[k] = dataclasses.replace(sc.meshes[k], opacity=0.35 + 0.1 * (k % 5),
                                               blend_mode=(1, 2, 3, 1)[k % 4])
    elif case == "shadow":
        k = next(i for i, l in enumerate(sc.lights) if l.type == scenes.LIGHT_DIRECTIONAL)
        sc.lights[k] = dataclasses.replace(sc.lights[k], cast_shadows=True)
    return sc


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["frame", "transparent", "shadow", "batch", "small"])
    ap.add_argument("--frames", type=int, default=3)
    ap.add_argument("--views", type=int, default=16)
    a = ap.parse_args(argv)
    dev = mopcuda.Device(0)
    try:
        if a.case == "batch":
            sc = scenes.config2()
            ibl = scenes.procedural_ibl(sc.sun_dir)
            r = mopcuda.BatchRenderer(dev, sc, scenes.batch_views(sc, n=a.views, seed=4), ibl)
        else:
            sc = _frame_scene(a.case)
            ibl = scenes.procedural_ibl(sc.sun_dir) if sc.env else None
            r = mopcuda.SceneRenderer(dev, sc, ibl)
        try:
            ms = []
            for _ in range(a.frames):
                r.render()
                ms.append(r.gpu_ms)
            print(f"{a.case}: {a.frames} launches, device ms {', '.join(f'{m:.4f}' for m in ms)}")
        finally:
            r.close()
    finally:
        dev.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
