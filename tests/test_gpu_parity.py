"""CUDA frame path vs the oracle (plain-C restatement of the reference CPU
backend) on seeded scenes, through the C ABI of libmopcuda.so.

IDs and depth must match bit for bit; colour within the contract tolerance
(tests/parity.py).  Scenes cover: multi-light smooth GGX (directional,
point, spot, ranged, inactive lights), textures, SSAA 2, IBL, flat shading
(lit and unlit), near-plane clipping (the config-1 ground plane passes
behind the camera), coplanar draw-order ties, the clipping/depth stress scene
(near-plane straddlers, coplanar pairs, host-skinned meshes), blended meshes
(alpha, additive, multiply) in the core's transparent-pass order, and picks.
"""
import dataclasses

import numpy as np
import pytest

import cpu_oracle
import mopcuda
import refdrive
import scenes
from parity import assert_frame_parity

pytestmark = pytest.mark.gpu


def _ibl_for(scene):
    if not scene.env:
        return None
    r = refdrive.Reference(scene)
    maps = r.env_maps()
    r.close()
    return maps


def _render_cuda(dev, scene, ibl):
    r = mopcuda.SceneRenderer(dev, scene, ibl)
    try:
        r.render()
        return {"object_id": r.object_id(), "depth": r.depth(), "color_full": r.color_full(),
                "color": r.color(), "renderer": r}
    finally:
        pass


CASES = {
    "config1": lambda: scenes.config1(),
    "small_mixed_a": lambda: scenes.small_scene(seed=0),
    "small_mixed_b": lambda: scenes.small_scene(seed=1, width=203, height=117),
    "small_ssaa2": lambda: scenes.small_scene(seed=5, ssaa=2),
    "small_ssaa3": lambda: scenes.small_scene(seed=6, width=90, height=70, ssaa=3),
    "small_ibl": lambda: scenes.small_scene(seed=9, env=1),
    "small_flat_lit": lambda: dataclasses.replace(scenes.small_scene(seed=6), smooth=False),
    "small_flat_unlit": lambda: dataclasses.replace(scenes.small_scene(seed=8, lights="none"),
                                                    smooth=False),
    "coplanar_ties": lambda: scenes.coplanar_scene(),
    "config2_reduced": lambda: scenes.config2(width=320, height=180, ssaa=2, instances=24,
                                              tex_size=64),
    # clipping / depth stress: near-plane straddlers, out-of-frustum triangles, coplanar pairs
    # in separate meshes, host-skinned tubes, 0.1-8 px triangles
    "config3_reduced": lambda: scenes.config3(n_tris=80_000, width=480, height=270),
    "config3_medium": lambda: scenes.config3(seed=4, n_tris=400_000, width=960, height=540),
    # blended meshes (alpha / additive / multiply), composited in submission order
    "transparent": lambda: scenes.transparent_scene(seed=21),
    "transparent_ssaa2_ibl": lambda: scenes.transparent_scene(seed=22, ssaa=2, env=1),
    "transparent_config2": lambda: _transparent_config2(),
}


def _transparent_config2():
    sc = scenes.config2(width=320, height=180, ssaa=2, instances=32, tex_size=64)
    for k in range(0, len(sc.meshes), 3):  # every third instance blended
        sc.meshes[k] = dataclasses.replace(sc.meshes[k], opacity=0.35 + 0.1 * (k % 5),
                                           blend_mode=(1, 2, 3, 1)[k % 4])
    return sc


@pytest.mark.parametrize("name", list(CASES))
def test_frame_parity(cuda_device, name):
    sc = CASES[name]()
    ibl = _ibl_for(sc)
    ref = cpu_oracle.render(sc, ibl)
    got = _render_cuda(cuda_device, sc, ibl)
    try:
        assert_frame_parity(got, ref, name)
        xy = scenes.pick_points(sc, 1000)
        i1, d1, h1 = got["renderer"].pick(xy)
        i2, d2, h2 = cpu_oracle.pick(sc, ref, xy)
        assert (i1 == i2).all() and (h1 == h2).all()
        assert (d1.view(np.uint32) == d2.view(np.uint32)).all()
    finally:
        got["renderer"].close()


def test_repeat_frames_identical(cuda_device):
    """Deterministic replay: two frames of one scene are byte-identical
    (reference tests/test_torture_picking.c:432-456 replays with bit-equal
    depth)."""
    sc = scenes.small_scene(seed=2)
    r = mopcuda.SceneRenderer(cuda_device, sc)
    try:
        a = (r.render().color_full(), r.depth(), r.object_id())
        b = (r.render().color_full(), r.depth(), r.object_id())
        for x, y in zip(a, b):
            assert x.tobytes() == y.tobytes()
    finally:
        r.close()
