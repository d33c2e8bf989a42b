"""Seeded random frames (scenes.fuzz_scene) on the device against the oracle.

The oracle is pinned to the reference on the same seeds (tests/test_oracle.py
test_oracle_matches_reference_fuzz).  Each frame mixes random geometry
(degenerate, sliver, huge, near-plane and off-screen triangles), every light
type, blend modes, flat / smooth / wireframe draws, editor-chrome IDs and
post effects.  IDs and depth must match bit for bit; colour too, except
where vignette takes the sRGB value itself (powf), where the contract's
tolerance applies.
"""
import numpy as np
import pytest

import cpu_oracle
import mopcuda
import scenes
from parity import assert_frame_parity, color_stats

pytestmark = pytest.mark.gpu

SEEDS = list(range(160))


@pytest.mark.parametrize("seed", SEEDS)
def test_fuzz_frame_matches_oracle(cuda_device, seed):
    sc = scenes.fuzz_scene(seed)
    ref = cpu_oracle.render(sc, None)
    r = mopcuda.SceneRenderer(cuda_device, sc)
    try:
        r.render()
        got = {"object_id": r.object_id(), "depth": r.depth(), "color_full": r.color_full(),
               "color": r.color()}
        assert_frame_parity(got, ref, f"fuzz{seed}")
        if not sc.post_effects & scenes.POST_VIGNETTE:
            for key in ("color_full", "color"):
                s = color_stats(got[key], ref[key])
                assert s["exact"] == 1.0, (seed, key, s)
        xy = scenes.pick_points(sc, 200, seed=seed)
        i1, d1, h1 = r.pick(xy)
        i2, d2, h2 = cpu_oracle.pick(sc, ref, xy)
        assert (i1 == i2).all() and (h1 == h2).all()
        assert (np.asarray(d1).view(np.uint32) == np.asarray(d2).view(np.uint32)).all()
    finally:
        r.close()
