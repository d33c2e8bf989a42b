"""The oracle (plain-C restatement, oracle/mop_oracle.c) pinned against the
reference: bit-exact on colour, depth, object IDs, camera matrices and picks.

* against committed golden fixtures made by the reference library itself
  (tests/golden/make_golden.py), always;
* against the reference library live (oracle/_ref/libmopref.so) on more and
  larger seeded scenes, when that library has been built.
"""
import dataclasses
import subprocess
from pathlib import Path

import numpy as np
import pytest

import cpu_oracle
import refdrive
import scenes

GOLDEN_DIR = Path(__file__).resolve().parent / "golden"


def _golden_cases():
    import sys
    sys.path.insert(0, str(GOLDEN_DIR))
    import make_golden
    return make_golden.GOLDEN


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint8)


def _assert_same(got, ref, label):
    for key in ("object_id", "depth", "color_full", "color"):
        bad = int((_bits(got[key]) != _bits(ref[key])).sum())
        assert bad == 0, f"{label}: {key} differs in {bad} bytes"


@pytest.mark.parametrize("name", list(_golden_cases()))
def test_oracle_matches_golden(name):
    sc = _golden_cases()[name]()
    g = np.load(GOLDEN_DIR / f"{name}.npz")
    ibl = None
    if sc.env:
        m = np.load(GOLDEN_DIR / f"{name}_maps.npz")
        ibl = {k: (m[k] if m[k].ndim else m[k].item()) for k in m.files}
    out = cpu_oracle.render(sc, ibl)
    _assert_same(out, g, name)
    for k in ("view", "proj", "eye"):
        assert (_bits(out[k]) == _bits(g[k])).all(), f"{name}: {k}"
    ids, dep, hits = cpu_oracle.pick(sc, out, g["pick_xy"])
    assert (ids == g["pick_ids"]).all() and (hits == g["pick_hits"]).all()
    assert (_bits(dep) == _bits(g["pick_depth"])).all()


LIVE = {
    "config1": lambda: scenes.config1(),
    "mixed_a": lambda: scenes.small_scene(seed=11),
    "mixed_b": lambda: scenes.small_scene(seed=12, width=211, height=97),
    "ssaa3": lambda: scenes.small_scene(seed=13, width=80, height=60, ssaa=3),
    "ibl": lambda: scenes.small_scene(seed=14, env=1),
    "flat": lambda: dataclasses.replace(scenes.small_scene(seed=15), smooth=False),
    "coplanar": lambda: scenes.coplanar_scene(seed=16),
    "config2_reduced": lambda: scenes.config2(width=256, height=144, ssaa=2, instances=16,
                                              tex_size=32),
    # blended meshes (alpha / additive / multiply) in the core's transparent pass order
    "transparent": lambda: scenes.transparent_scene(seed=17),
    "transparent_ssaa2_ibl": lambda: scenes.transparent_scene(seed=18, ssaa=2, env=1),
    # 64 stacked blended quads: more fragments on a sample than the device sorts in registers
    "transparent_deep": lambda: scenes.deep_transparent_scene(seed=19),
    # MOP_RENDER_WIREFRAME: anti-aliased lines in the flat colour, lit and unlit, SSAA 2
    "wireframe": lambda: scenes.wireframe_scene(seed=111),
    "wireframe_unlit_ssaa2": lambda: scenes.wireframe_scene(seed=112, ssaa=2, lights="none"),
    "wireframe_transparent": lambda: dataclasses.replace(scenes.transparent_scene(seed=113),
                                                         wireframe=True),
    "wireframe_instanced": lambda: dataclasses.replace(
        scenes.instanced_scene(seed=114), wireframe=True),
    "wireframe_chrome": lambda: dataclasses.replace(scenes.chrome_scene(seed=115),
                                                    wireframe=True),
    "config3_small": lambda: scenes.config3(seed=19, n_tris=30_000, width=320, height=180),
    # pass_shadow + PCF: smooth, flat, SSAA 2 with IBL, with the transparent pass
    "shadow": lambda: scenes.shadow_scene(seed=31),
    "shadow_flat": lambda: dataclasses.replace(scenes.shadow_scene(seed=32), smooth=False),
    "shadow_ssaa2_ibl": lambda: scenes.shadow_scene(seed=33, ssaa=2, env=1),
    "shadow_transparent": lambda: scenes.shadow_scene(seed=34, transparent=True),
    "transparent_flat": lambda: dataclasses.replace(scenes.transparent_scene(seed=36),
                                                    smooth=False),
    # no lights: legacy smooth path (silhouette edge AA) with blended meshes
    "unlit_transparent": lambda: dataclasses.replace(scenes.transparent_scene(seed=35),
                                                     lights=[]),
    # MOP_POST_FOG (mop_viewport_set_fog): colour blended towards the fog colour by each
    # sample's depth value, before tonemap / gamma / vignette; a zero range leaves it off
    "fog": lambda: dataclasses.replace(
        scenes.small_scene(seed=41), post_effects=scenes.DEFAULT_POST | scenes.POST_FOG,
        fog=((0.6, 0.65, 0.7, 1.0), 0.85, 0.99)),
    "fog_all_effects_ssaa2": lambda: dataclasses.replace(
        scenes.small_scene(seed=42, ssaa=2),
        post_effects=(scenes.POST_GAMMA | scenes.POST_TONEMAP | scenes.POST_VIGNETTE
                      | scenes.POST_FOG | scenes.POST_FXAA),
        fog=((0.2, 0.3, 0.5, 1.0), 0.9, 0.995)),
    "fog_zero_range": lambda: dataclasses.replace(
        scenes.small_scene(seed=43), post_effects=scenes.DEFAULT_POST | scenes.POST_FOG,
        fog=((1.0, 0.0, 0.0, 1.0), 0.95, 0.95)),
    # mop_viewport_add_instanced_mesh: pass_instanced after the transparent pass, one draw
    # per instance with the depth write off (depth saved and restored around each)
    "instanced": lambda: scenes.instanced_scene(seed=71),
    "instanced_zero_id_ssaa2": lambda: scenes.instanced_scene(seed=72, ssaa=2, zero_id=True),
    "instanced_transparent": lambda: scenes.instanced_scene(seed=73, transparent=True),
    "instanced_flat": lambda: dataclasses.replace(scenes.instanced_scene(seed=74), smooth=False),
    "instanced_unlit": lambda: dataclasses.replace(scenes.instanced_scene(seed=75), lights=[]),
    # meshes with editor-chrome IDs: depth test and culling off, legacy unlit path
    "chrome": lambda: scenes.chrome_scene(seed=81),
    "chrome_ssaa2_flat": lambda: dataclasses.replace(scenes.chrome_scene(seed=82, ssaa=2),
                                                     smooth=False),
    # BC1 / BC3 / BC5 textures made through mop_tex_create (texture_create_ex)
    "bc_textures": lambda: scenes.bc_scene(seed=91),
    # mop_viewport_set_environment_background: the procedural sky behind the scene
    "env_background": lambda: dataclasses.replace(scenes.small_scene(seed=92, env=1),
                                                  env_background=True),
    "env_background_ssaa2_transparent": lambda: dataclasses.replace(
        scenes.transparent_scene(seed=93, ssaa=2, env=1), env_background=True,
        env_rotation=0.7, env_intensity=1.3),
}


@pytest.mark.skipif(not refdrive.available(), reason="reference library not built")
@pytest.mark.parametrize("name", list(LIVE))
def test_oracle_matches_reference_live(name):
    _check_live(LIVE[name](), name)


# seeded random frames (scenes.fuzz_scene): random geometry incl. degenerate, sliver, huge and
# near-plane triangles, every light type, blend modes, flat / smooth / wireframe, chrome IDs,
# post effects; the same seeds drive the device sweep in tests/test_gpu_fuzz.py
FUZZ_SEEDS = list(range(96))


@pytest.mark.skipif(not refdrive.available(), reason="reference library not built")
@pytest.mark.parametrize("seed", FUZZ_SEEDS)
def test_oracle_matches_reference_fuzz(seed):
    _check_live(scenes.fuzz_scene(seed), f"fuzz{seed}")


def _check_live(sc, name):
    r = refdrive.Reference(sc, serial=True)
    try:
        ref = r.render()
        ibl = r.env_maps() if sc.env else None
        if sc.env_background:
            ibl["env"] = r.env_hdr()
        out = cpu_oracle.render(sc, ibl)
        _assert_same(out, ref, name)
        for k in ("view", "proj", "eye"):
            assert (_bits(out[k]) == _bits(ref[k])).all(), f"{name}: {k}"
        xy = scenes.pick_points(sc, 500)
        a = r.pick(xy)
        b = cpu_oracle.pick(sc, out, xy)
        for x, y in zip(a, b):
            assert (_bits(x) == _bits(y)).all()
    finally:
        r.close()


def test_gamma_lut_matches_formula():
    """The 256-entry sRGB byte map equals the per-pixel post-process."""
    lut = cpu_oracle.gamma_lut()
    assert lut[0] == 0 and lut[255] == 255
    assert (np.diff(lut.astype(int)) >= 0).all()


@pytest.mark.skipif(not refdrive.available(), reason="reference library not built")
def test_deform_oracle_matches_reference():
    """Skinning and morph restated in the oracle equal the reference core's
    own mop_skin_apply / mop_morph_apply, read back from its CPU backend."""
    from parity import deform_case
    lay = (44, 0, 12, 24, 28)
    for seed, vc in ((1, 500), (2, 2048)):
        raw, bones = deform_case(seed, vc)
        got = cpu_oracle.skin(lay, raw, vc, bones)
        ref = refdrive.deform_probe(raw, vc, bones=bones)
        assert (got == ref).all(), f"skin seed {seed}"
        rng = np.random.default_rng(seed)
        targets = rng.normal(size=(4, vc, 3)).astype(np.float32)
        weights = np.array([0.5, 0.0, -0.25, 1.5], np.float32)
        got = cpu_oracle.morph(lay, raw, vc, targets, weights)
        ref = refdrive.deform_probe(raw, vc, targets=targets, weights=weights)
        assert (got == ref).all(), f"morph seed {seed}"
        # both set: the core morphs, then skins from the bind pose again
        ref = refdrive.deform_probe(raw, vc, bones=bones, targets=targets, weights=weights)
        assert (cpu_oracle.skin(lay, raw, vc, bones) == ref).all(), f"skin+morph seed {seed}"


REFTESTS = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "tests"


@pytest.mark.parametrize("suite", ["test_torture_picking", "test_torture_depth",
                                   "test_torture_golden", "test_torture_geometry",
                                   "test_torture_lighting", "test_torture_hierarchy",
                                   "test_torture_camera", "test_exposure", "test_skinning",
                                   "test_morph_targets", "test_procedural_sky",
                                   "test_ortho_camera"])
def test_reference_suite_on_its_cpu_backend(suite):
    """The reference's own test program, built by oracle/Makefile `reftests`
    from the unmodified sources, passes on the reference's CPU backend: the
    baseline for the same programs linked to the CUDA backend
    (test_gpu_dropin.py)."""
    exe = REFTESTS / f"{suite}_cpu"
    if not exe.exists():
        pytest.skip("reference test programs not built (reference tree absent at build time)")
    p = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0 and "FAIL" not in p.stdout, p.stdout[-3000:]


@pytest.mark.skipif(not refdrive.available(), reason="reference library not built")
@pytest.mark.parametrize("fmt,w,h", [(scenes.TEX_BC1, 8, 8), (scenes.TEX_BC1, 13, 7),
                                     (scenes.TEX_BC3, 64, 36), (scenes.TEX_BC3, 5, 5),
                                     (scenes.TEX_BC5, 33, 70), (scenes.TEX_BC5, 1, 1)])
def test_bc_decode_matches_reference(fmt, w, h):
    """The oracle's block decode equals the CPU backend's texture_create_ex
    (read back through texture_read_rgba8), texel for texel, including the
    clamped last block row and column of odd sizes."""
    t = scenes.bc_texture(np.random.default_rng(100 * fmt + w), fmt, w, h)
    want = refdrive.bc_decode(t)
    assert want is not None
    assert (cpu_oracle.bc_decode(t) == want).all()


@pytest.mark.skipif(not refdrive.available(), reason="reference library not built")
def test_bc7_refused_by_reference():
    t = scenes.bc_texture(np.random.default_rng(7), scenes.TEX_BC7, 8, 8)
    assert refdrive.bc_decode(t) is None
