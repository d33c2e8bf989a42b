"""Drop-in check through the reference's own public API.

The unmodified reference viewport core (its compiled objects, with only the
backend-resolution function swapped so value 4 means the CUDA backend — the
integration patch does the same with a MOP_BACKEND_CUDA enumerator)
renders each scene twice in one process: once on its CPU backend, once on
mop_rhi_backend_cuda().  mop_viewport_read_color (SSAA box in the core),
the object-ID / depth readbacks and mop_viewport_pick must agree: IDs and
depth bit-exact, colour within the contract tolerance.

The unmodified core hands IBL state only to its CPU path (reference
viewport.c:2692-2706); on the CUDA side the harness's pre-scene hook passes
the viewport's maps to mopcuda_set_ibl, as the integration patch's IBL row
does (along with post effects and fog).
Twelve of the reference's own test programs also run unmodified on the
CUDA backend (a link-time wrapper of mop_viewport_create selects it).
The shadow scenes run the core's own pass_shadow on the CPU side; on the
CUDA side the harness registers the integration patch's shadow pass as a
MOP_STAGE_PRE_SCENE hook (the core runs pass_shadow for its CPU backend
only, viewport.c:3224).
"""
import dataclasses
import subprocess
from pathlib import Path

import numpy as np
import pytest

import refdrive
import scenes
from parity import color_stats, COLOR_MAX_LSB, COLOR_1LSB_FRACTION

pytestmark = pytest.mark.gpu

CASES = {
    "config1": lambda: scenes.config1(),
    "mixed": lambda: scenes.small_scene(seed=21, width=240, height=160),
    "ssaa2": lambda: scenes.small_scene(seed=22, width=160, height=120, ssaa=2),
    "flat": lambda: dataclasses.replace(scenes.small_scene(seed=23), smooth=False),
    "coplanar": lambda: scenes.coplanar_scene(seed=24),
    # blended meshes: the core's own transparent pass drives the ordered path
    "transparent": lambda: scenes.transparent_scene(seed=25),
    "transparent_ssaa2": lambda: scenes.transparent_scene(seed=26, width=128, height=96, ssaa=2),
    "transparent_flat": lambda: dataclasses.replace(
        scenes.transparent_scene(seed=62, width=128, height=96, ssaa=2), smooth=False),
    # no lights: the core's legacy smooth rasteriser (silhouette edge AA)
    "unlit_smooth": lambda: scenes.small_scene(seed=29, lights="none", width=192, height=144),
    # directional-light shadows: the core's pass_shadow vs the C-ABI shadow pass
    "shadow": lambda: scenes.shadow_scene(seed=27, width=192, height=144),
    "shadow_ssaa2_transparent": lambda: scenes.shadow_scene(seed=28, width=128, height=96,
                                                            ssaa=2, transparent=True),
    # MOP_POST_FOG through mop_viewport_set_fog: the core applies post effects for its CPU
    # backend only; the harness hands vp->post_effects and vp->fog_params to the device
    # (the integration patch's post-process row) from a MOP_STAGE_PRE_SCENE hook
    "fog": lambda: dataclasses.replace(
        scenes.small_scene(seed=63, width=192, height=144),
        post_effects=scenes.DEFAULT_POST | scenes.POST_FOG, fog=((0.6, 0.65, 0.7, 1.0), 0.85, 0.99)),
    "fog_all_effects_ssaa2": lambda: dataclasses.replace(
        scenes.small_scene(seed=64, width=160, height=120, ssaa=2),
        post_effects=(scenes.POST_GAMMA | scenes.POST_TONEMAP | scenes.POST_VIGNETTE
                      | scenes.POST_FOG | scenes.POST_FXAA),
        fog=((0.2, 0.3, 0.5, 1.0), 0.9, 0.995)),
    # mop_viewport_add_instanced_mesh: the core's pass_instanced calls the RHI's
    # draw_instanced with the depth write off (cpu_backend.c:638-657, 536-580)
    "instanced": lambda: scenes.instanced_scene(seed=65),
    "instanced_zero_id_ssaa2": lambda: scenes.instanced_scene(seed=66, width=160, height=120,
                                                              ssaa=2, zero_id=True),
    "instanced_transparent": lambda: scenes.instanced_scene(seed=67, transparent=True),
    # meshes with editor-chrome IDs: the core draws them with the depth test off
    "chrome": lambda: scenes.chrome_scene(seed=68),
    # BC1 / BC3 / BC5 textures through mop_tex_create -> texture_create_ex
    "bc_textures": lambda: scenes.bc_scene(seed=69),
    # the environment behind the scene: the core's CPU sky pass against the RHI's
    # draw_skybox (IBL maps handed over by the harness hook, as the patch's IBL row)
    "env_background": lambda: dataclasses.replace(scenes.small_scene(seed=74, env=1),
                                                  env_background=True),
    # MOP_RENDER_WIREFRAME through mop_viewport_set_render_mode: the core marks every
    # draw but ID 0 wireframe; with the chrome off its hidden grid (a zero-opacity blended
    # chrome mesh) is drawn as lines too, on both backends
    "wireframe_grid": lambda: dataclasses.replace(scenes.wireframe_scene(seed=75),
                                                  wireframe_grid=True),
    "wireframe_ssaa2_transparent": lambda: dataclasses.replace(
        scenes.transparent_scene(seed=76, width=128, height=96, ssaa=2), wireframe=True),
    "config2_reduced_no_ibl": lambda: dataclasses.replace(
        scenes.config2(width=480, height=270, ssaa=2, instances=48, tex_size=64), env=0),
}


@pytest.mark.parametrize("name", list(CASES))
def test_viewport_api_cuda_matches_cpu(name):
    if not refdrive.REF_CUDA_SO.exists():
        pytest.skip("drop-in harness library not built")
    sc = CASES[name]()
    cpu = refdrive.Reference(sc, serial=True)
    gpu = refdrive.Reference(sc, backend="cuda")
    try:
        a = cpu.render()
        b = gpu.render()
        assert (a["object_id"] == b["object_id"]).all(), "object IDs differ"
        assert (a["depth"].view(np.uint32) == b["depth"].view(np.uint32)).all(), "depth differs"
        for key in ("color", "color_full"):
            s = color_stats(a[key], b[key])
            assert s["max"] <= COLOR_MAX_LSB and s["within1"] >= COLOR_1LSB_FRACTION, (key, s)
        assert a["triangle_count"] == b["triangle_count"]
        xy = scenes.pick_points(sc, 500)
        for x, y in zip(cpu.pick(xy), gpu.pick(xy)):
            assert (np.ascontiguousarray(x).view(np.uint8) ==
                    np.ascontiguousarray(y).view(np.uint8)).all()
    finally:
        gpu.close()
        cpu.close()


@pytest.mark.parametrize("ssaa", [1, 2])
def test_present_to_texture_cuda_matches_cpu(ssaa):
    """mop_viewport_present_to_texture (framebuffer_copy_to_texture): into a
    texture of the framebuffer's size and, with SSAA, of the presented size
    (the box filter); a texture of another size is refused by both
    backends."""
    if not refdrive.REF_CUDA_SO.exists():
        pytest.skip("drop-in harness library not built")
    sc = scenes.small_scene(seed=70 + ssaa, width=160, height=120, ssaa=ssaa)
    cpu = refdrive.Reference(sc, serial=True)
    gpu = refdrive.Reference(sc, backend="cuda")
    try:
        a, b = cpu.render(), gpu.render()
        sizes = [(sc.width * ssaa, sc.height * ssaa)] + ([(sc.width, sc.height)] if ssaa > 1 else [])
        for tw, th in sizes:
            ta, tb = cpu.present_to_texture(tw, th), gpu.present_to_texture(tw, th)
            assert ta is not None and tb is not None
            s_ = color_stats(ta, tb)
            assert s_["max"] <= COLOR_MAX_LSB and s_["within1"] >= COLOR_1LSB_FRACTION, (tw, s_)
            key = "color_full" if tw == sc.width * ssaa else "color"
            assert (tb == b[key]).all()
        assert cpu.present_to_texture(sc.width + 3, sc.height) is None
        assert gpu.present_to_texture(sc.width + 3, sc.height) is None
    finally:
        gpu.close()
        cpu.close()


def test_render_target_cuda_matches_cpu():
    """MopViewportDesc.render_target (framebuffer_create_from_texture): the
    viewport renders into a host texture; after each frame its pixels equal
    the frame's colour, on both backends."""
    if not refdrive.REF_CUDA_SO.exists():
        pytest.skip("drop-in harness library not built")
    sc = scenes.small_scene(seed=73, width=160, height=120, ssaa=1)
    cpu = refdrive.Reference(sc, serial=True, render_target=True)
    gpu = refdrive.Reference(sc, backend="cuda", render_target=True)
    try:
        a, b = cpu.render(), gpu.render()
        ta, tb = cpu.read_target(), gpu.read_target()
        assert (ta == a["color_full"]).all() and (tb == b["color_full"]).all()
        s_ = color_stats(ta, tb)
        assert s_["max"] <= COLOR_MAX_LSB and s_["within1"] >= COLOR_1LSB_FRACTION, s_
        assert (a["object_id"] == b["object_id"]).all()
    finally:
        gpu.close()
        cpu.close()


REFTESTS = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "tests"

# the reference's own test programs that drive the public viewport API, with
# their check counts (each passes them all on the reference's CPU backend)
REFERENCE_SUITES = {"test_torture_picking": 10, "test_torture_depth": 8,
                    "test_torture_golden": 6, "test_torture_geometry": 12,
                    "test_torture_lighting": 8, "test_torture_hierarchy": 9,
                    "test_torture_camera": 10, "test_exposure": 3, "test_skinning": 8,
                    "test_morph_targets": 7, "test_procedural_sky": 4,
                    "test_ortho_camera": 6}


@pytest.mark.parametrize("suite", list(REFERENCE_SUITES))
def test_reference_suite_on_cuda_backend(suite):
    """The reference's own tests/<suite>.c, compiled unmodified and linked
    with the drop-in objects (oracle/Makefile `reftests`): every viewport it
    creates runs on the CUDA backend and all of its checks pass (picks at
    corners, boundaries, out of range, through hierarchies, with SSAA and
    transparency; depth order and planes; golden determinism; geometry,
    lighting, camera, exposure, skinning, morph and sky cases)."""
    exe = REFTESTS / f"{suite}_cuda"
    if not exe.exists():
        pytest.skip("reference test programs not built (reference tree absent at build time)")
    p = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    out = p.stdout
    assert p.returncode == 0, out[-3000:] + p.stderr[-2000:]
    assert f"Passed: {REFERENCE_SUITES[suite]}" in out and "FAIL" not in out, out[-3000:]
