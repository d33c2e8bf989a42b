"""Compressed textures and render-to-texture through the C ABI.

* mopcuda_texture_create_ex decodes BC1 / BC3 / BC5 blocks on the device to
  the bytes the oracle's restatement of the CPU backend's
  bc_decompress_to_rgba8 gives (the oracle itself is pinned to the reference
  in tests/test_oracle.py), for odd sizes too; BC7, unknown formats and short
  data are refused; frames sampling compressed textures match the oracle.
* mopcuda_framebuffer_copy_to_texture copies the post-processed colour into
  a texture of the framebuffer's size or box-filters it into one a whole SSAA
  factor smaller (the presented image), and refuses other sizes.
* mopcuda_framebuffer_create_from_texture makes a framebuffer whose frames
  land in the texture.
"""
import dataclasses

import numpy as np
import pytest

import cpu_oracle
import mopcuda
import scenes
from parity import assert_frame_parity

pytestmark = pytest.mark.gpu

BC = [(scenes.TEX_BC1, 8, 8), (scenes.TEX_BC1, 13, 7), (scenes.TEX_BC1, 1024, 1024),
      (scenes.TEX_BC3, 64, 36), (scenes.TEX_BC3, 5, 5), (scenes.TEX_BC5, 33, 70),
      (scenes.TEX_BC5, 1, 1)]


def _create(dev, t, size=None):
    b = np.ascontiguousarray(t.data, np.uint8)
    return dev.L.mopcuda_texture_create_ex(dev.h, t.width, t.height, t.format, 1, b.ctypes.data,
                                           b.size if size is None else size)


def _read(dev, tex, w, h):
    out = np.zeros((h, w, 4), np.uint8)
    assert dev.L.mopcuda_texture_read_rgba8(dev.h, tex, out.ctypes.data, out.nbytes) == 0
    return out


@pytest.mark.parametrize("fmt,w,h", BC)
def test_texture_create_ex_decodes_as_oracle(cuda_device, fmt, w, h):
    t = scenes.bc_texture(np.random.default_rng(10 * fmt + w), fmt, w, h)
    tex = _create(cuda_device, t)
    assert tex, mopcuda.last_error()
    try:
        assert (_read(cuda_device, tex, w, h) == cpu_oracle.bc_decode(t)).all()
    finally:
        cuda_device.L.mopcuda_texture_destroy(cuda_device.h, tex)


def test_texture_create_ex_refusals(cuda_device):
    L, d = cuda_device.L, cuda_device.h
    rng = np.random.default_rng(3)
    bc7 = scenes.bc_texture(rng, scenes.TEX_BC7, 8, 8)
    assert not _create(cuda_device, bc7)
    assert "BC7" in mopcuda.last_error()
    assert not _create(cuda_device, scenes.CompressedTexture(8, 8, 9, bc7.data))
    t = scenes.bc_texture(rng, scenes.TEX_BC3, 12, 12)
    assert not _create(cuda_device, t, size=t.data.size - 1)  # one byte short
    assert "needs" in mopcuda.last_error()
    # format 0 is the RGBA8 path
    rgba = rng.integers(0, 256, (5, 7, 4), dtype=np.uint8)
    tex = L.mopcuda_texture_create_ex(d, 7, 5, 0, 1, rgba.ctypes.data, rgba.nbytes)
    assert tex
    try:
        assert (_read(cuda_device, tex, 7, 5) == rgba).all()
    finally:
        L.mopcuda_texture_destroy(d, tex)


@pytest.mark.parametrize("ssaa", [1, 2])
def test_bc_textured_frame_matches_oracle(cuda_device, ssaa):
    sc = scenes.bc_scene(seed=92 + ssaa, ssaa=ssaa)
    ref = cpu_oracle.render(sc, None)
    r = mopcuda.SceneRenderer(cuda_device, sc)
    try:
        r.render()
        got = {"object_id": r.object_id(), "depth": r.depth(), "color_full": r.color_full(),
               "color": r.color()}
        assert_frame_parity(got, ref, f"bc ssaa{ssaa}")
        assert (got["color_full"] == ref["color_full"]).all()  # no IBL: bit-exact
    finally:
        r.close()


def test_copy_to_texture_same_size_and_box(cuda_device):
    sc = scenes.small_scene(seed=95, width=160, height=120, ssaa=2)
    r = mopcuda.SceneRenderer(cuda_device, sc)
    L, d = cuda_device.L, cuda_device.h
    made = []
    try:
        r.render()
        full, presented = r.color_full(), r.color()
        zero = np.zeros((r.sh, r.sw, 4), np.uint8)
        t_full = L.mopcuda_texture_create(d, r.sw, r.sh, zero.ctypes.data)
        t_pres = L.mopcuda_texture_create(d, sc.width, sc.height, zero.ctypes.data)
        t_odd = L.mopcuda_texture_create(d, 100, 60, zero.ctypes.data)
        made += [t_full, t_pres, t_odd]
        assert L.mopcuda_framebuffer_copy_to_texture(d, r.fb, t_full) == 0, mopcuda.last_error()
        assert L.mopcuda_framebuffer_copy_to_texture(d, r.fb, t_pres) == 0, mopcuda.last_error()
        assert (_read(cuda_device, t_full, r.sw, r.sh) == full).all()
        assert (_read(cuda_device, t_pres, sc.width, sc.height) == presented).all()
        assert L.mopcuda_framebuffer_copy_to_texture(d, r.fb, t_odd) == mopcuda.EINVAL
        assert "unsupported size" in mopcuda.last_error()
        # a pending frame is completed first: submit without waiting, then copy
        r.submit()
        assert L.mopcuda_framebuffer_copy_to_texture(d, r.fb, t_full) == 0
        assert (_read(cuda_device, t_full, r.sw, r.sh) == full).all()
    finally:
        for t in made:
            if t:
                L.mopcuda_texture_destroy(d, t)
        r.close()


def test_framebuffer_from_texture_receives_frames(cuda_device):
    sc = scenes.small_scene(seed=96, width=128, height=96, ssaa=1)
    L, d = cuda_device.L, cuda_device.h
    zero = np.zeros((sc.height, sc.width + 1, 4), np.uint8)
    tex = L.mopcuda_texture_create(d, sc.width, sc.height, zero.ctypes.data)
    wrong = L.mopcuda_texture_create(d, sc.width + 1, sc.height, zero.ctypes.data)
    assert not L.mopcuda_framebuffer_create_from_texture(d, wrong, sc.width, sc.height)
    assert "size mismatch" in mopcuda.last_error()
    r = mopcuda.SceneRenderer(cuda_device, sc)
    own = r.fb
    fb = L.mopcuda_framebuffer_create_from_texture(d, tex, sc.width, sc.height)
    assert fb, mopcuda.last_error()
    try:
        r.fb = fb
        r.render()
        first = r.color_full()
        assert (_read(cuda_device, tex, sc.width, sc.height) == first).all()
        assert (first == cpu_oracle.render(sc, None)["color_full"]).all()
        # the next frame (another camera) replaces the texture's contents
        r.scene = dataclasses.replace(sc, eye=(-4.0, 2.5, 6.0))
        r.update_camera()
        r.render()
        second = r.color_full()
        assert not (second == first).all()
        assert (_read(cuda_device, tex, sc.width, sc.height) == second).all()
    finally:
        r.fb = own
        L.mopcuda_framebuffer_destroy(d, fb)
        r.close()
        L.mopcuda_texture_destroy(d, tex)
        L.mopcuda_texture_destroy(d, wrong)
