"""Vertex deformation on the device (mopcuda_skin_apply / mopcuda_morph_apply)
against the oracle's restatement of the core's mop_skin_apply /
mop_morph_apply, byte for byte (the oracle is pinned to the reference core in
tests/test_oracle.py).  Cases: with and without normals, a padded stride,
weights <= 0 and joints beyond the bone count (skipped), zero normals, bones
beyond the shared-memory staging, morph with zero weights and with more
targets than the shared-memory staging."""
import numpy as np
import pytest

import cpu_oracle
import mopcuda
from parity import deform_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed,vc,bones,stride,normals", [
    (1, 1000, 64, 44, True),
    (2, 100_000, 64, 44, True),
    (3, 4096, 200, 48, False),
    (4, 3000, 300, 44, True),   # > 256 bones: read from global memory
])
def test_skin_matches_oracle(cuda_device, seed, vc, bones, stride, normals):
    raw, mats = deform_case(seed, vc, bones, stride)
    lay = (stride, 0, 12 if normals else -1, 24, 28)
    got = mopcuda.deform(cuda_device, raw, vc, lay, bones=mats)
    want = cpu_oracle.skin(lay, raw, vc, mats)
    assert (got == want).all(), f"{int((got != want).sum())} bytes differ"


@pytest.mark.parametrize("seed,vc,targets", [(5, 20_000, 4), (6, 64, 1100)])
def test_morph_matches_oracle(cuda_device, seed, vc, targets):
    raw, _ = deform_case(seed, vc)
    rng = np.random.default_rng(seed)
    t = rng.normal(size=(targets, vc, 3)).astype(np.float32)
    w = rng.normal(size=targets).astype(np.float32)
    w[::3] = 0.0
    lay = (44, 0, 12, 24, 28)
    got = mopcuda.deform(cuda_device, raw, vc, lay, targets=t, weights=w)
    want = cpu_oracle.morph(lay, raw, vc, t, w)
    assert (got == want).all(), f"{int((got != want).sum())} bytes differ"
