"""CPU-side checks of the drop-in boundary (no GPU needed):

* libmopcuda.so loads and exports every function include/mop_cuda.h declares;
* libmop_rhi_cuda.so exports mop_rhi_backend_cuda (the RHI table);
* the library's host-side matrices are bit-identical to the reference's
  (camera chain, mvp products, TRS composition);
* the ctypes structures of the Python binding have the header's sizes and
  field offsets (a C probe compiled against include/mop_cuda.h);
* every entry point given null handles and pointers returns an error or a
  neutral value (NULL, 0, "no hit") instead of crashing;
* without a CUDA device, device creation fails loudly (no CPU fallback).
"""
import ctypes as C
import json
import re
import shutil
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import cpu_oracle
import mopcuda
import refdrive
import scenes

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "mop_cuda.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mopcuda_[a-z0-9_]+)\s*\(", text)))


def exported(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib_path)], capture_output=True,
                         text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_header_symbols_exported():
    names = declared_functions()
    assert len(names) >= 40
    have = exported(mopcuda.LIB_PATH)
    missing = [n for n in names if n not in have]
    assert not missing, f"declared but not exported: {missing}"


def test_binding_covers_header():
    bound = {s[0] for s in mopcuda.SIGNATURES}
    assert set(declared_functions()) <= bound
    mopcuda.lib()  # every signature resolves


def test_rhi_table_exported():
    so = ROOT / "master-of-puppets_b200" / "libmop_rhi_cuda.so"
    if not so.exists():
        pytest.skip("RHI table library not built (needs the reference headers)")
    assert "mop_rhi_backend_cuda" in exported(so)


@pytest.mark.parametrize("make", [scenes.config1, lambda: scenes.small_scene(3),
                                  lambda: scenes.coplanar_scene(),
                                  lambda: scenes.config2(instances=6, tex_size=8)])
def test_host_matrices_match_oracle(make):
    sc = make()
    v1, p1, e1 = mopcuda.camera_matrices(sc)
    v2, p2, e2 = cpu_oracle.camera(sc)
    for a, b in ((v1, v2), (p1, p2), (e1, e2)):
        assert (a.view(np.uint32) == b.view(np.uint32)).all()
    for m in sc.meshes:
        a = mopcuda.mat4_multiply(p1, mopcuda.mat4_multiply(v1, m.transform))
        b = cpu_oracle.mat4_multiply(p2, cpu_oracle.mat4_multiply(v2, m.transform))
        assert (a.view(np.uint32) == b.view(np.uint32)).all()


def test_shadow_light_vp_matches_oracle():
    """mopcuda_shadow_light_vp (the product's pass_shadow light camera) vs
    the oracle's restatement, on random caster sets and light directions,
    including directions within the up-vector switch and scenes small enough
    for the radius clamp."""
    rng = np.random.default_rng(6)
    dirs = [(0.0, -1.0, 0.0), (0.05, -1.0, 0.02), (-0.4, -0.9, -0.3), (1.0, 0.0, 0.0),
            (0.0, 0.0, 0.0)]
    dirs += [tuple(rng.normal(size=3)) for _ in range(40)]
    for k, dr in enumerate(dirs):
        n = int(rng.integers(1, 12))
        scale = 0.05 if k % 5 == 0 else 2.0
        models = np.concatenate([
            scenes.mat_trs(rng.uniform(-8, 8, 3), scenes.random_rotation(rng),
                           rng.uniform(0.1, 1.0, 3) * scale) for _ in range(n)]).astype(np.float32)
        d = np.asarray(dr, np.float32)
        a = np.zeros(16, np.float32)
        b = np.zeros(16, np.float32)
        assert mopcuda.lib().mopcuda_shadow_light_vp(models.ctypes.data, n, d.ctypes.data,
                                                    a.ctypes.data) == 1
        assert cpu_oracle.lib().oracle_shadow_matrix(models.ctypes.data, n, d.ctypes.data,
                                                     b.ctypes.data) == 1
        assert (a.view(np.uint32) == b.view(np.uint32)).all(), dr
    assert mopcuda.lib().mopcuda_shadow_light_vp(models.ctypes.data, 0, d.ctypes.data,
                                                a.ctypes.data) == 0


@pytest.mark.skipif(not refdrive.available(), reason="reference library not built")
def test_compose_trs_matches_reference():
    """mopcuda_mat4_compose_trs vs the reference's own mop_mat4_compose_trs."""
    ref = refdrive.lib()

    class M4(C.Structure):
        _fields_ = [("d", C.c_float * 16)]

    class V3(C.Structure):
        _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]

    ref.mop_mat4_compose_trs.restype = M4
    ref.mop_mat4_compose_trs.argtypes = [V3, V3, V3]
    rng = np.random.default_rng(4)
    for _ in range(200):
        p, r, s = (rng.uniform(-5, 5, 3).astype(np.float32) for _ in range(3))
        want = np.array(ref.mop_mat4_compose_trs(V3(*p), V3(*r), V3(*s)).d[:], np.float32)
        got = np.zeros(16, np.float32)
        mopcuda.lib().mopcuda_mat4_compose_trs(p.ctypes.data, r.ctypes.data, s.ctypes.data,
                                              got.ctypes.data)
        assert (got.view(np.uint32) == want.view(np.uint32)).all()


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="a CUDA device is present")
def test_no_gpu_fails_loudly():
    with pytest.raises(RuntimeError):
        mopcuda.Device(0)


PUBLIC_STRUCTS = [mopcuda.MopCudaLight, mopcuda.MopCudaVertexLayout, mopcuda.MopCudaDraw,
                  mopcuda.MopCudaShadowCaster, mopcuda.MopCudaDeformLayout, mopcuda.MopCudaView,
                  mopcuda.MopCudaBatchConfig, mopcuda.MopCudaServerConfig,
                  mopcuda.MopCudaRequest, mopcuda.MopCudaServerStats]


@pytest.mark.skipif(shutil.which("cc") is None, reason="no C compiler")
def test_struct_layouts_match_header(tmp_path):
    """Every public struct of mop_cuda.h has a ctypes mirror of the same size
    whose fields sit at the C offsets (a field missing from the header fails
    the compile)."""
    text = HEADER.read_text()
    declared = set(re.findall(r"\}\s*(MopCuda[A-Za-z]+)\s*;", text))
    assert declared == {c.__name__ for c in PUBLIC_STRUCTS}, declared
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "mop_cuda.h"',
             "int main(void) {"]
    for cls in PUBLIC_STRUCTS:
        t = cls.__name__
        lines.append(f'  printf("{t} sizeof %zu\\n", sizeof({t}));')
        for name, *_ in cls._fields_:
            lines.append(f'  printf("{t} {name} %zu\\n", offsetof({t}, {name}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["cc", "-std=c11", "-I", str(HEADER.parent), str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True,
                               check=True).stdout.splitlines():
        t, name, v = line.split()
        got[(t, name)] = int(v)
    for cls in PUBLIC_STRUCTS:
        t = cls.__name__
        assert got[(t, "sizeof")] == C.sizeof(cls), t
        for name, *_ in cls._fields_:
            assert got[(t, name)] == getattr(cls, name).offset, f"{t}.{name}"


_NULL_SWEEP = r"""
import ctypes as C, json, sys
sys.path[:0] = [sys.argv[1]]
import mopcuda
L = mopcuda.lib()
out = {}
for name, res, argtypes in mopcuda.SIGNATURES:
    print(name, flush=True)
    args = [0.0 if t in (C.c_float, C.c_double) else
            (0 if t in (C.c_int, C.c_uint32, C.c_uint64, C.c_size_t, C.c_int32) else None)
            for t in argtypes]
    r = getattr(L, name)(*args)
    out[name] = r if isinstance(r, (int, float)) or r is None else str(r)
print(json.dumps(out))
"""

# int results that are counts, sizes or "nothing there" rather than status codes
NEUTRAL_INT = {"mopcuda_scene_file_mesh_count", "mopcuda_scene_file_light_count",
               "mopcuda_shadow_light_vp"}


def test_null_arguments_fail_cleanly():
    """Every C entry point called with null handles and pointers (and zero
    sizes) returns instead of crashing: status calls return an error code,
    creates return NULL, counts and sizes 0.  Run in a child process so a
    crash names the function."""
    p = subprocess.run([sys.executable, "-c", _NULL_SWEEP, str(ROOT / "master-of-puppets_b200")],
                       capture_output=True, text=True, timeout=300)
    lines = p.stdout.strip().splitlines()
    assert p.returncode == 0, f"crashed in {lines[-1] if lines else '?'} (rc {p.returncode})"
    got = json.loads(lines[-1])
    for name, res, _ in mopcuda.SIGNATURES:
        if res is C.c_int and name not in NEUTRAL_INT:
            assert got[name] != 0, f"{name} accepted null arguments"
        elif res is mopcuda._P:
            assert got[name] is None, f"{name} returned a handle for null arguments"
