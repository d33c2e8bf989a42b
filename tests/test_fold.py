"""fold_add (master-of-puppets_b200/csrc/fold.h) — the closed-form replacement
for the reference's incremental edge stepping (rasterizer.c:1926-2151) —
must equal the plain serial loop bit for bit.  The header is compiled for the
host here and checked on 1.2 M random cases (k up to 5000, including exact
ties d = (M + 1/2) ulp(w) of both parities, zero crossings and binade
changes)."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def test_fold_matches_serial(tmp_path):
    so = tmp_path / "fold_check.so"
    subprocess.run(["gcc", "-O2", "-std=c11", "-shared", "-fPIC", "-ffp-contract=off",
                    "-I", str(ROOT / "master-of-puppets_b200" / "csrc"),
                    str(ROOT / "tests" / "native" / "fold_check.c"), "-o", str(so)], check=True)
    lib = C.CDLL(str(so))
    lib.fold_check.argtypes = [C.c_int, C.c_uint64, C.c_void_p]
    bad = np.zeros(5, np.float32)
    for seed in (1, 2, 3, 4, 5, 6):
        fails = lib.fold_check(200000, seed, bad.ctypes.data)
        assert fails == 0, f"seed {seed}: first mismatch w,d,k,fold,serial = {bad}"
