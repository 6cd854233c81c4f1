"""tests/cxx/krylov_chain.cpp -- the C++ caller of srom_krylov_basis and srom_fom_sweep -- built
with g++ against the header and the library and run: the basis of the spring-mass chain has
the expected 8 columns (2 expansion points x order 4, nothing deflated) and is orthonormal, and
the full-order tip response equals a dense numpy solve."""
import math
import os
import shutil
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _tip(n, f):
    K = np.diag(np.full(n, 2.0))
    K[-1, -1] = 1.0
    K += np.diag(np.full(n - 1, -1.0), 1) + np.diag(np.full(n - 1, -1.0), -1)
    w = 2 * math.pi * f
    b = np.zeros(n)
    b[-1] = 1.0
    return np.linalg.solve(K - w * w * np.eye(n) / n, b)[-1]


def test_cxx_krylov_and_full_order_caller(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    lib_dir = os.path.join(ROOT, "staccato_b200")
    exe = tmp_path / "krylov_chain"
    subprocess.run([gxx, "-O2", "-std=c++17", "-I", "/usr/local/cuda/include", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cxx", "krylov_chain.cpp"), "-L", lib_dir, "-lstaccato_rom",
                    "-Wl,-rpath," + lib_dir, "-L", "/usr/local/cuda/lib64", "-lcudart", "-o", str(exe)], check=True)
    for n in (200, 37):
        out = subprocess.run([str(exe), str(n)], check=True, capture_output=True, text=True).stdout.split()
        cols, orth, tip_re, tip_im = int(out[1]), float(out[3]), float(out[5]), float(out[6])
        assert cols == 8 and orth <= 1e-12
        ref = _tip(n, 0.03)
        assert abs(tip_re - ref) <= 1e-10 * abs(ref) and abs(tip_im) <= 1e-10 * abs(ref)
