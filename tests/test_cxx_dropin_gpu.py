"""The C ABI from C++: tests/cxx/dropin_sweep.cpp, written like the body of
backTransformKMOR (KrylovROMSubstructure.cpp:1393-1460) with its frequency loop replaced by the C ABI,
is compiled with g++ against include/staccato_rom.h and the library, reads its ROM from dense
Matrix Market files, sweeps it through srom_sweep_host with the fused back-projection and
writes y.  y must equal the oracle's C_r x bit for bit (FP64 form)."""
import math
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from staccato_b200 import rom_io, workloads as W

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cxx_caller_sweeps_rom_files(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    exe = tmp_path / "dropin_sweep"
    lib_dir = os.path.join(ROOT, "staccato_b200")
    subprocess.run([gxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cxx", "dropin_sweep.cpp"), "-L", lib_dir, "-lstaccato_rom",
                    "-Wl,-rpath," + lib_dir, "-o", str(exe)], check=True)
    rom = W.plain_rom(F=2)
    n = rom.n
    rng = np.random.default_rng(8)
    B = rng.standard_normal((n, 2))
    F = rng.standard_normal((2, 3))
    C = rng.standard_normal((5, n))
    eta, f0, f1, count = 0.0, 1.0, 900.0, 37
    for name, a in (("K", rom.K), ("M", rom.M), ("BF", B @ F), ("C", C)):
        rom_io.write_mtx_dense(str(tmp_path / f"{name}.mtx"), a)
    subprocess.run([str(exe), str(tmp_path), str(eta), str(f0), str(f1), str(count)], check=True)
    Y = rom_io.read_mtx_dense(str(tmp_path / "Y.mtx"))  # (n_out*r, count)
    freq = np.array([f0 + (f1 - f0) * i / (count - 1) for i in range(count)])
    X, info = O.sweep(rom.K, rom.M, None, eta, (B @ F).astype(complex), 2 * math.pi * freq)
    Yo = O.backproject(C.astype(complex), X)  # (count, n_out, r)
    Yo = np.stack([Yo[f].ravel(order="F") for f in range(count)], axis=1)
    assert np.array_equal(np.ascontiguousarray(Y).view(np.uint64), np.ascontiguousarray(Yo).view(np.uint64))
    assert np.array_equal(np.loadtxt(tmp_path / "info.txt", dtype=int), info)
