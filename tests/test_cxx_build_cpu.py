"""The C++ callers in tests/cxx compile against include/staccato_rom.h and link against the
library with g++ (no GPU needed): the documented C usage of the Krylov basis and full-order
sweep entry points builds as written."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("src", ["krylov_chain.cpp", "dropin_sweep.cpp"])
def test_cxx_callers_compile_and_link(tmp_path, src):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    lib_dir = os.path.join(ROOT, "staccato_b200")
    cuda = "/usr/local/cuda"
    cmd = [gxx, "-O2", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cxx", src), "-L", lib_dir, "-lstaccato_rom", "-Wl,-rpath," + lib_dir,
           "-o", str(tmp_path / "a.out")]
    if src == "krylov_chain.cpp":
        cmd[5:5] = ["-I", os.path.join(cuda, "include")]
        cmd += ["-L", os.path.join(cuda, "lib64"), "-lcudart"]
    subprocess.run(cmd, check=True)
    assert (tmp_path / "a.out").exists()
