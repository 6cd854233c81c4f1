"""The C-ABI library loads and exports every declared symbol; struct layouts agree."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from staccato_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR_DIR = os.path.join(ROOT, "include")


def _declared():
    names = []
    for f in sorted(os.listdir(HDR_DIR)):
        if f.endswith(".h"):
            with open(os.path.join(HDR_DIR, f)) as fh:
                txt = fh.read()
            names += re.findall(r"SROM_API\s+[\w\s\*]+?\b(srom_\w+)\s*\(", txt)
    return names


def test_library_loads_and_exports_every_declared_symbol():
    lib = _capi.lib()
    names = _declared()
    assert names, "no SROM_API declarations found"
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_capi.EXPORTS)
    assert lib.srom_version() >= 100


def test_status_strings():
    lib = _capi.lib()
    assert lib.srom_status_string(0) == b"ok"
    assert b"unsupported" in lib.srom_status_string(5)


def test_struct_layout_matches_header():
    src = r'''
#include <stddef.h>
#include <stdio.h>
#include "staccato_rom.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(srom_rom_desc), offsetof(srom_rom_desc, eta),
         offsetof(srom_rom_desc, ldb), offsetof(srom_rom_desc, ipiv), sizeof(srom_sweep_opts),
         offsetof(srom_sweep_opts, flags));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        with open(c, "w") as fh:
            fh.write(src)
        subprocess.run(["gcc", "-I", HDR_DIR, c, "-o", exe], check=True)
        got = [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    R, S = _capi.RomDesc, _capi.SweepOpts
    want = [C.sizeof(R), R.eta.offset, R.ldb.offset, R.ipiv.offset, C.sizeof(S), S.flags.offset]
    assert got == want


def test_create_without_gpu_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    st = _capi.lib().srom_create(C.byref(h), 0)
    assert st != _capi.SROM_OK and not h


def test_noalloc_rejects_misaligned_arrays_before_any_cuda_call():
    """srom_complex only promises 8-byte alignment but the kernels access complex values as
    16-byte vectors: an array that is not 16-byte aligned is an argument error.  The check
    comes before any CUDA call, so fake addresses that are never dereferenced exercise it."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("fake device addresses are only used without a GPU")
    base = 0x10000

    def desc(**shift):
        d = _capi.RomDesc()
        d.n, d.r, d.F, d.ldk, d.ldb, d.eta = 4, 1, 2, 4, 4, 0.0
        for i, f in enumerate(("K", "M", "rhs", "omega", "X")):
            setattr(d, f, base + 0x1000 * i + shift.get(f, 0))
        return d

    err = C.create_string_buffer(256)
    for field, off in (("K", 8), ("M", 8), ("rhs", 8), ("X", 8), ("omega", 4)):
        d = desc(**{field: off})
        st = _capi.lib().srom_sweep_fp64_noalloc(C.byref(d), None, err, 256)
        assert st == _capi.SROM_ERR_INVALID, (field, err.value)
        assert b"aligned" in err.value
    d = desc()  # aligned: gets past the check and fails only for want of a device
    st = _capi.lib().srom_sweep_fp64_noalloc(C.byref(d), None, err, 256)
    assert st == _capi.SROM_ERR_CUDA, err.value


def test_null_handle_is_rejected_by_every_handle_call():
    """Calls that take a handle return SROM_ERR_INVALID for a null one (no CUDA call made)."""
    L = _capi.lib()
    n_cols = C.c_int(-1)
    assert L.srom_krylov_basis(None, 4, 4, None, None, 0, 0, None, None, None, None, 1, 4, None, 1, 1, 0.0,
                               None, 4, 4, C.byref(n_cols)) == _capi.SROM_ERR_INVALID
    assert L.srom_fom_sweep(None, 4, 4, None, None, 0, 0, None, None, None, None, 1, 4, None, 1, None,
                            4) == _capi.SROM_ERR_INVALID
    assert L.srom_sweep(None, None, 0, None) == _capi.SROM_ERR_INVALID
    assert L.srom_orthonormalize(None, None, 4, 1, 4, 2) == _capi.SROM_ERR_INVALID


def test_python_wrappers_refuse_host_tensors():
    """The wrappers pass device pointers to the C ABI; host tensors are refused before any call."""
    import numpy as np
    import torch

    from staccato_b200.krylov import fom_sweep, krylov_basis
    from staccato_b200.project import DeviceCsr, project, project_complex

    csr = DeviceCsr(n_rows=4, rowptr=torch.zeros(5, dtype=torch.int64), colind=torch.zeros(0, dtype=torch.int32))
    z = torch.zeros(0, dtype=torch.complex128)
    with pytest.raises(ValueError):
        project_complex(None, csr, [z], torch.zeros((2, 4), dtype=torch.complex128))
    with pytest.raises(ValueError):
        project(None, csr, [torch.zeros(0, dtype=torch.float64)], torch.zeros((2, 4), dtype=torch.float64))
    with pytest.raises(ValueError):
        krylov_basis(None, csr, z, z, None, torch.zeros((1, 4), dtype=torch.complex128), [1.0], 1)
    with pytest.raises(ValueError):
        fom_sweep(None, csr, z, z, None, torch.zeros((1, 4), dtype=torch.complex128), np.array([1.0]))
