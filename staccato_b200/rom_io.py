"""Dense ROM files of the reference's tests, read and written by the library's host code.

* ``read_mtx_dense(path)`` -- io::readMtxDense (test/krylovTestGPU/matrixInSingleLoop/gpu/
  src/io/io.cu:20-80): complex "re im" entries column after column (also standard Matrix
  Market "array real" files and the reference's "dense row major" banner);
* ``write_mtx_dense(path, A)`` -- AuxiliaryFunctions::writeMKLComplexDenseMatrixMtxFormat
  (src/tools/AuxiliaryFunctions.cpp:80-110), exact round trip;
* ``write_solution(path, x)`` -- io::writeSolVecComplex (io.cu:83-106);
* ``load_rom(directory, K=..., M=..., D=...)`` -- the K / M / D file triple a reference test
  reads (test/krylovTestGPU/matrixInSingleLoop/gpu/src/main.cu:106-114).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import _capi


class RomFileError(OSError):
    pass


def _check(status: int, err) -> None:
    if status != _capi.SROM_OK:
        raise RomFileError(err.value.decode() or _capi.lib().srom_status_string(status).decode())


def read_mtx_dense(path: str) -> np.ndarray:
    """rows x cols complex128 array (Fortran order) from a dense Matrix Market file."""
    L = _capi.lib()
    err = C.create_string_buffer(512)
    rows, cols = C.c_int64(), C.c_int64()
    p = os.fsencode(path)
    _check(L.srom_mtx_read_dense(p, C.byref(rows), C.byref(cols), None, 0, err, 512), err)
    A = np.empty((rows.value, cols.value), dtype=np.complex128, order="F")
    _check(L.srom_mtx_read_dense(p, C.byref(rows), C.byref(cols), A.ctypes.data_as(C.c_void_p), A.size, err, 512),
           err)
    return A


def write_mtx_dense(path: str, A) -> None:
    A = np.asfortranarray(np.asarray(A, dtype=np.complex128))
    if A.ndim == 1:
        A = A[:, None]
    err = C.create_string_buffer(512)
    rows, cols = A.shape
    _check(_capi.lib().srom_mtx_write_dense(os.fsencode(path), rows, cols, A.ctypes.data_as(C.c_void_p),
                                            max(rows, 1), err, 512), err)


def write_solution(path: str, x) -> None:
    x = np.ascontiguousarray(np.asarray(x, dtype=np.complex128).ravel(order="F"))
    err = C.create_string_buffer(512)
    _check(_capi.lib().srom_write_solution(os.fsencode(path), x.ctypes.data_as(C.c_void_p), x.size, err, 512), err)


def read_solution(path: str) -> np.ndarray:
    """The complex vector of a ``write_solution`` (or reference) solution table."""
    t = np.loadtxt(path, skiprows=1, ndmin=2)
    return t[:, 0] + 1j * t[:, 1]


def load_rom(directory: str, K: str, M: str, D: Optional[str] = None):
    """(K, M, D) complex matrices from the reference's per-ROM files (D None when absent)."""
    j = lambda f: os.path.join(directory, f)
    return read_mtx_dense(j(K)), read_mtx_dense(j(M)), (read_mtx_dense(j(D)) if D else None)
