"""ctypes binding of ``libstaccato_rom.so`` (the C ABI in include/staccato_rom.h).

The library is built in-tree by ``staccato_b200/build.py``.  There is no fallback: if the
shared object is missing or cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libstaccato_rom.so")

SROM_OK = 0
SROM_ERR_INVALID = 1
SROM_ERR_CUDA = 2
SROM_ERR_ALLOC = 3
SROM_ERR_TIMEOUT = 4
SROM_ERR_UNSUPPORTED = 5

SROM_FP64 = 0
SROM_MIXED_FP32 = 1
SROM_MIXED_TC = 2
SROM_MIXED_AUTO = 3

SROM_FLAG_FALLBACK_FP64 = 1
SROM_FLAG_KEEP_FACTORS = 2
SROM_FLAG_MIXED_EVERY = 4

SROM_INFO_NOT_CONVERGED = -1

#: every symbol include/staccato_rom.h declares (checked by the CPU test-suite)
EXPORTS = [
    "srom_create", "srom_destroy", "srom_set_stream", "srom_status_string", "srom_last_error",
    "srom_version", "srom_sweep", "srom_sweep_host", "srom_profile_enable", "srom_profile_read",
    "srom_sweep_fp64_noalloc", "srom_project_real", "srom_project_complex", "srom_orthonormalize",
    "srom_sweep_backward",
    "srom_graph_create", "srom_graph_launch", "srom_graph_destroy", "srom_tune",
    "srom_mtx_read_dense", "srom_mtx_write_dense", "srom_write_solution",
    "srom_krylov_basis", "srom_band_order", "srom_fom_sweep", "srom_zgemm_batched", "srom_band_pivot_report",
    "srom_band_cache_report", "srom_band_cache_release",
]

SROM_OP_N = 0
SROM_OP_T = 1
SROM_OP_C = 2

SROM_DPARAM_LOWRANK = 0
SROM_DPARAM_DENSE = 1


class Complex(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class DParam(C.Structure):
    _fields_ = [("kind", C.c_int), ("rank", C.c_int), ("U", C.c_void_p), ("W", C.c_void_p),
                ("s", C.c_void_p), ("G", C.c_void_p), ("c0", Complex), ("c1", Complex), ("c2", Complex)]


class KernelTime(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("ms", C.c_float), ("items", C.c_longlong),
                ("flops", C.c_double), ("bytes", C.c_double)]


class RomDesc(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("r", C.c_int), ("F", C.c_int), ("ldk", C.c_int),
        ("K", C.c_void_p), ("M", C.c_void_p), ("D", C.c_void_p),
        ("eta", C.c_double),
        ("rhs", C.c_void_p), ("ldb", C.c_int),
        ("omega", C.c_void_p),
        ("X", C.c_void_p), ("info", C.c_void_p), ("steps", C.c_void_p), ("berr", C.c_void_p),
        ("LU", C.c_void_p), ("ipiv", C.c_void_p),
        ("n_out", C.c_int), ("ldc", C.c_int), ("C", C.c_void_p), ("Y", C.c_void_p),
    ]


class SweepOpts(C.Structure):
    _fields_ = [("precision", C.c_int), ("max_refine", C.c_int), ("tol", C.c_double),
                ("flags", C.c_int)]


class SromError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"srom status {status}: {msg}")
        self.status = status


_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: run staccato_b200/build.py (or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        vp, i, pp = C.c_void_p, C.c_int, C.POINTER(C.c_void_p)
        L.srom_create.argtypes = [pp, i]
        L.srom_create.restype = i
        L.srom_destroy.argtypes = [vp]
        L.srom_destroy.restype = i
        L.srom_set_stream.argtypes = [vp, vp]
        L.srom_set_stream.restype = i
        L.srom_status_string.argtypes = [i]
        L.srom_status_string.restype = C.c_char_p
        L.srom_last_error.argtypes = [vp]
        L.srom_last_error.restype = C.c_char_p
        L.srom_version.restype = i
        L.srom_profile_enable.argtypes = [vp, i]
        L.srom_profile_enable.restype = i
        L.srom_profile_read.argtypes = [vp, C.POINTER(KernelTime), i, C.POINTER(C.c_int)]
        L.srom_profile_read.restype = i
        L.srom_project_real.argtypes = [vp, C.c_int64, vp, vp, i, i, C.POINTER(C.c_void_p), i, vp, i,
                                        C.c_int64, C.POINTER(C.c_void_p)]
        L.srom_project_real.restype = i
        L.srom_project_complex.argtypes = [vp, C.c_int64, C.c_int64, vp, vp, i, i, C.POINTER(C.c_void_p), i, vp, i,
                                           C.c_int64, vp, C.c_int64, C.POINTER(C.c_void_p)]
        L.srom_project_complex.restype = i
        L.srom_krylov_basis.argtypes = [vp, C.c_int64, C.c_int64, vp, vp, i, i, vp, vp, vp, vp, i, C.c_int64, vp, i, i,
                                        C.c_double, vp, C.c_int64, i, C.POINTER(i)]
        L.srom_krylov_basis.restype = i
        L.srom_fom_sweep.argtypes = [vp, C.c_int64, C.c_int64, vp, vp, i, i, vp, vp, vp, vp, i, C.c_int64, vp, i, vp,
                                     C.c_int64]
        L.srom_fom_sweep.restype = i
        L.srom_band_order.argtypes = [C.c_int64, C.c_int64, vp, vp, i, i, vp, C.POINTER(C.c_int64),
                                      C.POINTER(C.c_int64), C.c_char_p, i]
        L.srom_band_order.restype = i
        L.srom_zgemm_batched.argtypes = [vp, i, i, i, i, i, Complex, vp, C.c_int64, C.c_int64, vp, C.c_int64,
                                         C.c_int64, Complex, vp, C.c_int64, C.c_int64, i]
        L.srom_zgemm_batched.restype = i
        L.srom_band_pivot_report.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_double)]
        L.srom_band_pivot_report.restype = i
        L.srom_band_cache_report.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.srom_band_cache_report.restype = i
        L.srom_band_cache_release.argtypes = [vp]
        L.srom_band_cache_release.restype = i
        L.srom_orthonormalize.argtypes = [vp, vp, C.c_int64, i, C.c_int64, i]
        L.srom_orthonormalize.restype = i
        L.srom_graph_create.argtypes = [vp, C.POINTER(RomDesc), i, C.POINTER(SweepOpts), pp]
        L.srom_graph_create.restype = i
        L.srom_graph_launch.argtypes = [vp, vp]
        L.srom_graph_launch.restype = i
        L.srom_graph_destroy.argtypes = [vp]
        L.srom_graph_destroy.restype = i
        L.srom_tune.argtypes = [vp, C.POINTER(C.c_int), i, i, C.c_char_p]
        L.srom_tune.restype = i
        L.srom_sweep_backward.argtypes = [vp, C.POINTER(RomDesc), vp, i, C.POINTER(DParam), i, vp, vp]
        L.srom_sweep_backward.restype = i
        L.srom_sweep_fp64_noalloc.argtypes = [C.POINTER(RomDesc), vp, C.c_char_p, i]
        L.srom_sweep_fp64_noalloc.restype = i
        i64, cp = C.c_int64, C.c_char_p
        L.srom_mtx_read_dense.argtypes = [cp, C.POINTER(i64), C.POINTER(i64), vp, i64, cp, i]
        L.srom_mtx_read_dense.restype = i
        L.srom_mtx_write_dense.argtypes = [cp, i64, i64, vp, i64, cp, i]
        L.srom_mtx_write_dense.restype = i
        L.srom_write_solution.argtypes = [cp, vp, i64, cp, i]
        L.srom_write_solution.restype = i
        for name in ("srom_sweep", "srom_sweep_host"):
            fn = getattr(L, name)
            fn.argtypes = [vp, C.POINTER(RomDesc), i, C.POINTER(SweepOpts)]
            fn.restype = i
        _lib = L
    return _lib


def check(handle, status: int) -> None:
    if status != SROM_OK:
        L = lib()
        msg = L.srom_last_error(handle) if handle else None
        txt = (msg.decode() if msg else "") or L.srom_status_string(status).decode()
        raise SromError(status, txt)


class Handle:
    """Owns one ``srom_handle`` bound to a device (and optionally a CUDA stream)."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        st = lib().srom_create(C.byref(self._h), device)
        if st != SROM_OK:
            raise SromError(st, f"srom_create(device={device}) failed")
        self.device = device

    @property
    def ptr(self):
        return self._h

    def set_stream(self, stream_ptr: int) -> None:
        check(self._h, lib().srom_set_stream(self._h, C.c_void_p(stream_ptr)))

    def profile(self, enable: bool = True) -> None:
        check(self._h, lib().srom_profile_enable(self._h, int(enable)))

    def read_profile(self, max_records: int = 4096):
        """List of (name, ms, items, flops, bytes) for the launches since the last read."""
        buf = (KernelTime * max_records)()
        cnt = C.c_int()
        check(self._h, lib().srom_profile_read(self._h, buf, max_records, C.byref(cnt)))
        return [(buf[k].name.decode(), buf[k].ms, buf[k].items, buf[k].flops, buf[k].bytes)
                for k in range(min(cnt.value, max_records))], cnt.value

    def close(self) -> None:
        if self._h:
            lib().srom_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass
