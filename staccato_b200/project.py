"""Projection of sparse FE operators onto a basis, and FP64 Gram-Schmidt, through the C ABI.

``project(handle, csr, values, V)`` returns ``[V^T A_m V for each A_m]`` for matrices that
share one CSR pattern (``srom_project_real``); ``orthonormalize(handle, V)`` orthonormalises
the columns of V in place (``srom_orthonormalize``).  All arrays are torch CUDA tensors.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import List, Sequence

from . import _capi
from ._capi import check


@dataclasses.dataclass
class DeviceCsr:
    """CSR pattern in device memory (int64 row pointers, int32 column indices)."""

    n_rows: int
    rowptr: "object"
    colind: "object"
    base: int = 0
    upper: bool = False

    @classmethod
    def from_host(cls, indptr, indices, base: int = 0, upper: bool = False, device="cuda"):
        import numpy as np
        import torch

        rp = torch.from_numpy(np.ascontiguousarray(indptr, dtype=np.int64)).to(device)
        ci = torch.from_numpy(np.ascontiguousarray(indices, dtype=np.int32)).to(device)
        return cls(n_rows=len(indptr) - 1, rowptr=rp, colind=ci, base=base, upper=upper)


def _on_device(*tensors) -> None:
    """The C ABI takes device pointers: refuse host tensors before anything is launched."""
    for t in tensors:
        if not getattr(t, "is_cuda", False):
            raise ValueError("expected CUDA tensors (the C ABI takes device pointers)")


def project(handle: _capi.Handle, csr: DeviceCsr, values: Sequence, V) -> List:
    """R_m = V^T A_m V (k x k, returned as torch float64 tensors in column-major order).

    V: torch float64 tensor holding an n_rows x k column-major basis, i.e. a (k, n_rows)
    row-major tensor (``V_cm``) or a Fortran-ordered view; pass it via ``basis_colmajor``.
    """
    import torch

    Vt = V  # (k, n_rows) row-major == n_rows x k column-major
    k, n = int(Vt.shape[0]), int(Vt.shape[1])
    assert n == csr.n_rows and Vt.is_contiguous() and Vt.dtype == torch.float64
    _on_device(Vt, *values)
    outs = [torch.empty((k, k), dtype=torch.float64, device=Vt.device) for _ in values]
    vals = (C.c_void_p * len(values))(*[C.c_void_p(v.data_ptr()) for v in values])
    rs = (C.c_void_p * len(values))(*[C.c_void_p(o.data_ptr()) for o in outs])
    check(handle.ptr, _capi.lib().srom_project_real(
        handle.ptr, csr.n_rows, C.c_void_p(csr.rowptr.data_ptr()), C.c_void_p(csr.colind.data_ptr()),
        csr.base, int(csr.upper), vals, len(values), C.c_void_p(Vt.data_ptr()), k, n, rs))
    # each output holds a column-major k x k matrix: transpose the row-major view
    return [o.t() for o in outs]


def project_complex(handle: _capi.Handle, csr: DeviceCsr, values: Sequence, V, Z=None) -> List:
    """R_m = Z^H A_m V (Z = V by default) for complex values sharing one CSR pattern
    (``srom_project_complex``, k <= 2048).  values: complex128 tensors (nnz each); V, Z:
    contiguous (k, n_rows) complex128 tensors = n_rows x k column-major bases.  Returns k x k
    complex128 tensors."""
    import torch

    k, n = int(V.shape[0]), int(V.shape[1])
    assert n == csr.n_rows and V.is_contiguous() and V.dtype == torch.complex128
    _on_device(V, *values, *((Z,) if Z is not None else ()))
    if Z is not None:
        assert tuple(Z.shape) == (k, n) and Z.is_contiguous() and Z.dtype == torch.complex128
    nnz = int(values[0].numel())
    outs = [torch.empty((k, k), dtype=torch.complex128, device=V.device) for _ in values]
    vals = (C.c_void_p * len(values))(*[C.c_void_p(v.data_ptr()) for v in values])
    rs = (C.c_void_p * len(values))(*[C.c_void_p(o.data_ptr()) for o in outs])
    check(handle.ptr, _capi.lib().srom_project_complex(
        handle.ptr, csr.n_rows, nnz, C.c_void_p(csr.rowptr.data_ptr()), C.c_void_p(csr.colind.data_ptr()),
        csr.base, int(csr.upper), vals, len(values), C.c_void_p(V.data_ptr()), k, n,
        None if Z is None else C.c_void_p(Z.data_ptr()), n, rs))
    return [o.t() for o in outs]


def orthonormalize(handle: _capi.Handle, V, passes: int = 2) -> None:
    """In-place block Gram-Schmidt (``passes`` projection passes per 32-column panel) of an
    n x k column-major basis given as a contiguous (k, n) float64 tensor."""
    _on_device(V)
    k, n = int(V.shape[0]), int(V.shape[1])
    check(handle.ptr, _capi.lib().srom_orthonormalize(handle.ptr, C.c_void_p(V.data_ptr()), n, k, n, passes))
