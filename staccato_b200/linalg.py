"""Dense complex GEMM through the library (``srom_zgemm_batched``, FP64 tensor cores).

Operands are complex128 CUDA tensors addressed by their data pointers in column-major terms:
a contiguous row-major (rows, cols) tensor is the column-major cols x rows matrix, i.e. its
transpose, with leading dimension cols.  The substructure coupling uses it for its batched
products (the reference's cublasGemmBatchedEx calls, test/IJCSA/src/IJSA.cu:875-979).
"""
from __future__ import annotations

import ctypes as C

from . import _capi
from ._capi import check

OP_N, OP_T, OP_C = _capi.SROM_OP_N, _capi.SROM_OP_T, _capi.SROM_OP_C


def _ptr(t) -> C.c_void_p:
    import torch

    assert t.dtype == torch.complex128 and t.is_cuda, "complex128 CUDA tensors expected"
    return C.c_void_p(t.data_ptr())


def zgemm(handle: _capi.Handle, opa: int, opb: int, m: int, n: int, k: int, A, lda: int, sa: int, B, ldb: int,
          sb: int, C_, ldc: int, sc: int, batch: int = 1, alpha: complex = 1.0, beta: complex = 0.0) -> None:
    """C_b = alpha op(A_b) op(B_b) + beta C_b (column-major, strides in elements; 0 broadcasts)."""
    al = _capi.Complex(complex(alpha).real, complex(alpha).imag)
    be = _capi.Complex(complex(beta).real, complex(beta).imag)
    check(handle.ptr, _capi.lib().srom_zgemm_batched(
        handle.ptr, int(opa), int(opb), int(m), int(n), int(k), al, _ptr(A), int(lda), int(sa), _ptr(B), int(ldb),
        int(sb), be, _ptr(C_), int(ldc), int(sc), int(batch)))
