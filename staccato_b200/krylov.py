"""Krylov basis generation on the GPU (``srom_krylov_basis``) and the band ordering it uses
(``srom_band_order``).

Mirrors ``KrylovROMSubstructure::addKrylovModesForExpansionPoint``
(src/analysis/KrylovROMSubstructure.cpp:367-569): per expansion point the shifted matrix
K~ = -(K - w0^2 M + i w0 D) is factored (a band LDL^T on the GPU in place of PARDISO), the
search directions K~^-1 B and K~^-1 (M Q) are re-orthogonalised against the basis and reduced
by a rank-revealing pivoted QR (absolute tolerance on |R_ii|, 1e-8 by default as in the
reference), and the surviving columns are appended.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _capi
from ._capi import check
from .project import DeviceCsr, _on_device


def krylov_basis(handle: _capi.Handle, csr: DeviceCsr, K, M, D, B, exp_points_hz: Sequence[float], order: int,
                 tol: float = 1e-8, max_cols: Optional[int] = None):
    """Orthonormal basis V as a contiguous (k, n_rows) complex128 tensor (= n_rows x k
    column-major).  K, M, D (or None): complex128 device tensors of the pattern's nnz values;
    B: contiguous (n_in, n_rows) complex128 device tensor (n_rows x n_in column-major)."""
    import torch

    n = csr.n_rows
    n_in = int(B.shape[0])
    assert int(B.shape[1]) == n and B.is_contiguous() and B.dtype == torch.complex128
    for v in (K, M) + ((D,) if D is not None else ()):
        assert v.dtype == torch.complex128 and v.is_contiguous()
    _on_device(B, K, M, *((D,) if D is not None else ()), csr.rowptr, csr.colind)
    pts = np.ascontiguousarray(exp_points_hz, dtype=np.float64)
    if max_cols is None:
        max_cols = n_in * max(order, 1) * max(len(pts), 1)
    max_cols = min(max_cols, n)
    V = torch.zeros((max(max_cols, 1), n), dtype=torch.complex128, device=B.device)
    ncols = C.c_int(0)
    nnz = int(K.numel())
    check(handle.ptr, _capi.lib().srom_krylov_basis(
        handle.ptr, n, nnz, C.c_void_p(csr.rowptr.data_ptr()), C.c_void_p(csr.colind.data_ptr()), csr.base,
        int(csr.upper), C.c_void_p(K.data_ptr()), C.c_void_p(M.data_ptr()),
        None if D is None else C.c_void_p(D.data_ptr()), C.c_void_p(B.data_ptr()), n_in, n,
        pts.ctypes.data_as(C.c_void_p), len(pts), order, tol, C.c_void_p(V.data_ptr()), n, max_cols,
        C.byref(ncols)))
    return V[: ncols.value].contiguous()


def fom_sweep(handle: _capi.Handle, csr: DeviceCsr, K, M, D, F, freq_hz: Sequence[float]):
    """Full-order responses (performSolveFOM, KrylovROMSubstructure.cpp:1355-1391): X_f solving
    (K - w^2 M + i w D) X_f = F per frequency, as a (n_freq, r, n_rows) complex128 tensor (each
    [f] is n_rows x r column-major).  F: contiguous (r, n_rows) complex128 device tensor."""
    import torch

    n = csr.n_rows
    r = int(F.shape[0])
    assert int(F.shape[1]) == n and F.is_contiguous() and F.dtype == torch.complex128
    _on_device(F, K, M, *((D,) if D is not None else ()), csr.rowptr, csr.colind)
    f = np.ascontiguousarray(freq_hz, dtype=np.float64)
    X = torch.empty((len(f), r, n), dtype=torch.complex128, device=F.device)
    check(handle.ptr, _capi.lib().srom_fom_sweep(
        handle.ptr, n, int(K.numel()), C.c_void_p(csr.rowptr.data_ptr()), C.c_void_p(csr.colind.data_ptr()),
        csr.base, int(csr.upper), C.c_void_p(K.data_ptr()), C.c_void_p(M.data_ptr()),
        None if D is None else C.c_void_p(D.data_ptr()), C.c_void_p(F.data_ptr()), r, n,
        f.ctypes.data_as(C.c_void_p), len(f), C.c_void_p(X.data_ptr()), n))
    return X


def band_pivot_report(handle: _capi.Handle):
    """(factorisations, perturbed, min_pivot_ratio) of the band L D L^T factorisations of the
    handle's last krylov_basis / fom_sweep call (``srom_band_pivot_report``)."""
    nf, npert, mr = C.c_int64(0), C.c_int64(0), C.c_double(0.0)
    check(handle.ptr, _capi.lib().srom_band_pivot_report(handle.ptr, C.byref(nf), C.byref(npert), C.byref(mr)))
    return int(nf.value), int(npert.value), float(mr.value)


def band_cache_report(handle: _capi.Handle):
    """(reused, cached_rows, bandwidth): whether the handle's last krylov_basis / fom_sweep call
    reused the cached full pattern and RCM order of an earlier call on the same pattern, and the
    size of the cached pattern (``srom_band_cache_report``)."""
    ru, rows, bw = C.c_int(0), C.c_int64(0), C.c_int64(0)
    check(handle.ptr, _capi.lib().srom_band_cache_report(handle.ptr, C.byref(ru), C.byref(rows), C.byref(bw)))
    return bool(ru.value), int(rows.value), int(bw.value)


def band_cache_release(handle: _capi.Handle) -> None:
    """Free the handle's cached band pattern (``srom_band_cache_release``)."""
    check(handle.ptr, _capi.lib().srom_band_cache_release(handle.ptr))


def band_order(indptr, indices, base: int = 0, upper: bool = False):
    """(perm, bandwidth, band_bytes) of the reverse Cuthill-McKee ordering of a host CSR pattern:
    perm[k] = original row of row k."""
    rp = np.ascontiguousarray(indptr, dtype=np.int64)
    ci = np.ascontiguousarray(indices, dtype=np.int32)
    n = len(rp) - 1
    perm = np.zeros(max(n, 1), dtype=np.int32)
    bw = C.c_int64(0)
    nbytes = C.c_int64(0)
    err = C.create_string_buffer(256)
    st = _capi.lib().srom_band_order(n, int(rp[-1] - base) if n > 0 else 0, rp.ctypes.data_as(C.c_void_p),
                                     ci.ctypes.data_as(C.c_void_p), base, int(upper), perm.ctypes.data_as(C.c_void_p),
                                     C.byref(bw), C.byref(nbytes), err, 256)
    if st != _capi.SROM_OK:
        raise _capi.SromError(st, err.value.decode())
    return perm[:n], int(bw.value), int(nbytes.value)
