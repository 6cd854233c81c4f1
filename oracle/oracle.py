"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference arm import
this module, and only to check or to time the CPU restatement; the product path never does.

Every function here wraps ``oracle/srom_oracle.c`` (see its header for the reference lines it
restates: assembly src/analysis/KrylovROMSubstructure.cpp:1411-1420, zgetrf/zgetrs :1428-1430,
projection src/tools/MathLibrary.cpp:177-234 and :491-532) or ``oracle/cpu_baseline.c``
(srcPerformanceTest/main.cpp:359-404).
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "build")

_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_I64 = C.c_int64


def build() -> None:
    """Compile liboracle.so and libcpu_baseline.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load(name: str) -> C.CDLL:
    path = os.path.join(BUILD, name)
    if not os.path.exists(path):
        build()
    return C.CDLL(path)


_lib: Optional[C.CDLL] = None
_cpu: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        L = _load("liboracle.so")
        L.oracle_assemble.argtypes = [_I, _P, _P, _P, _D, _D, _P]
        L.oracle_zgetrf.argtypes = [_I, _P, _I, _P]
        L.oracle_zgetrf.restype = _I
        L.oracle_zgetrs.argtypes = [_I, _I, _P, _I, _P, _P, _I]
        L.oracle_zgetrs_conj.argtypes = [_I, _I, _P, _I, _P, _P, _I]
        L.oracle_sweep.argtypes = [_I, _I, _P, _P, _P, _D, _P, _I, _I, _P, _P, _P]
        L.oracle_refine_ld.argtypes = [_I, _I, _P, _P, _I, _I, _P]
        L.oracle_refine_ld.restype = _I
        L.oracle_csr_spmm.argtypes = [_I, _P, _P, _P, _I, _I, _P, _I, _I64, _P]
        L.oracle_gemm_tn.argtypes = [_I, _I, _P, _I64, _P, _P]
        L.oracle_mgs.argtypes = [_I, _I, _P, _I64, _I]
        L.oracle_backproject.argtypes = [_I, _I, _I, _I, _I, _P, _P, _P]
        _lib = L
    return _lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _cf(a) -> np.ndarray:
    return np.asfortranarray(np.asarray(a, dtype=np.complex128))


def assemble(K, M, D, eta: float, omega: float) -> np.ndarray:
    """A(w) in the reference's zaxpy order, bit-identical to the GPU assembly."""
    K = _cf(K)
    M = None if M is None else _cf(M)
    D = None if D is None else _cf(D)
    n = K.shape[0]
    A = np.empty((n, n), dtype=np.complex128, order="F")
    lib().oracle_assemble(n, _ptr(K), _ptr(M), _ptr(D), float(eta), float(omega), _ptr(A))
    return A


def zgetrf(A):
    """LAPACK-style partial-pivot LU: returns (LU, ipiv 1-based, info)."""
    LU = _cf(A).copy(order="F")
    n = LU.shape[0]
    ipiv = np.zeros(max(n, 1), dtype=np.int32)
    info = lib().oracle_zgetrf(n, _ptr(LU), n, _ptr(ipiv))
    return LU, ipiv[:n], info


def zgetrs(LU, ipiv, B, conj: bool = False) -> np.ndarray:
    B2 = _cf(B)
    if B2.ndim == 1:
        B2 = B2[:, None]
    X = B2.copy(order="F")
    n = LU.shape[0]
    ip = np.ascontiguousarray(ipiv, dtype=np.int32)
    fn = lib().oracle_zgetrs_conj if conj else lib().oracle_zgetrs
    fn(n, X.shape[1], _ptr(LU), n, _ptr(ip), _ptr(X), n)
    return X


def sweep(K, M, D, eta: float, rhs, omega):
    """Reference sequence for every frequency: X[f] (n x r) and info[f]."""
    K = _cf(K)
    M = None if M is None else _cf(M)
    D = None if D is None else _cf(D)
    rhs = _cf(rhs)
    if rhs.ndim == 1:
        rhs = rhs[:, None]
    omega = np.ascontiguousarray(omega, dtype=np.float64)
    n, r = rhs.shape
    F = omega.shape[0]
    X = np.zeros((F, r, n), dtype=np.complex128)  # per frequency: n x r column-major
    info = np.zeros(F, dtype=np.int32)
    lib().oracle_sweep(n, r, _ptr(K), _ptr(M), _ptr(D), float(eta), _ptr(rhs), n, F,
                       _ptr(omega), _ptr(X), _ptr(info))
    return np.ascontiguousarray(X.transpose(0, 2, 1)), info


def x_ref(K, M, D, eta: float, rhs, omega, iters: int = 3):
    """High-accuracy solutions of the FP64-assembled systems (long-double residuals)."""
    rhs = _cf(rhs)
    if rhs.ndim == 1:
        rhs = rhs[:, None]
    n, r = rhs.shape
    omega = np.atleast_1d(np.asarray(omega, dtype=np.float64))
    out = np.zeros((omega.shape[0], n, r), dtype=np.complex128)
    for f, w in enumerate(omega):
        A = assemble(K, M, D, eta, w)
        X = np.zeros((n, r), dtype=np.complex128, order="F")
        lib().oracle_refine_ld(n, r, _ptr(A), _ptr(rhs), n, iters, _ptr(X))
        out[f] = X
    return out


def backproject(C, X) -> np.ndarray:
    """Y[f] = C X[f] for X of shape (F, n, r): returns (F, n_out, r), summed over j in
    increasing order with the GPU kernel's FMA pattern."""
    C = _cf(C)
    X = np.asarray(X, dtype=np.complex128)
    F, n, r = X.shape
    n_out = C.shape[0]
    Xc = np.ascontiguousarray(X.transpose(0, 2, 1))  # (F, r, n): blocks of n x r, ld n
    Y = np.empty((F, r, n_out), dtype=np.complex128)
    lib().oracle_backproject(n, r, F, n_out, n_out, _ptr(C), _ptr(Xc), _ptr(Y))
    return np.ascontiguousarray(Y.transpose(0, 2, 1))


def rel_err(X, Xref) -> np.ndarray:
    """Per-frequency ||x - x_ref||_2 / ||x_ref||_2 over all RHS columns."""
    X = np.asarray(X).reshape(Xref.shape[0], -1)
    R = np.asarray(Xref).reshape(Xref.shape[0], -1)
    return np.linalg.norm(X - R, axis=1) / np.linalg.norm(R, axis=1)


# ------------------------------------------------------------------ projection

def csr_spmm(indptr, indices, data, V, upper: bool = False, base: int = 0) -> np.ndarray:
    V = np.asfortranarray(V, dtype=np.float64)
    n_rows, k = V.shape
    Y = np.zeros((n_rows, k), dtype=np.float64, order="F")
    ip = np.ascontiguousarray(indptr, dtype=np.int64)
    ix = np.ascontiguousarray(indices, dtype=np.int32)
    dv = np.ascontiguousarray(data, dtype=np.float64)
    lib().oracle_csr_spmm(n_rows, _ptr(ip), _ptr(ix), _ptr(dv), base, int(upper), _ptr(V), k,
                          n_rows, _ptr(Y))
    return Y


def gemm_tn(V, Y) -> np.ndarray:
    V = np.asfortranarray(V, dtype=np.float64)
    Y = np.asfortranarray(Y, dtype=np.float64)
    n_rows, k = V.shape
    R = np.zeros((k, k), dtype=np.float64, order="F")
    lib().oracle_gemm_tn(n_rows, k, _ptr(V), n_rows, _ptr(Y), _ptr(R))
    return R


def project(indptr, indices, data, V, upper: bool = False, base: int = 0) -> np.ndarray:
    """K_r = V^T (K V): SpMM then GEMM, as generateROM does for each FE matrix."""
    return gemm_tn(V, csr_spmm(indptr, indices, data, V, upper, base))


def mgs(V, passes: int = 2) -> np.ndarray:
    V = np.array(V, dtype=np.float64, order="F", copy=True)
    N, k = V.shape
    lib().oracle_mgs(N, k, _ptr(V), N, passes)
    return V


# ------------------------------------------------------------------ adjoint

def adjoint_gradient(K, M, D, eta: float, rhs, omega, gbar, dA_terms):
    """FP64 CPU adjoint.

    For each frequency: x = A^-1 b, A^H lam = gbar[f], dJ/dp_j += -Re(lam^H dA_j(w) x).
    ``gbar[f]`` is the cotangent 2 dJ/d conj(x) (n x r).  ``dA_terms(j, w)`` returns the dense
    complex derivative matrix dA/dp_j at angular frequency w.
    """
    rhs = _cf(rhs)
    if rhs.ndim == 1:
        rhs = rhs[:, None]
    P = dA_terms.count
    grad = np.zeros(P)
    for f, w in enumerate(np.asarray(omega, dtype=np.float64)):
        A = assemble(K, M, D, eta, w)
        LU, ipiv, _ = zgetrf(A)
        x = zgetrs(LU, ipiv, rhs)
        g = _cf(gbar[f]).reshape(x.shape)
        lam = zgetrs(LU, ipiv, g, conj=True)
        for j in range(P):
            dA = dA_terms(j, w)
            grad[j] += -np.real(np.sum(np.conj(lam) * (dA @ x)))
    return grad


# ------------------------------------------------------------------ CPU baseline

def openblas_candidates():
    import numpy as _np
    import scipy as _sp
    pats = [os.path.join(os.path.dirname(_sp.__file__) + ".libs", "libscipy_openblas-*.so")]
    out = []
    for p in pats:
        out.extend(sorted(glob.glob(p)))
    return out


def cpu_lib(use_openblas: bool = True) -> C.CDLL:
    global _cpu
    if _cpu is None:
        L = _load("libcpu_baseline.so")
        L.cpu_baseline_load_lapacke.argtypes = [C.c_char_p, C.c_char_p]
        L.cpu_baseline_load_lapacke.restype = _I
        L.cpu_baseline_using_lapacke.restype = _I
        L.cpu_baseline_default_threads.restype = _I
        L.cpu_baseline_sweep.argtypes = [_I, _I, _P, _P, _P, _D, _P, _I, _P, _I, _I, _P, _I]
        L.cpu_baseline_sweep.restype = _I
        if use_openblas:
            try:
                cands = openblas_candidates()
            except Exception:
                cands = []
            for path in cands:
                if L.cpu_baseline_load_lapacke(path.encode(), b"scipy_"):
                    break
        _cpu = L
    return _cpu


def cpu_sweep(K, M, D, eta, rhs, omega, f0: int, f1: int, threads: int = 0) -> np.ndarray:
    K = _cf(K)
    M = None if M is None else _cf(M)
    D = None if D is None else _cf(D)
    rhs = _cf(rhs)
    if rhs.ndim == 1:
        rhs = rhs[:, None]
    n, r = rhs.shape
    omega = np.ascontiguousarray(omega, dtype=np.float64)
    X = np.zeros((f1 - f0, r, n), dtype=np.complex128)
    cpu_lib().cpu_baseline_sweep(n, r, _ptr(K), _ptr(M), _ptr(D), float(eta), _ptr(rhs), n,
                                 _ptr(omega), f0, f1, _ptr(X), threads)
    return np.ascontiguousarray(X.transpose(0, 2, 1))
