"""CPU restatement of the Krylov basis generation -- TEST INFRASTRUCTURE ONLY.

Only tests/ import this module, to check the GPU basis generation; the product path never
does.

It restates ``KrylovROMSubstructure::addKrylovModesForExpansionPoint``
(src/analysis/KrylovROMSubstructure.cpp:367-569), the block Arnoldi process with block
Gram-Schmidt re-orthogonalisation and rank-revealing deflation, per expansion point f0:

* K~ = -(K - w0^2 M + i w0 D), w0 = 2 pi f0                         (:387-399)
* Q = K~^-1 B, the first search direction                           (:405-406)
* for every expansion point after the first: Q <- Q - V (V^H Q), repeated while the
  norm ratio ||Q_new||_F / ||Q_old||_F stays <= 1/sqrt(2) ("twice is enough", :411-456)
* pivoted QR of Q (zgeqp3, :467), RR = number of leading |R_ii| > tol, counting stops at the
  first that is not (reveilRankQR_R, :796-812), Q = first RR columns of the pivoted QR's
  orthonormal factor (zungqr, :474, :477), appended to V (:487)
* Krylov orders 2..order: Q <- K~^-1 (M Q) (:495-500), re-orthogonalised against V in the
  same loop (:503-531), pivoted QR, rank, append (:543-558); no columns left ends the point.

The sparse solves use SuperLU (scipy) -- a direct solve, like the reference's PARDISO
(:571-707) -- and the QR uses LAPACK's geqp3 / ungqr through scipy, the routines the
reference calls.  The deflation tolerance is absolute (1e-8 in the reference, :378), on the
unnormalised columns, as in the reference.
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def k_tilde(K, M, D, omega: float):
    """-(K - w^2 M + i w D) as a sparse CSC matrix (KrylovROMSubstructure.cpp:387-399)."""
    A = sp.csr_matrix(K, dtype=np.complex128) - (omega * omega) * sp.csr_matrix(M, dtype=np.complex128)
    if D is not None:
        A = A + (1j * omega) * sp.csr_matrix(D, dtype=np.complex128)
    return (-A).tocsc()


def reorthogonalize(V: Optional[np.ndarray], Q: np.ndarray) -> np.ndarray:
    """Block Gram-Schmidt of Q against V, repeated until ||Q_new|| / ||Q_old|| > 1/sqrt(2)
    (KrylovROMSubstructure.cpp:424-456 and :503-531)."""
    if V is None or V.shape[1] == 0:
        return Q
    eta = 1.0 / math.sqrt(2.0)
    qk_ = Q
    for _ in range(64):  # the GPU path's cap; a zero block (ratio NaN) also ends the loop
        sk = V.conj().T @ qk_
        uk = qk_ - V @ sk
        with np.errstate(invalid="ignore", divide="ignore"):
            lim = np.linalg.norm(uk) / np.linalg.norm(qk_)
        qk_ = uk
        if not lim <= eta:
            return uk
    return qk_


def rank_revealing_q(Q: np.ndarray, tol: float):
    """(Q_RR, RR): the first RR columns of the orthonormal factor of the column-pivoted QR of Q,
    RR = leading |R_ii| > tol (KrylovROMSubstructure.cpp:467-477, :543-547, :796-812)."""
    m = Q.shape[1]
    if m == 0:
        return Q[:, :0], 0, np.zeros(0)
    Qf, R, piv = sla.qr(Q, mode="economic", pivoting=True)
    d = np.abs(np.diag(R))
    rr = 0
    for v in d:
        if v > tol:
            rr += 1
        else:
            break
    return Qf[:, :rr], rr, d


def krylov_basis(K, M, D, B: np.ndarray, exp_points_hz: Sequence[float], order: int, tol: float = 1e-8,
                 return_log: bool = False):
    """V (N x k): the basis the reference builds for the given expansion points (Hz) and Krylov
    order.  With return_log, also [(point, order, RR, |R_ii|)] per block."""
    B = np.asarray(B, dtype=np.complex128)
    N = B.shape[0]
    V = np.zeros((N, 0), dtype=np.complex128)
    log: List[tuple] = []
    Mc = sp.csr_matrix(M, dtype=np.complex128)
    for ip, f0 in enumerate(exp_points_hz):
        w = 2.0 * math.pi * float(f0)
        lu = spla.splu(k_tilde(K, M, D, w))
        Q = lu.solve(B)
        if ip > 0:
            Q = reorthogonalize(V, Q)
        Q, rr, d = rank_revealing_q(Q, tol)
        log.append((float(f0), 1, rr, d))
        if rr == 0:
            continue
        V = np.concatenate([V, Q], axis=1)
        for o in range(2, order + 1):
            Q = lu.solve(Mc @ Q)
            Q = reorthogonalize(V, Q)
            Q, rr, d = rank_revealing_q(Q, tol)
            log.append((float(f0), o, rr, d))
            if rr == 0:
                break
            V = np.concatenate([V, Q], axis=1)
    return (V, log) if return_log else V


def subspace_gap(V: np.ndarray, W: np.ndarray) -> float:
    """max over columns of W of ||w - V V^H w|| / ||w|| (V orthonormal): 0 when span W is in span V."""
    if W.shape[1] == 0:
        return 0.0
    R = W - V @ (V.conj().T @ W)
    return float(np.max(np.linalg.norm(R, axis=0) / np.linalg.norm(W, axis=0)))
