"""The Krylov oracle (oracle/krylov.py) against independent dense computations, on the CPU:
its basis spans the Krylov space {K~^-1 B, (K~^-1 M) K~^-1 B, ...} of every expansion point,
is orthonormal, deflates dependent directions by the reference's rule, and the rank count stops
at the first |R_ii| <= tol."""
import math

import numpy as np
import scipy.sparse as sp

from oracle import krylov as KR


def _system(n=60, seed=0):
    rng = np.random.default_rng(seed)
    A = sp.random(n, n, density=0.08, random_state=seed)
    K = (A @ A.T + sp.eye(n) * n).tocsr()
    M = sp.diags(rng.uniform(0.5, 1.5, n)).tocsr()
    D = (0.01 * K + 0.02 * M).tocsr()
    B = rng.standard_normal((n, 2)) + 1j * rng.standard_normal((n, 2))
    return K, M, D, B


def _krylov_space(K, M, D, B, f0, order):
    w = 2 * math.pi * f0
    Kt = -(K.toarray() - w * w * M.toarray() + 1j * w * D.toarray())
    blocks = [np.linalg.solve(Kt, B)]
    for _ in range(order - 1):
        blocks.append(np.linalg.solve(Kt, M.toarray() @ blocks[-1]))
    Q, _ = np.linalg.qr(np.concatenate(blocks, axis=1))
    return Q


def test_basis_spans_the_krylov_spaces_of_every_point():
    K, M, D, B = _system()
    pts = [0.3, 1.1]
    V = KR.krylov_basis(K, M, D, B, pts, 3)
    assert V.shape[1] == 12
    assert np.abs(V.conj().T @ V - np.eye(12)).max() <= 1e-12
    for f in pts:
        W = _krylov_space(K, M, D, B, f, 3)
        assert KR.subspace_gap(V, W) <= 1e-9
    both, _ = np.linalg.qr(np.concatenate([_krylov_space(K, M, D, B, f, 3) for f in pts], axis=1))
    assert KR.subspace_gap(both, V) <= 1e-9  # and nothing outside the two spaces


def test_dependent_inputs_are_deflated():
    K, M, D, B = _system(seed=1)
    B3 = np.concatenate([B, B[:, :1] * (2 - 1j)], axis=1)  # third column parallel to the first
    V, log = KR.krylov_basis(K, M, D, B3, [0.5], 2, return_log=True)
    assert [blk[2] for blk in log] == [2, 2]
    assert V.shape[1] == 4
    assert log[0][3][2] <= 1e-8 < log[0][3][1]


def test_a_repeated_point_adds_nothing_new_beyond_rounding():
    K, M, D, B = _system(seed=2)
    V, log = KR.krylov_basis(K, M, D, B * 1e3, [0.4, 0.4], 1, tol=1e-6, return_log=True)
    assert [blk[2] for blk in log] == [2, 0]
    assert V.shape[1] == 2


def test_rank_count_stops_at_the_first_small_diagonal():
    rng = np.random.default_rng(3)
    Q, _ = np.linalg.qr(rng.standard_normal((40, 4)) + 1j * rng.standard_normal((40, 4)))
    for d, want in (([3.0, 2.0, 1e-3, 1e-12], 3), ([3.0, 1e-12, 2.0, 1.0], 3), ([1e-12] * 4, 0)):
        A = Q * np.asarray(d)  # orthogonal columns with norms d: pivoted R = diag(d) in norm order
        _, rr, rdiag = KR.rank_revealing_q(A, 1e-8)
        assert rr == want, (d, rdiag)
