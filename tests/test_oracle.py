"""The CPU oracle, pinned against LAPACK (scipy/OpenBLAS) and closed-form solutions."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from staccato_b200 import workloads as W

GOLD = os.path.join(os.path.dirname(__file__), "golden", "sweep_golden.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def _case(g, key):
    get = lambda s: g[key + s] if key + s in g.files else None
    return (get("_K"), get("_M"), get("_D"), float(get("_eta")), get("_b"), get("_w"),
            get("_X"), get("_ipiv"))


def test_oracle_pivots_and_solutions_match_lapack(gold):
    for key in gold["cases"]:
        if not str(key).startswith("lapack"):
            continue
        K, M, D, eta, b, w, X, ipiv = _case(gold, str(key))
        Xo, info = O.sweep(K, M, D, eta, b, w)
        assert (info == 0).all()
        for f, wf in enumerate(w):
            A = O.assemble(K, M, D, eta, wf)
            _, ip, _ = O.zgetrf(A)
            assert np.array_equal(ip, ipiv[f]), key
        rel = O.rel_err(Xo, X)
        assert rel.max() < 1e-12, (key, rel.max())


def test_oracle_closed_form(gold):
    for key in gold["cases"]:
        if not str(key).startswith("exact"):
            continue
        K, M, D, eta, b, w, X, _ = _case(gold, str(key))
        Xr = O.x_ref(K, M, D, eta, b, w)
        assert O.rel_err(Xr, X).max() < 1e-9, key
        Xo, _ = O.sweep(K, M, D, eta, b, w)
        assert O.rel_err(Xo, X).max() < 1e-8, key


def test_oracle_hand_cases():
    # n = 1: x = b / (k - w^2 m)
    X, info = O.sweep(np.array([[4.0 + 1j]]), np.array([[2.0]]), None, 0.0, np.array([[3.0]]), [1.0])
    assert info[0] == 0 and np.allclose(X[0, 0, 0], 3.0 / (4.0 + 1j - 2.0), rtol=0, atol=1e-15)
    # n = 2 needing a row swap
    K = np.array([[0.0, 1.0], [2.0, 3.0]], dtype=np.complex128)
    LU, ip, info = O.zgetrf(K)
    assert list(ip) == [2, 2] and info == 0
    x = O.zgetrs(LU, ip, np.array([1.0, 2.0]))
    assert np.allclose(K @ x[:, 0], [1.0, 2.0], atol=1e-15)
    # zero column -> info = column index (1-based)
    Z = np.eye(3, dtype=np.complex128)
    Z[:, 1] = 0
    _, _, info = O.zgetrf(Z)
    assert info == 2


def test_oracle_tie_break_first_index():
    # |re|+|im| ties: IZAMAX keeps the first maximal entry
    A = np.array([[1 + 1j, 5], [2 + 0j, 7], [0 + 2j, 1]], dtype=np.complex128)
    A = np.concatenate([A, np.array([[1], [0], [3]], dtype=np.complex128)], axis=1)
    _, ip, _ = O.zgetrf(A)
    assert ip[0] == 1


def test_oracle_conj_solve():
    rng = np.random.default_rng(0)
    A = rng.standard_normal((9, 9)) + 1j * rng.standard_normal((9, 9))
    LU, ip, _ = O.zgetrf(A)
    g = rng.standard_normal((9, 2)) + 1j * rng.standard_normal((9, 2))
    lam = O.zgetrs(LU, ip, g, conj=True)
    assert np.allclose(A.conj().T @ lam, g, atol=1e-12)


def test_oracle_fp64_accuracy_on_plain_workload():
    rom = W.plain_rom()
    sel = rom.omega[::50]
    X, _ = O.sweep(rom.K, rom.M, rom.D, 0.0, rom.rhs, sel)
    Xr = O.x_ref(rom.K, rom.M, rom.D, 0.0, rom.rhs, sel)
    assert O.rel_err(X, Xr).max() < 1e-10


def test_cpu_baseline_matches_oracle():
    rom = W.plain_rom()
    Xc = O.cpu_sweep(rom.K, rom.M, rom.D, 0.0, rom.rhs, rom.omega, 0, 20, threads=2)
    Xo, _ = O.sweep(rom.K, rom.M, rom.D, 0.0, rom.rhs, rom.omega[:20])
    assert O.rel_err(Xc, Xo).max() < 1e-9


def test_oracle_no_mass_term_equals_zero_mass():
    """M = NULL leaves the mass term out; a zero M adds -0 = (-w^2)*0 to every entry, which is
    an exact identity for finite w -- the library relies on this when it gives the kernels a
    zero matrix in place of a missing M."""
    rng = np.random.default_rng(4)
    n = 12
    K = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    K[0, 1] = complex(-0.0, 0.0)
    K[2, 3] = complex(0.0, -0.0)
    D = rng.standard_normal((n, n)) * 1e-3 + 0j
    rhs = rng.standard_normal((n, 2)) + 0j
    for w in (0.0, 1.0, 37.5, 1e4):
        A0 = O.assemble(K, None, D, 0.02, w)
        Az = O.assemble(K, np.zeros((n, n), complex), D, 0.02, w)
        assert np.array_equal(np.ascontiguousarray(A0).view(np.uint64), np.ascontiguousarray(Az).view(np.uint64))
    X0, _ = O.sweep(K, None, D, 0.02, rhs, [0.0, 3.0])
    Xz, _ = O.sweep(K, np.zeros((n, n), complex), D, 0.02, rhs, [0.0, 3.0])
    assert np.array_equal(np.ascontiguousarray(X0).view(np.uint64), np.ascontiguousarray(Xz).view(np.uint64))
