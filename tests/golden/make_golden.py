"""Generate the golden fixtures that pin the CPU oracle.

The reference ships no ROM files, golden vectors or known-answer tests for its sweep
(its test programs read .mtx files that are not part of the project), and its LAPACK
(Intel MKL) is not available here.  The fixtures therefore come from two independent
sources:
  * LAPACK zgetrf/zgetrs as shipped with scipy (OpenBLAS) -- the same LAPACK routines the
    reference calls through MKL (src/analysis/KrylovROMSubstructure.cpp:1428-1430,
    srcPerformanceTest/main.cpp:393-395): pivots must match the oracle exactly, solutions
    to rounding level;
  * closed-form solutions: diagonal K_r, M_r give x_i = b_i / (k_i (1 + i eta) - w^2 m_i),
    and an orthogonal change of basis Q keeps x = Q x_diag.
Run:  python tests/golden/make_golden.py   (writes tests/golden/sweep_golden.npz)
"""
import os

import numpy as np
import scipy.linalg as sl

HERE = os.path.dirname(os.path.abspath(__file__))


def assemble(K, M, D, eta, w):
    k = K.copy()
    if eta:
        k = (K.real - eta * K.imag) + 1j * (K.imag + eta * K.real)
    A = k + (-(w * w)) * M
    if D is not None:
        A = A + (1j * w) * D
    return A


def main():
    rng = np.random.default_rng(20261203)
    out = {}
    cases = []
    for ci, n in enumerate([1, 2, 3, 4, 7, 16, 33]):
        r = 1 + ci % 3
        K = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        M = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        D = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) if ci % 2 else None
        b = rng.standard_normal((n, r)) + 1j * rng.standard_normal((n, r))
        w = rng.uniform(0.2, 2.0, size=3)
        eta = 0.02 if ci % 3 == 0 else 0.0
        piv, X = [], []
        for wf in w:
            A = assemble(K, M, D, eta, wf)
            lu, p = sl.lu_factor(A)
            piv.append(p + 1)
            X.append(sl.lu_solve((lu, p), b))
        key = f"lapack{ci}"
        out[key + "_K"] = K
        out[key + "_M"] = M
        if D is not None:
            out[key + "_D"] = D
        out[key + "_b"] = b
        out[key + "_w"] = w
        out[key + "_eta"] = np.array(eta)
        out[key + "_ipiv"] = np.array(piv, dtype=np.int32)
        out[key + "_X"] = np.array(X)
        cases.append(key)
    # closed-form cases
    for ci, n in enumerate([5, 24]):
        k = np.exp(rng.uniform(np.log(1e2), np.log(1e6), size=n))
        m = rng.uniform(0.5, 2.0, size=n)
        eta = 0.02
        q, rr = np.linalg.qr(rng.standard_normal((n, n)))
        q = q * np.sign(np.diag(rr))
        K = (q * k) @ q.T
        M = (q * m) @ q.T
        b = rng.standard_normal((n, 1))
        w = np.sqrt(k[:3] / m[:3]) * np.array([0.9, 1.0005, 1.3])
        X = []
        for wf in w:
            xd = (q.T @ b)[:, 0] / (k * (1 + 1j * eta) - wf * wf * m)
            X.append((q @ xd)[:, None])
        key = f"exact{ci}"
        out[key + "_K"] = K.astype(np.complex128)
        out[key + "_M"] = M.astype(np.complex128)
        out[key + "_b"] = b.astype(np.complex128)
        out[key + "_w"] = w
        out[key + "_eta"] = np.array(eta)
        out[key + "_X"] = np.array(X)
        cases.append(key)
    out["cases"] = np.array(cases)
    np.savez_compressed(os.path.join(HERE, "sweep_golden.npz"), **out)
    print("wrote", len(cases), "cases")


if __name__ == "__main__":
    main()
