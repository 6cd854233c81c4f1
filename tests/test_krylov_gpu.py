"""Krylov basis generation on the GPU (srom_krylov_basis) against the oracle's restatement of
addKrylovModesForExpansionPoint (oracle/krylov.py: SuperLU solves, LAPACK pivoted QR).

Gate: the same rank for every block (so the same number of columns), the GPU basis spanning
the oracle's to 1e-8 and vice versa, orthonormal to 1e-12; and the reduced model built on it
reproducing the full-order response near the expansion points."""
import math

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle import krylov as KR
from staccato_b200 import _capi
from staccato_b200 import fe_tet10 as T
from staccato_b200.krylov import krylov_basis
from staccato_b200.project import DeviceCsr, project_complex

pytestmark = pytest.mark.gpu


def _block(dims=(4, 4, 8), keep_clamped=False):
    """Tet10 block, clamped DOFs removed, K and M scaled to unit maximum (so that the absolute
    deflation tolerance of the reference, 1e-8, separates rank)."""
    m = T.clamped_block(*dims)
    K = sp.csr_matrix((m.K, m.indices, m.indptr), shape=(m.n_dof, m.n_dof))
    M = sp.csr_matrix((m.M, m.indices, m.indptr), shape=(m.n_dof, m.n_dof))
    if not keep_clamped:
        keep = ~m.clamped
        K, M = K[keep][:, keep].tocsr(), M[keep][:, keep].tocsr()
    K = K / abs(K).max()
    M = M / abs(M).max()
    K.sort_indices()
    M.sort_indices()
    assert np.array_equal(M.indptr, K.indptr) and np.array_equal(M.indices, K.indices)
    return K, M


def _first_f(K, M):
    return math.sqrt(spla.eigsh(K, k=1, M=M, sigma=0, which="LM")[0][0]) / (2 * math.pi)


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.complex128)).cuda()


def _inputs(N, seed=0):
    rng = np.random.default_rng(seed)
    B = np.zeros((N, 3), dtype=np.complex128)
    idx = rng.choice(N, 3, replace=False)
    B[idx, [0, 1, 2]] = 1.0
    B[:, 2] = B[:, 0]  # a dependent input: deflated by the rank test
    return B


def _upper(K, *mats):
    """Upper-triangle storage of matrices sharing K's (sorted) CSR pattern: one mask for all."""
    rows = np.repeat(np.arange(K.shape[0]), np.diff(K.indptr))
    keep = K.indices >= rows
    indptr = np.concatenate([[0], np.cumsum(np.bincount(rows[keep], minlength=K.shape[0]))])
    return indptr, K.indices[keep], [m.data[keep] for m in (K,) + mats]


def _run(handle, K, M, D, B, pts, order, upper=False, base=0):
    import torch

    mats = (M,) if D is None else (M, D)
    if upper:
        indptr, indices, data = _upper(K, *mats)
    else:
        indptr, indices, data = K.indptr, K.indices, [K.data] + [m.data for m in mats]
    csr = DeviceCsr.from_host(indptr + base, indices + base, base=base, upper=upper)
    vals = [_dev(torch, data[0]), _dev(torch, data[1])]
    dv = None if D is None else _dev(torch, data[2])
    Bt = _dev(torch, B.T)  # (n_in, N) row-major == N x n_in column-major
    V = krylov_basis(handle, csr, vals[0], vals[1], dv, Bt, pts, order)
    torch.cuda.synchronize()
    return V.cpu().numpy().T  # N x k


@pytest.fixture(scope="module")
def problem():
    K, M = _block()
    f1 = _first_f(K, M)
    D = sp.csr_matrix((0.01 * K.data + 0.001 * M.data, K.indices, K.indptr), shape=K.shape)
    return K, M, D, f1


def test_basis_matches_oracle(handle, problem):
    K, M, D, f1 = problem
    B = _inputs(K.shape[0])
    pts = [0.5 * f1, 3.0 * f1]
    Vo, log = KR.krylov_basis(K, M, D, B, pts, 4, 1e-8, return_log=True)
    V = _run(handle, K, M, D, B, pts, 4)
    assert V.shape == Vo.shape, (V.shape, Vo.shape, [l[2] for l in log])
    assert np.abs(V.conj().T @ V - np.eye(V.shape[1])).max() <= 1e-12
    assert KR.subspace_gap(V, Vo) <= 1e-8
    assert KR.subspace_gap(Vo, V) <= 1e-8


def test_without_damping_and_single_point(handle, problem):
    K, M, _, f1 = problem
    B = _inputs(K.shape[0], seed=3)[:, :2]
    Vo = KR.krylov_basis(K, M, None, B, [0.3 * f1], 3, 1e-8)
    V = _run(handle, K, M, None, B, [0.3 * f1], 3)
    assert V.shape == Vo.shape
    assert KR.subspace_gap(V, Vo) <= 1e-8 and KR.subspace_gap(Vo, V) <= 1e-8


def test_upper_storage_and_base_one(handle, problem):
    K, M, D, f1 = problem
    B = _inputs(K.shape[0], seed=5)
    pts = [0.5 * f1, 2.0 * f1]
    V0 = _run(handle, K, M, D, B, pts, 2)
    V1 = _run(handle, K, M, D, B, pts, 2, upper=True, base=1)
    assert V0.shape == V1.shape
    assert np.abs(V0 - V1).max() <= 1e-12


def test_reduced_model_reproduces_the_full_order_response(handle, problem):
    """Project K, M, D on the basis and solve the reduced model at frequencies around the
    expansion points: the reduced transfer function matches the full-order solve."""
    import torch

    K, M, D, f1 = problem
    N = K.shape[0]
    B = _inputs(N, seed=7)[:, :2]
    pts = [0.5 * f1, 2.5 * f1]
    V = _run(handle, K, M, D, B, pts, 4)
    csr = DeviceCsr.from_host(K.indptr, K.indices)
    Vt = torch.from_numpy(np.ascontiguousarray(V.T)).cuda()
    Kr, Mr, Dr = [r.cpu().numpy() for r in project_complex(
        handle, csr, [_dev(torch, K.data), _dev(torch, M.data), _dev(torch, D.data)], Vt)]
    Br = V.conj().T @ B
    for f in (0.45 * f1, 0.55 * f1, 2.4 * f1, 2.6 * f1):
        w = 2 * math.pi * f
        x_full = spla.spsolve((K - w * w * M + 1j * w * D).tocsc(), B)
        x_red = V @ np.linalg.solve(Kr - w * w * Mr + 1j * w * Dr, Br)
        err = np.linalg.norm(x_red - x_full) / np.linalg.norm(x_full)
        assert err <= 1e-6, (f / f1, err)


def test_singular_shift_and_column_limit(handle):
    import torch

    K, M = _block(keep_clamped=True)  # clamped DOFs left in: empty rows, K~ singular
    B = _inputs(K.shape[0])
    with pytest.raises(_capi.SromError) as e:
        _run(handle, K, M, None, B, [1e-4], 2)
    assert e.value.status == _capi.SROM_ERR_INVALID and "pivot" in str(e.value)
    K, M = _block()
    csr = DeviceCsr.from_host(K.indptr, K.indices)
    with pytest.raises(_capi.SromError) as e:
        krylov_basis(handle, csr, _dev(torch, K.data), _dev(torch, M.data), None,
                     _dev(torch, _inputs(K.shape[0]).T), [1e-4], 3, max_cols=2)
    assert e.value.status == _capi.SROM_ERR_INVALID and "max_cols" in str(e.value)
    # the handle still works after both errors
    V = krylov_basis(handle, csr, _dev(torch, K.data), _dev(torch, M.data), None,
                     _dev(torch, _inputs(K.shape[0]).T), [1e-4], 1)
    assert V.shape[0] == 2


def test_rom_interface_generates_basis_then_rom(handle, problem):
    """KrylovROMSubstructure mirror: basis, projection and sweep in a row; the sweep's output
    matches the full-order solve at an expansion point."""
    import torch

    from staccato_b200.rom import KrylovROMSubstructure

    K, M, D, f1 = problem
    N = K.shape[0]
    B = _inputs(N, seed=11)[:, :2]
    C = np.zeros((3, N))
    C[np.arange(3), np.random.default_rng(12).choice(N, 3, replace=False)] = 1.0
    sub = KrylovROMSubstructure(handle=handle)
    csr = DeviceCsr.from_host(K.indptr, K.indices)
    V = sub.add_krylov_modes_for_expansion_point(csr, K.data, M.data, B, [0.5 * f1], 4, D_vals=D.data)
    sub.generate_rom(csr, _dev(torch, K.data), _dev(torch, M.data), V, D_vals=_dev(torch, D.data), B=B, C=C)
    f = 0.5 * f1
    Y, info = sub.back_transform_kmor([f], np.eye(2))
    y = Y[0].cpu().numpy()
    assert (info.cpu().numpy() == 0).all()
    w = 2 * math.pi * f
    y_full = C @ spla.spsolve((K - w * w * M + 1j * w * D).tocsc(), B)
    assert np.linalg.norm(y - y_full) <= 1e-8 * np.linalg.norm(y_full)


def test_fom_sweep_matches_sparse_direct_solve(handle, problem):
    """srom_fom_sweep (performSolveFOM): each frequency's full-order solve against SuperLU,
    near resonance included, full and upper storage, with and without damping."""
    import torch

    from staccato_b200.krylov import fom_sweep

    K, M, D, f1 = problem
    N = K.shape[0]
    rng = np.random.default_rng(21)
    F = rng.standard_normal((N, 2)) + 1j * rng.standard_normal((N, 2))
    freqs = [0.0, 0.3 * f1, 0.999 * f1, 1.7 * f1, 4.0 * f1]
    for Dm, upper in ((D, False), (D, True), (None, False)):
        mats = (M,) if Dm is None else (M, Dm)
        if upper:
            indptr, indices, data = _upper(K, *mats)
        else:
            indptr, indices, data = K.indptr, K.indices, [K.data] + [m.data for m in mats]
        csr = DeviceCsr.from_host(indptr, indices, upper=upper)
        X = fom_sweep(handle, csr, _dev(torch, data[0]), _dev(torch, data[1]),
                      None if Dm is None else _dev(torch, data[2]), _dev(torch, F.T), freqs)
        X = X.cpu().numpy()
        for i, f in enumerate(freqs):
            w = 2 * math.pi * f
            A = K - w * w * M + (0 if Dm is None else 1j * w * Dm)
            ref = spla.spsolve(sp.csc_matrix(A), F)
            err = np.linalg.norm(X[i].T - ref) / np.linalg.norm(ref)
            assert err <= 1e-9, (f / f1, upper, Dm is None, err)


def test_band_small_pivot_perturbed_like_pardiso(handle):
    """A pivot below 1e-13 ||A||_inf is replaced by the value of the same phase and modulus
    1e-13 ||A||_inf (PARDISO with the reference's iparm[9] = 13) and counted; a regular
    problem perturbs nothing and reports its smallest pivot ratio."""
    import torch

    from staccato_b200.krylov import band_pivot_report, fom_sweep

    n = 300
    rng = np.random.default_rng(3)
    main = 4.0 + rng.uniform(0, 1, n) + 0.1j
    off = -1.0 + 0.05j * rng.standard_normal(n - 1)
    A = sp.diags([off, main, off], [-1, 0, 1], format="lil").astype(complex)
    # DOF 150 decoupled, with a diagonal 1e-20 of the matrix norm
    A[150, 149] = A[149, 150] = A[150, 151] = A[151, 150] = 0.0
    A[150, 150] = 1e-20 * (1 + 1j)
    A = A.tocsr()
    A.eliminate_zeros()
    A.sort_indices()
    anorm = abs(A).sum(axis=1).max()
    csr = DeviceCsr.from_host(A.indptr, A.indices)
    Kv = torch.from_numpy(A.data.astype(np.complex128)).cuda()
    Mv = torch.zeros_like(Kv)
    F = torch.ones((1, n), dtype=torch.complex128, device="cuda")
    X = fom_sweep(handle, csr, Kv, Mv, None, F, [10.0, 20.0]).cpu().numpy()
    nf, npert, ratio = band_pivot_report(handle)
    assert nf == 2 and npert == 2
    assert ratio == pytest.approx(abs(1e-20 * (1 + 1j)) / anorm, rel=1e-12)
    d = 1e-13 * anorm * (1 + 1j) / abs(1 + 1j)
    assert np.allclose(X[:, 0, 150], 1.0 / d, rtol=1e-12)
    # the rest of the solution is the exact solve of the coupled part
    keep = np.r_[0:150, 151:n]
    ref = spla.spsolve(A[keep][:, keep].tocsc(), np.ones(n - 1))
    assert np.abs(X[0, 0, keep] - ref).max() <= 1e-12 * np.abs(ref).max()
    # a regular matrix: no perturbation
    B = sp.diags([off, main, off], [-1, 0, 1], format="csr").astype(complex)
    B.sort_indices()
    csr = DeviceCsr.from_host(B.indptr, B.indices)
    Kv = torch.from_numpy(B.data.astype(np.complex128)).cuda()
    fom_sweep(handle, csr, Kv, torch.zeros_like(Kv), None, F, [10.0])
    nf, npert, ratio = band_pivot_report(handle)
    assert nf == 1 and npert == 0 and 0.0 < ratio <= 1.0


def test_pattern_cache_reuse_is_exact(problem):
    """A second call on the same pattern reuses the handle's cached full pattern and RCM order
    (srom_band_cache_report) and gives bit-identical results, the full-order sweep included; a
    different pattern of the same sizes replaces the cache and gives what a fresh handle gives;
    srom_band_cache_release frees it."""
    import torch

    from staccato_b200.krylov import band_cache_release, band_cache_report, fom_sweep

    K, M, D, f1 = problem
    N = K.shape[0]
    B = _inputs(N, seed=7)
    pts = [0.5 * f1, 2.0 * f1]
    rng = np.random.default_rng(8)
    F = rng.standard_normal((N, 2)) + 1j * rng.standard_normal((N, 2))
    freqs = [0.4 * f1, 1.3 * f1]

    def fom(h, K_, M_, D_):
        csr = DeviceCsr.from_host(K_.indptr, K_.indices)
        X = fom_sweep(h, csr, _dev(torch, K_.data), _dev(torch, M_.data), _dev(torch, D_.data), _dev(torch, F.T), freqs)
        torch.cuda.synchronize()
        return X.cpu().numpy()

    h, fresh = _capi.Handle(0), _capi.Handle(0)
    try:
        assert band_cache_report(h) == (False, 0, 0)
        V1 = _run(h, K, M, D, B, pts, 2)
        reused, rows, bw = band_cache_report(h)
        assert not reused and rows == N and bw > 0
        V2 = _run(h, K, M, D, B, pts, 2)
        assert band_cache_report(h) == (True, N, bw)
        assert np.array_equal(V1, V2)
        X1 = fom(h, K, M, D)
        assert band_cache_report(h)[0]
        assert np.array_equal(X1, fom(fresh, K, M, D))
        # the same sizes, another pattern: a symmetric permutation of the matrices
        p = rng.permutation(N)
        Kp, Mp, Dp = (A[p][:, p].tocsr() for A in (K, M, D))
        for A in (Kp, Mp, Dp):
            A.sort_indices()
        assert np.array_equal(Mp.indices, Kp.indices) and np.array_equal(Dp.indices, Kp.indices)
        assert Kp.nnz == K.nnz and not np.array_equal(Kp.indices, K.indices)
        Xp = fom(h, Kp, Mp, Dp)
        assert not band_cache_report(h)[0]
        band_cache_release(fresh)
        assert np.array_equal(Xp, fom(fresh, Kp, Mp, Dp))
        assert not band_cache_report(fresh)[0]
        band_cache_release(h)
        assert band_cache_report(h) == (False, 0, 0)
        V3 = _run(h, K, M, D, B, pts, 2)
        assert not band_cache_report(h)[0] and np.array_equal(V1, V3)
    finally:
        h.close()
        fresh.close()
