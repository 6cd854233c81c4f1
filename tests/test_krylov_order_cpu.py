"""The reverse Cuthill-McKee ordering behind srom_krylov_basis (host code, no GPU needed):
a valid permutation whose reported bandwidth is the true one, independent of storage form and
index base, and close to scipy's RCM on a scrambled mesh."""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.csgraph import reverse_cuthill_mckee

from staccato_b200 import _capi
from staccato_b200.krylov import band_order


def _grid(nx, ny, seed=None):
    A = sp.kron(sp.eye(ny), sp.diags([1.0, 4.0, 1.0], [-1, 0, 1], shape=(nx, nx))) + sp.kron(
        sp.diags([1.0, 1.0], [-1, 1], shape=(ny, ny)), sp.eye(nx))
    A = sp.csr_matrix(A)
    if seed is not None:
        p = np.random.default_rng(seed).permutation(A.shape[0])
        A = A[p][:, p].tocsr()
    A.sort_indices()
    return A


def _bandwidth(A, perm):
    ip = np.empty_like(perm)
    ip[perm] = np.arange(len(perm))
    C = A.tocoo()
    return int(np.max(np.abs(ip[C.row] - ip[C.col]))) if C.nnz else 0


def test_rcm_is_a_permutation_with_the_reported_bandwidth():
    A = _grid(30, 20, seed=1)
    perm, bw, nbytes = band_order(A.indptr, A.indices)
    assert sorted(perm.tolist()) == list(range(A.shape[0]))
    assert bw == _bandwidth(A, perm)
    assert bw <= 32  # a 30 x 20 grid: a level structure of about 20-30 nodes
    assert _bandwidth(A, reverse_cuthill_mckee(A, symmetric_mode=True)) <= 32
    assert nbytes == (A.shape[0] + 128) * (bw + 129) * 16


def test_upper_storage_and_base_one_give_the_same_order():
    A = _grid(17, 9, seed=2)
    U = sp.triu(A).tocsr()
    U.sort_indices()
    p0, bw0, _ = band_order(A.indptr, A.indices)
    p1, bw1, _ = band_order(U.indptr, U.indices, upper=True)
    p2, bw2, _ = band_order(U.indptr + 1, U.indices + 1, base=1, upper=True)
    assert bw0 == bw1 == bw2
    assert np.array_equal(p0, p1) and np.array_equal(p1, p2)


def test_disconnected_and_diagonal_patterns():
    A = sp.block_diag([_grid(5, 4), sp.eye(7), _grid(3, 3)]).tocsr()
    A.sort_indices()
    perm, bw, _ = band_order(A.indptr, A.indices)
    assert sorted(perm.tolist()) == list(range(A.shape[0])) and bw == _bandwidth(A, perm)
    D = sp.eye(9).tocsr()
    perm, bw, _ = band_order(D.indptr, D.indices)
    assert bw == 0 and sorted(perm.tolist()) == list(range(9))


def test_bad_patterns_are_rejected():
    A = _grid(4, 4)
    bad = A.indices.copy()
    bad[3] = 99
    with pytest.raises(_capi.SromError) as e:
        band_order(A.indptr, bad)
    assert e.value.status == _capi.SROM_ERR_INVALID
    rp = A.indptr.copy()
    rp[5], rp[6] = rp[6], rp[5]  # a row pointer that decreases (ends still right)
    with pytest.raises(_capi.SromError) as e:
        band_order(rp, A.indices)
    assert "rowptr" in str(e.value)
    L = sp.tril(A).tocsr()  # lower triangle passed as upper storage
    with pytest.raises(_capi.SromError):
        band_order(L.indptr, L.indices, upper=True)
