"""Projection R = V^T A V (SpMM + FP64 tensor-core GEMM) and Gram-Schmidt on the GPU,
against the CPU oracle (oracle/srom_oracle.c: CSR SpMM, V^T Y, modified Gram-Schmidt)."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import oracle as O
from staccato_b200 import _capi, fe_tet10
from staccato_b200.project import DeviceCsr, orthonormalize, project

pytestmark = pytest.mark.gpu


def _rand_sym_csr(n, density, seed):
    rng = np.random.default_rng(seed)
    A = sp.random(n, n, density=density, random_state=seed, format="csr")
    A = (A + A.T + sp.eye(n) * 3.0).tocsr()
    A.sort_indices()
    B = sp.random(n, n, density=density, random_state=seed + 1, format="csr")
    B = (B + B.T + sp.eye(n)).tocsr()
    # same pattern for both values: use A's pattern with B's values resampled
    Bv = rng.standard_normal(A.nnz)
    Bm = sp.csr_matrix((Bv, A.indices, A.indptr), shape=A.shape)
    Bm = ((Bm + Bm.T) * 0.5).tocsr()
    Bm = sp.csr_matrix((np.asarray(Bm[A.nonzero()]).ravel(), A.indices, A.indptr), shape=A.shape)
    return A, Bm


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


# k > 128: several SpMM passes and V^T Y windows (128 columns each), ragged last window
@pytest.mark.parametrize("k", [1, 8, 33, 96, 128, 129, 200, 300])
@pytest.mark.parametrize("base,upper", [(0, False), (1, False), (1, True)])
def test_projection_random(handle, k, base, upper):
    n = 1500
    A, B = _rand_sym_csr(n, 0.01, 7 + k)
    rng = np.random.default_rng(k)
    V = np.asfortranarray(rng.standard_normal((n, k)))
    if upper:
        Au, Bu = sp.triu(A).tocsr(), sp.triu(B).tocsr()
        Au.sort_indices()
        Bu = sp.csr_matrix((np.asarray(B[Au.nonzero()]).ravel(), Au.indices, Au.indptr), shape=A.shape)
        indptr, indices, va, vb = Au.indptr, Au.indices, Au.data, Bu.data
    else:
        indptr, indices, va, vb = A.indptr, A.indices, A.data, B.data
    csr = DeviceCsr.from_host(indptr.astype(np.int64) + base, indices.astype(np.int32) + base, base=base, upper=upper)
    Vt = _dev(np.ascontiguousarray(V.T))
    RA, RB = project(handle, csr, [_dev(va), _dev(vb)], Vt)
    refA = O.project(indptr, indices, va, V, upper=upper)
    refB = O.project(indptr, indices, vb, V, upper=upper)
    for R, ref in ((RA, refA), (RB, refB)):
        R = R.cpu().numpy()
        assert np.abs(R - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("k", [17, 96])
def test_projection_node_blocked_pattern(handle, k):
    """3x3-blocked pattern (rows of a node share their columns) with some node triples broken
    (one entry dropped) and a trailing partial node: both SpMM row paths in one matrix."""
    nn = 701
    P = sp.random(nn, nn, density=0.03, random_state=11, format="csr")
    P = (P + P.T + sp.eye(nn)).tocsr()
    A = sp.kron(P, np.ones((3, 3)), format="csr")[: 3 * nn - 1, : 3 * nn - 1].tocsr()
    A.sort_indices()
    A = A.tolil()
    rng = np.random.default_rng(5)
    for node in rng.choice(nn - 1, 40, replace=False):
        row = 3 * node + int(rng.integers(3))
        cols = A.rows[row]
        if len(cols) > 1:
            A[row, cols[-1]] = 0.0
    A = A.tocsr()
    A.eliminate_zeros()
    A.sort_indices()
    n = A.shape[0]
    va, vb = rng.standard_normal(A.nnz), rng.standard_normal(A.nnz)
    V = np.asfortranarray(rng.standard_normal((n, k)))
    csr = DeviceCsr.from_host(A.indptr, A.indices)
    RA, RB = project(handle, csr, [_dev(va), _dev(vb)], _dev(np.ascontiguousarray(V.T)))
    for R, vals in ((RA, va), (RB, vb)):
        ref = O.project(A.indptr, A.indices, vals, V)
        assert np.abs(R.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()


def test_projection_identity_basis_extracts_block(handle):
    n, k = 400, 24
    A, B = _rand_sym_csr(n, 0.05, 3)
    V = np.zeros((n, k), order="F")
    V[np.arange(k), np.arange(k)] = 1.0
    csr = DeviceCsr.from_host(A.indptr, A.indices)
    (RA,) = project(handle, csr, [_dev(A.data)], _dev(np.ascontiguousarray(V.T)))
    assert np.array_equal(RA.cpu().numpy(), A.toarray()[:k, :k])


@pytest.fixture(scope="module")
def block_model():
    return fe_tet10.clamped_block()


def test_projection_tet10_block(handle, block_model):
    m = block_model
    V = O.mgs(fe_tet10.basis(m.n_dof, 96, seed=1), passes=2)
    csr = DeviceCsr.from_host(m.indptr, m.indices)
    Kr, Mr = project(handle, csr, [_dev(m.K), _dev(m.M)], _dev(np.ascontiguousarray(V.T)))
    refK = O.project(m.indptr, m.indices, m.K, V)
    refM = O.project(m.indptr, m.indices, m.M, V)
    Kr, Mr = Kr.cpu().numpy(), Mr.cpu().numpy()
    assert np.abs(Kr - refK).max() <= 1e-12 * np.abs(refK).max()
    assert np.abs(Mr - refM).max() <= 1e-12 * np.abs(refM).max()
    # size-independent properties: symmetry and positive semi-definiteness of the projections
    assert np.abs(Kr - Kr.T).max() <= 1e-12 * np.abs(Kr).max()
    assert np.linalg.eigvalsh(0.5 * (Mr + Mr.T)).min() > 0


@pytest.mark.parametrize("n,k", [(64, 1), (1000, 17), (20000, 96)])
def test_gram_schmidt_matches_mgs(handle, n, k):
    import torch

    V0 = np.asfortranarray(np.random.default_rng(n + k).standard_normal((n, k)))
    Vt = _dev(np.ascontiguousarray(V0.T))
    orthonormalize(handle, Vt, passes=2)
    torch.cuda.synchronize()
    Vg = Vt.cpu().numpy().T
    Vo = O.mgs(V0, passes=2)
    assert np.abs(Vg - Vo).max() <= 1e-12
    assert np.abs(Vg.T @ Vg - np.eye(k)).max() <= 1e-13


def test_gram_schmidt_full_basis(handle, block_model):
    import torch

    V0 = fe_tet10.basis(block_model.n_dof, 96, seed=1)
    Vt = _dev(np.ascontiguousarray(V0.T))
    orthonormalize(handle, Vt, passes=2)
    torch.cuda.synchronize()
    Vg = Vt.cpu().numpy().T
    assert np.abs(Vg.T @ Vg - np.eye(96)).max() <= 1e-13
    Vo = O.mgs(V0, passes=2)
    assert np.abs(Vg - Vo).max() <= 1e-12


def _gs_device(handle, V0, passes=2, pad=0):
    """Run srom_orthonormalize on a column-major copy of V0 with leading dimension n + pad."""
    import ctypes as C

    import torch

    n, k = V0.shape
    buf = np.zeros((k, n + pad))
    buf[:, :n] = V0.T
    d = _dev(buf)
    check = _capi.check
    check(handle.ptr, _capi.lib().srom_orthonormalize(handle.ptr, C.c_void_p(d.data_ptr()), n, k, n + pad, passes))
    torch.cuda.synchronize()
    out = d.cpu().numpy()
    assert np.array_equal(out[:, n:], buf[:, n:])  # the padding rows are not touched
    return out[:, :n].T


@pytest.mark.parametrize("n,k,pad", [(5000, 200, 0), (3001, 40, 7)])
def test_gram_schmidt_wide_and_padded(handle, n, k, pad):
    """k > 128 takes several reduction windows per panel; ldv > n leaves the padding alone."""
    V0 = np.random.default_rng(n).standard_normal((n, k))
    Q = _gs_device(handle, V0, pad=pad)
    assert np.abs(Q.T @ Q - np.eye(k)).max() <= 1e-13
    assert np.abs(Q - O.mgs(V0, passes=2)).max() <= 1e-12


def test_gram_schmidt_ill_conditioned(handle):
    """Singular values from 1 down to 1e-6: two passes still give an orthonormal basis of the
    same nested spans (the unique Q with a positive diagonal R, like the oracle's MGS)."""
    n, k = 4000, 48
    rng = np.random.default_rng(3)
    U, _ = np.linalg.qr(rng.standard_normal((n, k)))
    W, _ = np.linalg.qr(rng.standard_normal((k, k)))
    V0 = (U * np.logspace(0, -6, k)) @ W.T
    Q = _gs_device(handle, V0)
    assert np.abs(Q.T @ Q - np.eye(k)).max() <= 1e-13
    Qo = O.mgs(V0, passes=2)
    assert np.abs(Q - Qo).max() <= 1e-8
    # V0 lies in span(Q): the projection residual is at rounding level
    assert np.linalg.norm(V0 - Q @ (Q.T @ V0)) <= 1e-12 * np.linalg.norm(V0)
