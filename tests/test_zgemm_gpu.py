"""Batched complex GEMM (srom_zgemm_batched, FP64 tensor cores) against numpy.

The kernel stands in for cuBLAS ZGEMM in the band solver (trailing updates, solve updates,
re-orthogonalisation) and for the batched products of the substructure coupling; tolerance
1e-13 of |alpha| ||op(A)|| ||op(B)|| + |beta| ||C|| per entry (FP64 rounding of k-term sums).
"""
import numpy as np
import pytest

from staccato_b200 import _capi
from staccato_b200.linalg import OP_C, OP_N, OP_T, zgemm

pytestmark = pytest.mark.gpu


def _c(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def _op(X, op):
    return X if op == OP_N else (X.T if op == OP_T else X.conj().T)


def _colmajor_dev(mats, ld):
    """Stack column-major matrices (rows <= ld) into one device buffer of stride ld * cols."""
    import torch

    rows, cols = mats[0].shape
    buf = np.full((len(mats), cols, ld), np.nan + 1j * np.nan)
    for b, Mx in enumerate(mats):
        buf[b, :, :rows] = Mx.T
    return torch.from_numpy(buf).cuda()


def _back(t, rows, cols, ld):
    a = t.cpu().numpy().reshape(-1, cols, ld)
    return [a[b, :, :rows].T for b in range(a.shape[0])]


@pytest.mark.parametrize("opa,opb", [(OP_N, OP_N), (OP_N, OP_T), (OP_T, OP_N), (OP_C, OP_N), (OP_N, OP_C),
                                     (OP_T, OP_T), (OP_C, OP_C)])
@pytest.mark.parametrize("m,n,k,batch", [(1, 1, 1, 1), (64, 64, 64, 3), (100, 37, 70, 2), (129, 65, 9, 1)])
def test_zgemm_ops_shapes(handle, opa, opb, m, n, k, batch):
    rng = np.random.default_rng(m * 7 + n + k + opa * 3 + opb)
    ar, ac = (m, k) if opa == OP_N else (k, m)
    br, bc = (k, n) if opb == OP_N else (n, k)
    A = [_c(rng, (ar, ac)) for _ in range(batch)]
    B = [_c(rng, (br, bc)) for _ in range(batch)]
    Cm = [_c(rng, (m, n)) for _ in range(batch)]
    lda, ldb, ldc = ar + 3, br + 1, m + 2
    dA, dB, dC = _colmajor_dev(A, lda), _colmajor_dev(B, ldb), _colmajor_dev(Cm, ldc)
    alpha, beta = 0.7 - 0.2j, -1.1 + 0.4j
    zgemm(handle, opa, opb, m, n, k, dA, lda, lda * ac, dB, ldb, ldb * bc, dC, ldc, ldc * n, batch=batch,
          alpha=alpha, beta=beta)
    got = _back(dC, m, n, ldc)
    for b in range(batch):
        ref = alpha * _op(A[b], opa) @ _op(B[b], opb) + beta * Cm[b]
        scale = abs(alpha) * np.abs(A[b]).max() * np.abs(B[b]).max() * k + abs(beta) * np.abs(Cm[b]).max()
        assert np.abs(got[b] - ref).max() <= 1e-13 * scale
        # the padding rows of C are left untouched
    raw = dC.cpu().numpy().reshape(batch, n, ldc)
    assert np.isnan(raw[:, :, m:]).all()


def test_zgemm_split_k_and_beta_zero(handle):
    """A short, wide product (k = 6000, one tile): the k range is split over CTAs
    and the partials reduced in order; beta = 0 must not read C (NaN there)."""
    import torch

    rng = np.random.default_rng(5)
    m, n, k = 40, 8, 6000
    A = _c(rng, (k, m))  # used as A^H
    B = _c(rng, (k, n))
    dA, dB = _colmajor_dev([A], k), _colmajor_dev([B], k)
    dC = torch.full((n * m,), complex(np.nan, np.nan), dtype=torch.complex128, device="cuda")
    zgemm(handle, OP_C, OP_N, m, n, k, dA, k, 0, dB, k, 0, dC, m, 0)
    got = dC.cpu().numpy().reshape(n, m).T
    ref = A.conj().T @ B
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(A).max() * np.abs(B).max() * k
    # deterministic: the same call gives the same bits
    dC2 = torch.empty_like(dC)
    zgemm(handle, OP_C, OP_N, m, n, k, dA, k, 0, dB, k, 0, dC2, m, 0)
    assert torch.equal(dC.view(torch.float64), dC2.view(torch.float64))


def test_zgemm_broadcast_operand(handle):
    """stride 0 broadcasts one A over the batch (the coupling's dR/dY)."""
    rng = np.random.default_rng(9)
    m, n, k, batch = 12, 5, 7, 6
    A = _c(rng, (m, k))
    B = [_c(rng, (k, n)) for _ in range(batch)]
    dA, dB = _colmajor_dev([A], m), _colmajor_dev(B, k)
    dC = _colmajor_dev([np.zeros((m, n))] * batch, m)
    zgemm(handle, OP_N, OP_N, m, n, k, dA, m, 0, dB, k, k * n, dC, m, m * n, batch=batch)
    got = _back(dC, m, n, m)
    for b in range(batch):
        assert np.abs(got[b] - A @ B[b]).max() <= 1e-13 * np.abs(A).max() * np.abs(B[b]).max() * k


def test_zgemm_invalid_arguments(handle):
    import torch

    x = torch.zeros(64, dtype=torch.complex128, device="cuda")
    with pytest.raises(_capi.SromError) as e:
        zgemm(handle, OP_N, OP_N, 8, 8, 8, x, 4, 0, x, 8, 0, x, 8, 0)  # lda < m
    assert e.value.status == _capi.SROM_ERR_INVALID
    with pytest.raises(_capi.SromError) as e:
        zgemm(handle, 3, OP_N, 2, 2, 2, x, 2, 0, x, 2, 0, x, 2, 0)
    assert e.value.status == _capi.SROM_ERR_INVALID
