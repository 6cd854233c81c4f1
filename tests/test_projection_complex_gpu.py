"""Complex projection R_m = Z^H A_m V (srom_project_complex), the complex form of the
reference's generateROM, against a numpy evaluation of the same product (complex CSR, full or
upper complex-symmetric storage, one- and two-sided bases)."""
import numpy as np
import pytest
import scipy.sparse as sp

from staccato_b200 import _capi, fe_tet10
from staccato_b200.project import DeviceCsr, project_complex

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _csym(n, density, seed):
    """Complex-symmetric matrices (A^T = A) on one pattern: real part + i * another values."""
    rng = np.random.default_rng(seed)
    A = sp.random(n, n, density=density, random_state=seed, format="csr")
    A = (A + A.T + sp.eye(n) * 3.0).tocsr()
    A.sort_indices()
    vals = []
    for _ in range(2):
        re = rng.standard_normal(A.nnz)
        im = rng.standard_normal(A.nnz)
        B = sp.csr_matrix((re + 1j * im, A.indices, A.indptr), shape=A.shape)
        B = ((B + B.T) * 0.5).tocsr()
        vals.append(np.asarray(B[A.nonzero()]).ravel())
    return A, vals


# k > 64: the 2k real columns take several windows of 128
@pytest.mark.parametrize("k", [1, 13, 64, 65, 100, 150])
@pytest.mark.parametrize("base,upper,two_sided", [(0, False, False), (1, True, False), (0, False, True)])
def test_complex_projection(handle, k, base, upper, two_sided):
    n = 1200
    A, vals = _csym(n, 0.01, 5 + k)
    rng = np.random.default_rng(k)
    V = rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k))
    Z = rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k)) if two_sided else None
    if upper:
        Au = sp.triu(A).tocsr()
        Au.sort_indices()
        stored = [np.asarray(sp.csr_matrix((v, A.indices, A.indptr), shape=A.shape)[Au.nonzero()]).ravel()
                  for v in vals]
        indptr, indices = Au.indptr, Au.indices
    else:
        stored, indptr, indices = vals, A.indptr, A.indices
    csr = DeviceCsr.from_host(indptr.astype(np.int64) + base, indices.astype(np.int32) + base, base=base, upper=upper)
    Rs = project_complex(handle, csr, [_dev(v) for v in stored], _dev(V.T),
                         None if Z is None else _dev(Z.T))
    L = V if Z is None else Z
    for R, v in zip(Rs, vals):
        Am = sp.csr_matrix((v, A.indices, A.indptr), shape=A.shape)
        ref = L.conj().T @ (Am @ V)
        assert np.abs(R.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()


def test_complex_projection_tet10_hysteretic(handle):
    """The Tet10 block's K with a hysteretic factor (1 + 0.02 i) and M on a complex basis."""
    m = fe_tet10.clamped_block(4, 4, 12)
    n, k = m.n_dof, 48
    rng = np.random.default_rng(2)
    V = np.linalg.qr(rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k)))[0]
    Kc = m.K * (1 + 0.02j)
    Mc = m.M.astype(complex)
    csr = DeviceCsr.from_host(m.indptr, m.indices)
    Kr, Mr = project_complex(handle, csr, [_dev(Kc), _dev(Mc)], _dev(V.T))
    for R, v in ((Kr, Kc), (Mr, Mc)):
        Am = sp.csr_matrix((v, m.indices, m.indptr), shape=(n, n))
        ref = V.conj().T @ (Am @ V)
        assert np.abs(R.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()
    # Hermitian M projects to a Hermitian positive definite matrix
    Mh = Mr.cpu().numpy()
    assert np.abs(Mh - Mh.conj().T).max() <= 1e-12 * np.abs(Mh).max()
    assert np.linalg.eigvalsh(0.5 * (Mh + Mh.conj().T)).min() > 0


def test_complex_projection_rejects_wide_basis(handle):
    import torch

    A, vals = _csym(100, 0.05, 1)
    csr = DeviceCsr.from_host(A.indptr, A.indices)
    V = torch.zeros((2049, 100), dtype=torch.complex128, device="cuda")
    with pytest.raises(_capi.SromError) as e:
        project_complex(handle, csr, [_dev(vals[0])], V)
    assert e.value.status == _capi.SROM_ERR_UNSUPPORTED
