"""Known-answer cases on the GPU, independent of the oracle: diagonal ROMs solved in closed
form, their rotations by an orthogonal Q (x = Q * diagonal solution), hand cases for n = 1 and
a row swap, and projections onto permuted identity columns."""
import numpy as np
import pytest
import scipy.sparse as sp

from staccato_b200 import _capi
from staccato_b200.project import DeviceCsr, project
from staccato_b200.sweep import DeviceRom, sweep

pytestmark = pytest.mark.gpu

# the mixed form with every system in the mixed kernel (small ones included)
FORMS = [(_capi.SROM_FP64, 0),
         (_capi.SROM_MIXED_FP32, _capi.SROM_FLAG_FALLBACK_FP64 | _capi.SROM_FLAG_MIXED_EVERY)]


def _run(handle, K, M, rhs, omega, eta, form):
    import torch

    rom = DeviceRom.from_host(K, M, None, rhs, omega, eta=eta)
    sweep(handle, [rom], precision=form[0], flags=form[1])
    torch.cuda.synchronize()
    return rom.solutions(), rom.info.cpu().numpy()


def _rel(X, ref):
    X, ref = np.asarray(X), np.asarray(ref)
    num = np.linalg.norm((X - ref).reshape(len(X), -1), axis=1)
    return num / np.linalg.norm(ref.reshape(len(X), -1), axis=1)


@pytest.mark.parametrize("form", FORMS, ids=["fp64", "mixed"])
@pytest.mark.parametrize("n", [7, 64, 300])
def test_diagonal_rom_closed_form(handle, form, n):
    rng = np.random.default_rng(n)
    k = (2 * np.pi * np.exp(rng.uniform(np.log(20), np.log(2000), n))) ** 2
    m = rng.uniform(0.5, 2.0, n)
    eta = 0.02
    f = rng.standard_normal((n, 2)) + 1j * rng.standard_normal((n, 2))
    omega = 2 * np.pi * np.linspace(1.0, 1000.0, 23)
    X, info = _run(handle, np.diag(k).astype(complex), np.diag(m).astype(complex), f, omega, eta, form)
    ref = f[None, :, :] / (k[None, :, None] * (1 + 1j * eta) - omega[:, None, None] ** 2 * m[None, :, None])
    assert (info == 0).all()
    assert _rel(X, ref).max() <= (1e-15 if form[0] == _capi.SROM_FP64 else 1e-10)


@pytest.mark.parametrize("form", FORMS, ids=["fp64", "mixed"])
def test_rotated_diagonal_rom(handle, form):
    n = 96
    rng = np.random.default_rng(5)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    k = (2 * np.pi * np.exp(rng.uniform(np.log(20), np.log(2000), n))) ** 2
    m = rng.uniform(0.5, 2.0, n)
    eta = 0.02
    K = (Q * k) @ Q.T
    M = (Q * m) @ Q.T
    f = rng.standard_normal((n, 1)) + 0j
    omega = 2 * np.pi * np.linspace(5.0, 900.0, 17)
    X, info = _run(handle, K.astype(complex), M.astype(complex), f, omega, eta, form)
    g = Q.T @ f
    ref = np.einsum("ij,fjc->fic", Q, g[None] / (k[None, :, None] * (1 + 1j * eta) - omega[:, None, None] ** 2 * m[None, :, None]))
    assert (info == 0).all()
    # K and M are rounded once when formed, so the bound is relative to the conditioning
    assert _rel(X, ref).max() <= 1e-9


def test_hand_cases(handle):
    X, info = _run(handle, np.array([[4.0 + 1j]]), np.array([[2.0 + 0j]]), np.array([[3.0 + 0j]]), [1.0], 0.0,
                   FORMS[0])
    assert info[0] == 0 and X[0, 0, 0] == 3.0 / (4.0 + 1j - 2.0)
    # a zero leading entry forces a row swap: A = [[0, 1], [2, 3]] at w = 0
    K = np.array([[0.0, 1.0], [2.0, 3.0]], dtype=complex)
    X, info = _run(handle, K, np.zeros((2, 2), complex), np.array([[1.0], [2.0]], complex), [0.0], 0.0, FORMS[0])
    assert info[0] == 0 and np.allclose(X[0, :, 0], [-0.5, 1.0], rtol=0, atol=1e-15)


def test_projection_onto_permuted_columns(handle):
    """V = columns of the identity in a permuted order: R = V^T A V picks those rows and
    columns of A exactly (one nonzero product per entry)."""
    import torch

    n, k = 500, 40
    rng = np.random.default_rng(2)
    A = sp.random(n, n, density=0.04, random_state=3, format="csr")
    A = (A + A.T + sp.eye(n)).tocsr()
    A.sort_indices()
    cols = rng.permutation(n)[:k]
    V = np.zeros((n, k))
    V[cols, np.arange(k)] = 1.0
    csr = DeviceCsr.from_host(A.indptr, A.indices)
    (R,) = project(handle, csr, [torch.from_numpy(A.data).cuda()],
                   torch.from_numpy(np.ascontiguousarray(V.T)).cuda())
    assert np.array_equal(R.cpu().numpy(), A.toarray()[np.ix_(cols, cols)])
