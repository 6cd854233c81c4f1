"""Systems without a mass term (srom_rom_desc.M = NULL) and the batched solve of given
matrices built on it (solve_batched: the getrf + getrs batches of the reference's coupling and
batched-LU programs), against the oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from staccato_b200 import _capi
from staccato_b200.sweep import DeviceRom, Graph, HostRom, solve_batched, sweep, sweep_host

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


def _c(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("n", [40, 200])
def test_sweep_without_mass_term(handle, n):
    """A(w) = (1 + i eta) K + i w D: FP64 bit-identical to the oracle, mixed within the gate;
    the host entry point accepts M = NULL too."""
    import torch

    rng = np.random.default_rng(n)
    K = _c(rng, (n, n)) + 4.0 * n ** 0.5 * np.eye(n)
    D = _c(rng, (n, n)) * 0.1
    rhs = _c(rng, (n, 2))
    omega = rng.uniform(0.5, 5.0, size=9)
    rom = DeviceRom.from_host(K, None, D, rhs, omega, eta=0.03)
    sweep(handle, [rom])
    torch.cuda.synchronize()
    Xo, info = O.sweep(K, None, D, 0.03, rhs, omega)
    assert np.array_equal(_bits(rom.solutions()), _bits(Xo)) and (info == 0).all()
    hr = HostRom(K, None, D, rhs, omega, eta=0.03)
    sweep_host(handle, [hr])
    assert np.array_equal(_bits(hr.solutions()), _bits(Xo))
    rom.X.fill_(float("nan"))
    g = Graph(handle, [rom])  # the graph owns its zero matrix
    g.launch(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    g.close()
    assert np.array_equal(_bits(rom.solutions()), _bits(Xo))
    rm = DeviceRom.from_host(K, None, D, rhs, omega, eta=0.03)
    sweep(handle, [rm], precision=_capi.SROM_MIXED_FP32, flags=_capi.SROM_FLAG_FALLBACK_FP64)
    torch.cuda.synchronize()
    assert O.rel_err(rm.solutions(), O.x_ref(K, None, D, 0.03, rhs, omega)).max() <= 1e-10


@pytest.mark.parametrize("count,n,r", [(100, 30, 1), (20, 150, 3)])
def test_solve_batched_fp64_matches_getrf_getrs(handle, count, n, r):
    rng = np.random.default_rng(count + n)
    A = _c(rng, (count, n, n))
    B = _c(rng, (count, n, r))
    X, info = solve_batched(handle, A, B)
    X = X.cpu().numpy()
    for i in range(count):
        LU, ip, inf = O.zgetrf(A[i])
        assert inf == int(info[i])
        assert np.array_equal(_bits(X[i]), _bits(O.zgetrs(LU, ip, B[i])))


def test_solve_batched_mixed_and_singular(handle):
    rng = np.random.default_rng(3)
    count, n = 40, 64
    A = _c(rng, (count, n, n)) + 3.0 * np.sqrt(n) * np.eye(n)
    B = _c(rng, (n, 2))  # one right-hand side block shared by the batch
    X, info = solve_batched(handle, A, B, precision=_capi.SROM_MIXED_FP32)
    ref = np.linalg.solve(A, np.broadcast_to(B, (count, n, 2)))
    err = np.linalg.norm((X.cpu().numpy() - ref).reshape(count, -1), axis=1) / np.linalg.norm(ref.reshape(count, -1), axis=1)
    assert err.max() <= 1e-10 and (info.cpu().numpy() == 0).all()
    S = A[:3].copy()
    S[1][:, 5] = 0.0  # exactly singular: zero column 6
    _, info = solve_batched(handle, S, B)
    assert list(info.cpu().numpy()) == [0, 6, 0]
