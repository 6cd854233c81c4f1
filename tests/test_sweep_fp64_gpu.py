"""FP64 sweep on the GPU against the CPU oracle: bit-for-bit, through the C ABI.

The FP64 kernels restate LAPACK zgetrf/zgetrs (IZAMAX pivots, right-looking updates in
pivot-column order, the same fused multiply-adds), so their solutions, factors and pivots
must equal the oracle's exactly -- not merely within a tolerance.
"""
import numpy as np
import pytest

from oracle import oracle as O
from staccato_b200 import _capi, workloads as W
from staccato_b200.sweep import DeviceRom, HostRom, sweep, sweep_host

pytestmark = pytest.mark.gpu


def _rand_rom(rng, n, r, F, with_d=True, eta=0.0, sym=False):
    def c(shape):
        return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)

    K = c((n, n)) * 10.0 + np.eye(n) * 3.0
    M = c((n, n))
    D = c((n, n)) if with_d else None
    if sym:
        K = K + K.T
        M = M + M.T
    rhs = c((n, r))
    omega = rng.uniform(0.1, 3.0, size=F)
    return K, M, D, rhs, omega


def _assert_bitexact(a, b, what):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    assert a.shape == b.shape, what
    same = (a.view(np.uint64) == b.view(np.uint64)).reshape(a.shape[0], -1).all(axis=1)
    if not same.all():
        bad = np.flatnonzero(~same)[0]
        err = np.abs(a[bad] - b[bad]).max() / max(np.abs(b[bad]).max(), 1e-300)
        pytest.fail(f"{what}: {int((~same).sum())} of {len(same)} systems differ; first #{bad} rel {err:.3e}")


@pytest.mark.parametrize("n", [1, 2, 3, 5, 31, 32, 33, 64, 65, 100, 112, 113, 128, 200, 257, 449, 480, 512])
def test_fp64_matches_oracle_bitwise(handle, n):
    rng = np.random.default_rng(1000 + n)
    r = 1 if n > 300 else (3 if n % 2 else 8)
    F = 2 if n > 300 else 4
    K, M, D, rhs, omega = _rand_rom(rng, n, r, F, with_d=(n % 2 == 1), eta=0.0)
    rom = DeviceRom.from_host(K, M, D, rhs, omega)
    sweep(handle, [rom])
    X = rom.solutions()
    Xo, info_o = O.sweep(K, M, D, 0.0, rhs, omega)
    _assert_bitexact(X, Xo, f"n={n}")
    assert np.array_equal(rom.info.cpu().numpy(), info_o)


@pytest.mark.parametrize("n", [7, 64, 150])
def test_fp64_keep_factors_and_eta(handle, n):
    rng = np.random.default_rng(7 + n)
    K, M, D, rhs, omega = _rand_rom(rng, n, 2, 3, with_d=True, sym=True)
    eta = 0.035
    rom = DeviceRom.from_host(K, M, D, rhs, omega, eta=eta, keep_factors=True)
    sweep(handle, [rom], flags=_capi.SROM_FLAG_KEEP_FACTORS)
    LU = rom.LU.cpu().numpy().reshape(rom.F, n, n).transpose(0, 2, 1)
    ipiv = rom.ipiv.cpu().numpy().reshape(rom.F, n)
    for f, w in enumerate(omega):
        A = O.assemble(K, M, D, eta, w)
        LUo, ipo, info = O.zgetrf(A)
        assert np.array_equal(ipiv[f], ipo)
        _assert_bitexact(LU[f][None], LUo[None], f"LU n={n} f={f}")
    Xo, _ = O.sweep(K, M, D, eta, rhs, omega)
    _assert_bitexact(rom.solutions(), Xo, "X with eta")


def test_fp64_many_roms_one_call(handle):
    rng = np.random.default_rng(5)
    sizes = [24, 37, 64, 90, 113, 140, 260]
    roms, refs = [], []
    for n in sizes:
        r = int(rng.choice([1, 4]))
        K, M, D, rhs, omega = _rand_rom(rng, n, r, 3, with_d=bool(n % 2))
        roms.append(DeviceRom.from_host(K, M, D, rhs, omega))
        refs.append(O.sweep(K, M, D, 0.0, rhs, omega)[0])
    sweep(handle, roms)
    for rom, ref, n in zip(roms, refs, sizes):
        _assert_bitexact(rom.solutions(), ref, f"batched n={n}")


def test_fp64_singular_reports_info(handle):
    n = 6
    K = np.eye(n, dtype=np.complex128)
    K[:, 3] = 0.0
    M = np.zeros((n, n), dtype=np.complex128)
    rhs = np.ones((n, 1), dtype=np.complex128)
    omega = np.array([1.0, 2.0])
    rom = DeviceRom.from_host(K, M, None, rhs, omega)
    sweep(handle, [rom])
    _, info_o = O.sweep(K, M, None, 0.0, rhs, omega)
    assert info_o[0] == 4
    assert np.array_equal(rom.info.cpu().numpy(), info_o)


def test_fp64_pivoting_required(handle):
    # zero leading entry: an unpivoted LU (what the reference's cuBLAS/cuSOLVER calls do)
    # breaks down here; the pivoted one must not.
    K = np.array([[0, 1, 2], [1, 0, 3], [2, 3, 0]], dtype=np.complex128)
    M = np.zeros_like(K)
    rhs = np.array([[1.0], [2.0], [3.0]], dtype=np.complex128)
    rom = DeviceRom.from_host(K, M, None, rhs, [0.0])
    sweep(handle, [rom])
    x = rom.solutions()[0]
    assert np.allclose(K @ x, rhs, rtol=1e-14, atol=1e-14)
    assert int(rom.info.cpu()[0]) == 0


def test_fp64_plain_workload_slice(handle):
    rom = W.plain_rom()
    sel = rom.omega[::25]
    d = DeviceRom.from_host(rom.K, rom.M, rom.D, rom.rhs, sel)
    sweep(handle, [d])
    Xo, _ = O.sweep(rom.K, rom.M, rom.D, 0.0, rom.rhs, sel)
    _assert_bitexact(d.solutions(), Xo, "plain workload")
    xr = O.x_ref(rom.K, rom.M, rom.D, 0.0, rom.rhs, sel)
    assert O.rel_err(d.solutions(), xr).max() <= 1e-10


def test_fp64_host_entry_point(handle):
    rng = np.random.default_rng(9)
    K, M, D, rhs, omega = _rand_rom(rng, 48, 2, 5)
    h = HostRom(K, M, D, rhs, omega)
    sweep_host(handle, [h])
    Xo, info_o = O.sweep(K, M, D, 0.0, rhs, omega)
    _assert_bitexact(h.solutions(), Xo, "host entry")
    assert np.array_equal(h.info, info_o)


def test_invalid_arguments_raise(handle):
    rng = np.random.default_rng(3)
    K, M, D, rhs, omega = _rand_rom(rng, 4, 1, 2)
    rom = DeviceRom.from_host(K, M, D, rhs, omega)
    d = rom.desc()
    d.ldk = 2
    import ctypes as C

    arr = (_capi.RomDesc * 1)(d)
    o = _capi.SweepOpts(0, 5, 0.0, 0)
    st = _capi.lib().srom_sweep(handle.ptr, arr, 1, C.byref(o))
    assert st == _capi.SROM_ERR_INVALID
    assert b"ldk" in _capi.lib().srom_last_error(handle.ptr)
