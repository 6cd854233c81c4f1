"""Large reduced orders (panels beyond shared memory, up to n = 2560) on the GPU against the CPU oracle.

The reference's largest dense ROM is r2520 (test/krylovTestGPU/matrixInSingleLoop/gpu/src/
main.cu:344-364, one right-hand side per frequency).  Systems whose panel does not fit the
global kernel's shared memory (n > 673 at r = 1, every n > 768) run on the large-order
instances of the FP64 global kernel: 3, 6 or 10 rows per thread in the panel search, the panel
in the CTA's global scratch instead of shared memory, and the tile-staged blocked solve.  The
factorisation restates zgetrf exactly as the smaller instances do, so solutions, factors and
pivots equal the oracle's exactly.  The mixed precisions have no kernel at these orders: they
solve such systems in FP64 (steps = 0).
"""
import numpy as np
import pytest

from oracle import oracle as O
from staccato_b200 import _capi
from staccato_b200.sweep import DeviceRom, Graph, sweep

pytestmark = pytest.mark.gpu


def _rand_rom(seed, n, r, F, with_d=True):
    rng = np.random.default_rng(seed)

    def c(shape):
        return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)

    K = c((n, n)) * 10.0 + np.eye(n) * 3.0
    M = c((n, n))
    D = c((n, n)) if with_d else None
    return K, M, D, c((n, r)), rng.uniform(0.1, 3.0, size=F)


def _assert_bitexact(a, b, what):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    assert a.shape == b.shape, what
    same = (a.view(np.uint64) == b.view(np.uint64)).reshape(a.shape[0], -1).all(axis=1)
    assert same.all(), f"{what}: {int((~same).sum())} of {len(same)} systems differ"


def _kernels(handle, fn):
    handle.profile(True)
    handle.read_profile()
    fn()
    recs, _ = handle.read_profile()
    handle.profile(False)
    return [rec[0] for rec in recs]


# The shared-memory panel of the global kernel holds n <= 673 at r = 1 (583 at r = 3); larger
# panels go to the large-order kernel, whose instances hold 3, 6 or 10 rows a thread.
@pytest.mark.parametrize("n,r,F,kernel", [(660, 1, 2, "fp64_global"), (700, 3, 2, "fp64_large"),
                                          (769, 2, 2, "fp64_large"), (1024, 1, 2, "fp64_large"),
                                          (1500, 4, 1, "fp64_large"), (1380, 8, 1, "fp64_large")])
def test_large_orders_match_oracle_bitwise(handle, n, r, F, kernel):
    K, M, D, rhs, omega = _rand_rom(5000 + n, n, r, F, with_d=(n % 2 == 1))
    rom = DeviceRom.from_host(K, M, D, rhs, omega)
    names = _kernels(handle, lambda: sweep(handle, [rom]))
    assert kernel in names, names
    Xo, info_o = O.sweep(K, M, D, 0.0, rhs, omega)
    _assert_bitexact(rom.solutions(), Xo, f"n={n}")
    assert np.array_equal(rom.info.cpu().numpy(), info_o)


def test_reference_largest_order_2520(handle):
    """n = 2520, one right-hand side (the reference's r2520 case), one frequency."""
    n = 2520
    K, M, D, rhs, omega = _rand_rom(2520, n, 1, 1, with_d=False)
    rom = DeviceRom.from_host(K, M, D, rhs, omega)
    sweep(handle, [rom])
    Xo, info_o = O.sweep(K, M, D, 0.0, rhs, omega)
    _assert_bitexact(rom.solutions(), Xo, "n=2520")
    assert rom.info.cpu().numpy()[0] == 0 == info_o[0]


def test_large_order_keeps_factors(handle):
    n = 800
    K, M, D, rhs, omega = _rand_rom(31, n, 2, 2)
    eta = 0.02
    rom = DeviceRom.from_host(K, M, D, rhs, omega, eta=eta, keep_factors=True)
    sweep(handle, [rom], flags=_capi.SROM_FLAG_KEEP_FACTORS)
    LU = rom.LU.cpu().numpy().reshape(rom.F, n, n).transpose(0, 2, 1)
    ipiv = rom.ipiv.cpu().numpy().reshape(rom.F, n)
    for f, w in enumerate(omega):
        LUo, ipo, _ = O.zgetrf(O.assemble(K, M, D, eta, w))
        assert np.array_equal(ipiv[f], ipo)
        _assert_bitexact(LU[f][None], LUo[None], f"LU f={f}")
    Xo, _ = O.sweep(K, M, D, eta, rhs, omega)
    _assert_bitexact(rom.solutions(), Xo, "X with eta")


def test_all_three_fp64_kernels_in_one_call(handle):
    """Orders 90 (shared-memory kernel), 600 (global kernel) and 900 (large-order kernel) in one
    call: the global and large-order launches share the scratch buffer one after the other."""
    specs = [(90, 2, 5), (600, 1, 3), (900, 2, 3), (610, 3, 2)]
    roms, refs = [], []
    for i, (n, r, F) in enumerate(specs):
        K, M, D, rhs, omega = _rand_rom(70 + i, n, r, F)
        roms.append(DeviceRom.from_host(K, M, D, rhs, omega))
        refs.append(O.sweep(K, M, D, 0.0, rhs, omega)[0])
    names = _kernels(handle, lambda: sweep(handle, roms))
    assert {"fp64_smem", "fp64_global", "fp64_large"} <= set(names), names
    for d, xo, s in zip(roms, refs, specs):
        _assert_bitexact(d.solutions(), xo, f"n={s[0]}")


@pytest.mark.parametrize("precision", [_capi.SROM_MIXED_FP32, _capi.SROM_MIXED_TC, _capi.SROM_MIXED_AUTO])
def test_mixed_precisions_solve_large_orders_in_fp64(handle, precision):
    n = 1024
    K, M, D, rhs, omega = _rand_rom(11, n, 2, 2)
    rom = DeviceRom.from_host(K, M, D, rhs, omega)
    small = DeviceRom.from_host(*_rand_rom(12, 300, 2, 3))
    names = _kernels(handle, lambda: sweep(handle, [rom, small], precision=precision,
                                           flags=_capi.SROM_FLAG_FALLBACK_FP64))
    assert "fp64_large" in names
    Xo, _ = O.sweep(K, M, D, 0.0, rhs, omega)
    _assert_bitexact(rom.solutions(), Xo, "mixed plan, n=1024")
    assert (rom.steps.cpu().numpy() == 0).all()
    assert (small.steps.cpu().numpy() >= 1).all()


def test_large_order_graph_replay_equals_direct_sweep(handle):
    import torch

    K, M, D, rhs, omega = _rand_rom(41, 880, 1, 3)
    a = DeviceRom.from_host(K, M, D, rhs, omega)
    b = DeviceRom.from_host(K, M, D, rhs, omega)
    sweep(handle, [a])
    g = Graph(handle, [b])
    try:
        g.launch()
        g.launch()
        torch.cuda.synchronize()
    finally:
        g.close()
    _assert_bitexact(b.solutions(), a.solutions(), "graph n=880")


def test_large_order_limits(handle):
    # above 2560 rows: no kernel
    K, M, D, rhs, omega = _rand_rom(1, 2561, 1, 1, with_d=False)
    rom = DeviceRom.from_host(K, M, None, rhs, omega)
    with pytest.raises(_capi.SromError) as e:
        sweep(handle, [rom])
    assert e.value.status == _capi.SROM_ERR_UNSUPPORTED
    # the right-hand sides live in shared memory: n * r * 16 bytes, r <= 4 at n = 2520
    # (r <= 8 up to n = 1388, r <= 16 up to n = 724)
    K, M, D, rhs, omega = _rand_rom(2, 2520, 5, 1, with_d=False)
    rom = DeviceRom.from_host(K, M, None, rhs, omega)
    with pytest.raises(_capi.SromError) as e:
        sweep(handle, [rom])
    assert e.value.status == _capi.SROM_ERR_UNSUPPORTED
    assert b"shared memory" in _capi.lib().srom_last_error(handle.ptr)
