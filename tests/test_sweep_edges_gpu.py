"""Edge cases of the sweep's C-ABI contract on the GPU: padded leading dimensions (the padding
holds NaN, so any read of it would show), non-finite entries (IZAMAX's NaN rule), more
right-hand sides than one solve chunk, the mixed form's limit on r, and empty ROMs inside a
batch.  FP64 results are compared bit for bit with the oracle (NaN positions included)."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from staccato_b200 import _capi
from staccato_b200._capi import RomDesc, SweepOpts
from staccato_b200.sweep import DeviceRom, sweep

pytestmark = pytest.mark.gpu


def _bits_equal(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    if a.shape != b.shape:
        return False
    na, nb = np.isnan(a.real) | np.isnan(a.imag), np.isnan(b.real) | np.isnan(b.imag)
    if not np.array_equal(na, nb):
        return False
    return np.array_equal(a[~na].view(np.uint64), b[~nb].view(np.uint64))


def _system(seed, n, r, F, with_d=False):
    rng = np.random.default_rng(seed)
    c = lambda s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    return (c((n, n)) * 10.0 + 3.0 * np.eye(n), c((n, n)), c((n, n)) if with_d else None, c((n, r)),
            rng.uniform(0.1, 3.0, size=F))


def _padded(a, ld):
    """Column-major copy of a with leading dimension ld, NaN in the padding rows."""
    import torch

    rows, cols = a.shape
    buf = np.full((cols, ld), complex(np.nan, np.nan))
    buf[:, :rows] = a.T
    return torch.from_numpy(buf.ravel()).cuda()


# n = 700 (r = 3) runs on the large-order kernel, in the mixed form too (FP64 there)
@pytest.mark.parametrize("form", [0, 1], ids=["fp64", "mixed"])
@pytest.mark.parametrize("n", [50, 200, 700])
def test_padded_leading_dimensions(handle, form, n):
    import torch

    r, F, ldk, ldb = 3, (9 if n < 500 else 3), n + 5, n + 3
    K, M, D, rhs, omega = _system(n, n, r, F, with_d=True)
    dK, dM, dD, dB = _padded(K, ldk), _padded(M, ldk), _padded(D, ldk), _padded(rhs, ldb)
    dw = torch.from_numpy(omega).cuda()
    X = torch.empty(F * n * r, dtype=torch.complex128, device="cuda")
    info = torch.empty(F, dtype=torch.int32, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr())
    d = RomDesc(n=n, r=r, F=F, ldk=ldk, K=p(dK), M=p(dM), D=p(dD), eta=0.01, rhs=p(dB), ldb=ldb,
                omega=p(dw), X=p(X), info=p(info))
    o = SweepOpts(precision=form, max_refine=5, tol=0.0, flags=_capi.SROM_FLAG_FALLBACK_FP64 if form else 0)
    _capi.check(handle.ptr, _capi.lib().srom_sweep(handle.ptr, C.byref(d), 1, C.byref(o)))
    torch.cuda.synchronize()
    Xg = X.cpu().numpy().reshape(F, r, n).transpose(0, 2, 1)
    Xo, info_o = O.sweep(K, M, D, 0.01, rhs, omega)
    assert np.array_equal(info.cpu().numpy(), info_o)
    if form == 0:
        assert _bits_equal(Xg, Xo)
    else:
        Xr = O.x_ref(K, M, D, 0.01, rhs, omega)
        assert O.rel_err(Xg, Xr).max() <= 1e-10


@pytest.mark.parametrize("n", [20, 150, 800])
def test_nonfinite_entries_follow_the_oracle(handle, n):
    """A NaN at the top of a column is taken as that column's pivot (IZAMAX's first entry);
    an Inf elsewhere spreads through the factors.  info, the positions of NaN and every
    finite bit must match the oracle."""
    import torch

    K, M, _, rhs, omega = _system(7 + n, n, 2, 6)
    K[0, 0] = complex(np.nan, 0.0)
    K[n // 2, 3] = complex(np.inf, 1.0)
    rom = DeviceRom.from_host(K, M, None, rhs, omega)
    sweep(handle, [rom])
    torch.cuda.synchronize()
    Xo, info_o = O.sweep(K, M, None, 0.0, rhs, omega)
    assert np.array_equal(rom.info.cpu().numpy(), info_o)
    assert _bits_equal(rom.solutions(), Xo)


@pytest.mark.parametrize("n", [40, 180])
def test_fp64_more_rhs_than_a_solve_chunk(handle, n):
    import torch

    K, M, D, rhs, omega = _system(3 + n, n, 21, 5)
    rom = DeviceRom.from_host(K, M, D, rhs, omega, eta=0.02)
    sweep(handle, [rom])
    torch.cuda.synchronize()
    Xo, _ = O.sweep(K, M, D, 0.02, rhs, omega)
    assert _bits_equal(rom.solutions(), Xo)


def test_mixed_rhs_limit(handle):
    import torch

    n = 96
    K, M, _, rhs, omega = _system(11, n, 16, 7)
    rom = DeviceRom.from_host(K, M, None, rhs, omega)
    sweep(handle, [rom], precision=_capi.SROM_MIXED_FP32, flags=_capi.SROM_FLAG_FALLBACK_FP64)
    torch.cuda.synchronize()
    assert O.rel_err(rom.solutions(), O.x_ref(K, M, None, 0.0, rhs, omega)).max() <= 1e-10
    K, M, _, rhs, omega = _system(12, n, 17, 3)
    rom = DeviceRom.from_host(K, M, None, rhs, omega)
    with pytest.raises(_capi.SromError) as e:
        sweep(handle, [rom], precision=_capi.SROM_MIXED_FP32)
    assert e.value.status == _capi.SROM_ERR_UNSUPPORTED


@pytest.mark.parametrize("form", [0, 1], ids=["fp64", "mixed"])
def test_empty_roms_in_a_batch(handle, form):
    """ROMs with F = 0 or r = 0 are skipped; the others in the call are solved as usual."""
    import torch

    a = _system(1, 30, 1, 4)
    b = _system(2, 70, 2, 5)
    ra = DeviceRom.from_host(*a)
    rb = DeviceRom.from_host(*b)
    empty_f = DeviceRom.from_host(*_system(3, 10, 1, 1))
    empty_f.F = 0
    empty_r = DeviceRom.from_host(*_system(4, 12, 1, 2))
    empty_r.r = 0
    flags = _capi.SROM_FLAG_FALLBACK_FP64 if form else 0
    sweep(handle, [empty_f, ra, empty_r, rb], precision=form, flags=flags)
    torch.cuda.synchronize()
    for rom, sysd in ((ra, a), (rb, b)):
        Xo, _ = O.sweep(sysd[0], sysd[1], None, 0.0, sysd[3], sysd[4])
        if form == 0:
            assert _bits_equal(rom.solutions(), Xo)
        else:
            assert O.rel_err(rom.solutions(), O.x_ref(sysd[0], sysd[1], None, 0.0, sysd[3], sysd[4])).max() <= 1e-10


@pytest.mark.parametrize("field", ["K", "M", "rhs", "X", "Y"])
def test_misaligned_device_arrays_are_rejected(handle, field):
    """A complex array that is 8- but not 16-byte aligned is refused on the host before any
    launch (the kernels access complex values as 16-byte vectors)."""
    import torch

    K, M, _, rhs, omega = _system(21, 8, 2, 3)
    Cm = np.ones((2, 8), dtype=np.complex128)
    rom = DeviceRom.from_host(K, M, None, rhs, omega, C=Cm)
    d = rom.desc()
    setattr(d, field, getattr(d, field) + 8)
    arr = (_capi.RomDesc * 1)(d)
    for prec in (_capi.SROM_FP64, _capi.SROM_MIXED_FP32):
        o = _capi.SweepOpts(precision=prec, max_refine=5, tol=0.0, flags=0)
        st = _capi.lib().srom_sweep(handle.ptr, arr, 1, C.byref(o))
        assert st == _capi.SROM_ERR_INVALID
        assert b"aligned" in _capi.lib().srom_last_error(handle.ptr)
    torch.cuda.synchronize()
    sweep(handle, [rom])  # the aligned descriptor still works on the same handle
    torch.cuda.synchronize()
    Xo, _ = O.sweep(K, M, None, 0.0, rhs, omega)
    assert _bits_equal(rom.solutions(), Xo)
