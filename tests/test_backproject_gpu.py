"""Back-projection y(w) = C x(w) fused after the sweep (srom_rom_desc.C / .Y): the output of
the reference's backTransformKMOR (KrylovROMSubstructure.cpp:1446-1449) and, with B_R as the
right-hand sides, its transfer functions H_R = C_R A^-1 B_R (:1433-1441).

FP64 outputs are compared bit for bit with the oracle (oracle/srom_oracle.c:
oracle_backproject, the same summation order), both on the GPU's own x and on the oracle's
x; mixed outputs against C x_ref with the sweep's 1e-10 gate."""
import ctypes as C
import math

import numpy as np
import pytest

from oracle import oracle as O
from staccato_b200 import _capi, workloads as W
from staccato_b200.rom import KrylovROMSubstructure
from staccato_b200.sweep import DeviceRom, Graph, HostRom, sweep, sweep_host

pytestmark = pytest.mark.gpu


def _same(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def _case(seed, n, r, F, n_out, with_d=False):
    rng = np.random.default_rng(seed)
    c = lambda s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    K = c((n, n)) * 10.0 + 3.0 * np.eye(n)
    M = c((n, n))
    D = c((n, n)) if with_d else None
    rhs = c((n, r))
    omega = rng.uniform(0.1, 3.0, size=F)
    Cm = c((n_out, n))
    return K, M, D, rhs, omega, Cm


# n = 64 runs in the shared-memory kernel, 200 and 320 in the global one; n_out * r > 256
# makes threads loop over outputs; n = 320, r = 10 is too large to stage x in shared memory.
@pytest.mark.parametrize("n,r,F,n_out", [(64, 1, 33, 1), (64, 4, 20, 7), (200, 3, 17, 90),
                                         (320, 10, 5, 40), (31, 2, 9, 300)])
def test_fp64_backprojection_bitwise(handle, n, r, F, n_out):
    import torch

    K, M, D, rhs, omega, Cm = _case(n + r, n, r, F, n_out, with_d=(n == 200))
    rom = DeviceRom.from_host(K, M, D, rhs, omega, eta=0.01, C=Cm)
    sweep(handle, [rom])
    torch.cuda.synchronize()
    X, Y = rom.solutions(), rom.outputs()
    assert _same(Y, O.backproject(Cm, X))
    Xo, _ = O.sweep(K, M, D, 0.01, rhs, omega)
    assert _same(X, Xo)
    assert _same(Y, O.backproject(Cm, Xo))


def test_mixed_backprojection_meets_gate(handle):
    import torch

    rom_w = W.precision_rom(F=64)
    n = rom_w.n
    rng = np.random.default_rng(4)
    Cm = rng.standard_normal((5, n)) + 1j * rng.standard_normal((5, n))
    rom = DeviceRom.from_host(rom_w.K, rom_w.M, rom_w.D, rom_w.rhs, rom_w.omega, C=Cm)
    sweep(handle, [rom], precision=_capi.SROM_MIXED_FP32, flags=_capi.SROM_FLAG_FALLBACK_FP64)
    torch.cuda.synchronize()
    Xref = O.x_ref(rom_w.K, rom_w.M, rom_w.D, 0.0, rom_w.rhs, rom_w.omega)
    Yref = np.einsum("on,fnr->for", Cm, Xref)
    Y = rom.outputs()
    num = np.linalg.norm((Y - Yref).reshape(len(Y), -1), axis=1)
    err = num / np.linalg.norm(Yref.reshape(len(Y), -1), axis=1)
    assert err.max() <= 1e-10
    assert _same(Y, O.backproject(Cm, rom.solutions()))


def test_backprojection_host_graph_and_mixed_batch(handle):
    """srom_sweep_host and a captured graph give the same bits as srom_sweep; ROMs with and
    without C in one call."""
    import torch

    a = _case(1, 48, 2, 11, 6)
    b = _case(2, 150, 1, 7, 3)
    c = _case(3, 90, 3, 5, 2)
    roms = [DeviceRom.from_host(*a[:5], C=a[5]), DeviceRom.from_host(*b[:5]), DeviceRom.from_host(*c[:5], C=c[5])]
    sweep(handle, roms)
    torch.cuda.synchronize()
    Ys = [roms[0].outputs().copy(), roms[2].outputs().copy()]
    assert roms[1].Y is None
    hr = [HostRom(*a[:5], C=a[5]), HostRom(*b[:5]), HostRom(*c[:5], C=c[5])]
    sweep_host(handle, hr)
    assert _same(hr[0].outputs(), Ys[0]) and _same(hr[2].outputs(), Ys[1])
    for rm in roms:
        if rm.Y is not None:
            rm.Y.fill_(float("nan"))
    g = Graph(handle, roms)
    g.launch(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    g.close()
    assert _same(roms[0].outputs(), Ys[0]) and _same(roms[2].outputs(), Ys[1])


def test_transfer_functions_match_oracle(handle):
    rom_w = W.plain_rom(F=24)
    n = rom_w.n
    rng = np.random.default_rng(9)
    B = rng.standard_normal((n, 3))
    Cm = rng.standard_normal((4, n))
    s = KrylovROMSubstructure(handle=handle)
    s.set_reduced(rom_w.K, rom_w.M, None, B, Cm)
    freq = rom_w.omega / (2 * math.pi)
    H, info = s.transfer_functions(freq)
    Xo, _ = O.sweep(rom_w.K, rom_w.M, None, 0.0, B.astype(complex), 2 * math.pi * freq)
    Href = O.backproject(Cm.astype(complex), Xo)
    assert _same(H.cpu().numpy(), Href)
    assert (info.cpu().numpy() == 0).all()


def test_backprojection_argument_checks(handle):
    K, M, D, rhs, omega, Cm = _case(5, 16, 1, 3, 2)
    rom = DeviceRom.from_host(K, M, D, rhs, omega, C=Cm)
    o = _capi.SweepOpts(precision=0, max_refine=5, tol=0.0, flags=0)
    d = rom.desc()
    d.C = None
    assert _capi.lib().srom_sweep(handle.ptr, C.byref(d), 1, C.byref(o)) == _capi.SROM_ERR_INVALID
    d = rom.desc()
    d.ldc = 1
    assert _capi.lib().srom_sweep(handle.ptr, C.byref(d), 1, C.byref(o)) == _capi.SROM_ERR_INVALID
