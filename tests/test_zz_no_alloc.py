"""srom_sweep_fp64_noalloc: the sweep entry point that allocates no device memory.

It exists for callers that cannot let a library allocate -- host programs that own all
device memory through their own pool, or real-time loops in which cudaMalloc's implicit
synchronisation and possible failure are not acceptable.  Its results must equal those of
srom_sweep (FP64 results are bit-identical, the tolerance every FP64 test here uses), on
two calls in a row, because every call reuses the library's scratch array.  This file is
named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from staccato_b200 import _capi
from staccato_b200.sweep import DeviceRom, sweep

pytestmark = pytest.mark.gpu


def _rom(seed, n, r, F, with_d):
    rng = np.random.default_rng(seed)
    c = lambda s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    K = c((n, n)) * 10.0 + 3.0 * np.eye(n)
    return DeviceRom.from_host(K, c((n, n)), c((n, n)) if with_d else None, c((n, r)),
                               rng.uniform(0.1, 3.0, size=F), eta=0.01)


def _noalloc(rom, stream):
    d = rom.desc()
    err = C.create_string_buffer(256)
    st = _capi.lib().srom_sweep_fp64_noalloc(C.byref(d), C.c_void_p(stream), err, 256)
    return st, err.value.decode()


def _same(a, b):
    return np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_noalloc_matches_srom_sweep_on_consecutive_calls(handle):
    import torch

    stream = torch.cuda.current_stream().cuda_stream
    handle.set_stream(stream)
    cases = [_rom(11, 100, 3, 37, True), _rom(12, 300, 2, 19, False), _rom(13, 512, 1, 9, True)]
    refs = []
    for rom in cases:
        sweep(handle, [rom])
        torch.cuda.synchronize()
        refs.append((rom.solutions().copy(), rom.info.cpu().numpy().copy()))
    for rnd in range(2):  # two calls in a row per case, and the cases back to back
        for rom, (X, info) in zip(cases, refs):
            rom.X.fill_(float("nan"))
            rom.info.fill_(-7)
            st, msg = _noalloc(rom, stream)
            assert st == _capi.SROM_OK, msg
            torch.cuda.synchronize()
            assert _same(rom.solutions(), X), f"round {rnd} n={rom.n}"
            assert np.array_equal(rom.info.cpu().numpy(), info)


def test_noalloc_rejects_sizes_beyond_its_limit(handle):
    import torch

    rom = _rom(14, 4, 1, 2, False)
    d = rom.desc()
    d.n = 600
    d.ldk = d.ldb = 600
    err = C.create_string_buffer(256)
    st = _capi.lib().srom_sweep_fp64_noalloc(C.byref(d), None, err, 256)
    assert st == _capi.SROM_ERR_UNSUPPORTED
    assert b"exceeds the limit of 512" in err.value
    d = rom.desc()
    d.F = 70000
    st = _capi.lib().srom_sweep_fp64_noalloc(C.byref(d), None, err, 256)
    assert st == _capi.SROM_ERR_UNSUPPORTED and b"65536" in err.value
    torch.cuda.synchronize()


def test_noalloc_shared_memory_limit_at_the_largest_order(handle):
    """At n = 512 the blocked kernel's shared memory holds r <= 5 right-hand sides: r = 5 runs
    (bit-identical to srom_sweep), r = 6 is refused before anything is launched."""
    import torch

    stream = torch.cuda.current_stream().cuda_stream
    handle.set_stream(stream)
    rom = _rom(15, 512, 5, 3, False)
    sweep(handle, [rom])
    torch.cuda.synchronize()
    X = rom.solutions().copy()
    rom.X.fill_(float("nan"))
    st, msg = _noalloc(rom, stream)
    assert st == _capi.SROM_OK, msg
    torch.cuda.synchronize()
    assert _same(rom.solutions(), X)
    big = _rom(16, 512, 6, 2, False)
    st, msg = _noalloc(big, stream)
    assert st == _capi.SROM_ERR_UNSUPPORTED and "shared memory" in msg, msg


def test_noalloc_allocates_no_device_memory(handle):
    """Free device memory (the driver's count) is the same before and after a run of calls: the
    entry point takes its scratch from the library's static array.  The first call, which may
    load the library's device code (and with it the array), is made before the first count."""
    import torch

    stream = torch.cuda.current_stream().cuda_stream
    roms = [_rom(17, 200, 2, 64, True), _rom(18, 512, 1, 40, False)]
    st, msg = _noalloc(roms[0], stream)
    assert st == _capi.SROM_OK, msg
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        for rom in roms:
            st, msg = _noalloc(rom, stream)
            assert st == _capi.SROM_OK, msg
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_backprojection_matches_srom_sweep(handle):
    """With n_out > 0 the entry point also writes y = C x, bit-identical to srom_sweep."""
    import torch

    stream = torch.cuda.current_stream().cuda_stream
    handle.set_stream(stream)
    rng = np.random.default_rng(21)
    n, r, F, n_out = 120, 2, 13, 9
    c = lambda s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    rom = DeviceRom.from_host(c((n, n)) * 10.0 + 3.0 * np.eye(n), c((n, n)), None, c((n, r)),
                              rng.uniform(0.1, 3.0, size=F), C=c((n_out, n)))
    sweep(handle, [rom])
    torch.cuda.synchronize()
    Y = rom.outputs().copy()
    rom.Y.fill_(float("nan"))
    st, msg = _noalloc(rom, stream)
    assert st == _capi.SROM_OK, msg
    torch.cuda.synchronize()
    assert _same(rom.outputs(), Y)

