"""Mixed-precision sweep (complex FP32 factors + FP64 refinement) on the GPU.

Gate: relative error <= 1e-10 against the oracle's long-double-refined solution for every
frequency (after FP64 fallback of the frequencies that do not converge), on the workload
shapes; and the reported steps / info / fallback markers must be consistent.
"""
import numpy as np
import pytest

from oracle import oracle as O
from staccato_b200 import _capi, workloads as W
from staccato_b200.sweep import DeviceRom, sweep

pytestmark = pytest.mark.gpu

MIXED = _capi.SROM_MIXED_FP32
FALLBACK = _capi.SROM_FLAG_FALLBACK_FP64
EVERY = _capi.SROM_FLAG_MIXED_EVERY  # keeps the smallest systems in the mixed kernel


def _run(handle, rom_like, omega, precision=MIXED, flags=FALLBACK, max_refine=5):
    d = DeviceRom.from_host(rom_like.K, rom_like.M, rom_like.D, rom_like.rhs, omega)
    sweep(handle, [d], precision=precision, flags=flags, max_refine=max_refine)
    return d


@pytest.mark.parametrize("n", [1, 2, 17, 64, 100, 255, 256, 511])
def test_mixed_random_wellconditioned(handle, n):
    rng = np.random.default_rng(40 + n)
    c = lambda s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    K = c((n, n)) + 4.0 * np.sqrt(n) * np.eye(n)
    M = c((n, n)) * 0.1
    r = 3 if n < 300 else 1
    rom = W.Rom(K=K, M=M, D=c((n, n)) * 0.01, rhs=c((n, r)), omega=rng.uniform(0.1, 1.0, 4))
    d = _run(handle, rom, rom.omega, flags=EVERY)
    xr = O.x_ref(rom.K, rom.M, rom.D, 0.0, rom.rhs, rom.omega)
    err = O.rel_err(d.solutions(), xr)
    assert err.max() <= 1e-10, err
    steps = d.steps.cpu().numpy()
    assert (steps >= 0).all() and (steps <= 5).all()
    assert (d.info.cpu().numpy() == 0).all()
    assert (d.berr.cpu().numpy() <= 2.0 ** -34).all()


def test_mixed_plain_workload(handle):
    rom = W.plain_rom()
    sel = rom.omega  # all 500 frequencies: the gate is on the maximum
    d = _run(handle, rom, sel, flags=FALLBACK | EVERY)
    xr = O.x_ref(rom.K, rom.M, rom.D, 0.0, rom.rhs, sel)
    assert O.rel_err(d.solutions(), xr).max() <= 1e-10
    assert (d.steps.cpu().numpy() >= 1).all()  # refined, and no fallback needed on this workload


@pytest.mark.parametrize("n,r,routed", [(40, 2, True), (80, 4, True), (96, 1, False), (128, 4, False)])
def test_mixed_form_solves_small_systems_in_fp64(n, r, routed):
    """Without SROM_FLAG_MIXED_EVERY, systems held two per SM by the FP64 shared-memory kernel
    are solved by it outright: the FP64 form's bits, steps = 0, berr = 0.  Larger ones are
    refined.  A fresh handle, so that no tuning table changes the kernel choice."""
    h = _capi.Handle(0)
    try:
        rom = W.plain_rom(n=n, F=40)
        rng = np.random.default_rng(n)
        rhs = rng.standard_normal((n, r)) + 1j * rng.standard_normal((n, r))
        d = DeviceRom.from_host(rom.K, rom.M, rom.D, rhs, rom.omega)
        sweep(h, [d], precision=MIXED, flags=FALLBACK)
        steps = d.steps.cpu().numpy()
        xr = O.x_ref(rom.K, rom.M, rom.D, 0.0, rhs, rom.omega)
        assert O.rel_err(d.solutions(), xr).max() <= 1e-10
        if routed:
            d64 = DeviceRom.from_host(rom.K, rom.M, rom.D, rhs, rom.omega)
            sweep(h, [d64], precision=_capi.SROM_FP64)
            assert np.array_equal(d.solutions().view(np.uint64), d64.solutions().view(np.uint64))
            assert (steps == 0).all() and (d.berr.cpu().numpy() == 0.0).all()
        else:
            assert (steps != 0).all()
    finally:
        h.close()


def test_mixed_precision_workload_near_resonance(handle):
    rom = W.precision_rom()
    sel = rom.omega[:96]
    d = _run(handle, rom, sel)
    xr = O.x_ref(rom.K, rom.M, rom.D, 0.0, rom.rhs, sel)
    err = O.rel_err(d.solutions(), xr)
    assert err.max() <= 1e-10, (err.max(), int(np.argmax(err)))
    steps = d.steps.cpu().numpy()
    assert ((steps >= 0) | (steps == -1)).all()
    assert (d.info.cpu().numpy() == 0).all()


def test_mixed_batching_roms(handle):
    roms = W.batching_roms()
    pick = [roms[i] for i in (0, 5, 17, 42)]
    devs, refs = [], []
    for r in pick:
        sel = r.omega[:: max(1, r.F // 6)][:6]
        devs.append(DeviceRom.from_host(r.K, r.M, r.D, r.rhs, sel))
        refs.append(O.x_ref(r.K, r.M, r.D, 0.0, r.rhs, sel))
    sweep(handle, devs, precision=MIXED, flags=FALLBACK)
    for d, xr in zip(devs, refs):
        assert O.rel_err(d.solutions(), xr).max() <= 1e-10, d.n


def test_mixed_nonconvergence_and_fallback(handle):
    # kappa ~ 1e12: complex-FP32 factors cannot drive the refinement to convergence.
    n = 48
    rng = np.random.default_rng(99)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    s = np.logspace(0, -12, n)
    K = (q * s) @ q.T + 0j
    M = np.zeros((n, n), dtype=np.complex128)
    rhs = rng.standard_normal((n, 1)) + 0j
    rom = W.Rom(K=K, M=M, D=None, rhs=rhs, omega=np.array([0.0, 0.0]))
    d0 = _run(handle, rom, rom.omega, flags=EVERY, max_refine=3)
    assert (d0.info.cpu().numpy() == -1).all()
    assert (d0.steps.cpu().numpy() == 3).all()
    d1 = _run(handle, rom, rom.omega, flags=FALLBACK | EVERY, max_refine=3)
    assert (d1.steps.cpu().numpy() == -1).all()
    d64 = _run(handle, rom, rom.omega, precision=_capi.SROM_FP64, flags=0)
    assert np.array_equal(d1.solutions().view(np.uint64), d64.solutions().view(np.uint64))


def test_mixed_rejects_keep_factors(handle):
    rng = np.random.default_rng(1)
    K = rng.standard_normal((8, 8)) + 8 * np.eye(8) + 0j
    d = DeviceRom.from_host(K, np.eye(8), None, np.ones((8, 1)), [1.0], keep_factors=True)
    with pytest.raises(_capi.SromError) as e:
        sweep(handle, [d], precision=MIXED)
    assert e.value.status == _capi.SROM_ERR_UNSUPPORTED
