"""Tensor-core mixed form (SROM_MIXED_TC) on the GPU.

The factorisation is the complex-FP32 blocked LU of the CUDA-core mixed form with every Schur
update run as tcgen05 MMAs on three-piece bf16 splits; the refinement is the same FP64 one.
Gate: relative error <= 1e-10 against the oracle's long-double-refined x_ref on every tested
frequency.  Because the FP64 fallback would hide a wrong factorisation, the tests also require
convergence without it (info = 0) and a refinement-step count no worse than the CUDA-core FP32
factors need on the same systems (one step of slack): a wrong Schur update cannot converge.
"""
import numpy as np
import pytest

from oracle import oracle as O
from staccato_b200 import _capi, workloads as W
from staccato_b200.sweep import DeviceRom, sweep

pytestmark = pytest.mark.gpu

TC = _capi.SROM_MIXED_TC
FP32 = _capi.SROM_MIXED_FP32
FALLBACK = _capi.SROM_FLAG_FALLBACK_FP64
EVERY = _capi.SROM_FLAG_MIXED_EVERY


def _sweep(handle, rom, omega, precision, flags, max_refine=5):
    d = DeviceRom.from_host(rom.K, rom.M, rom.D, rom.rhs, omega)
    sweep(handle, [d], precision=precision, flags=flags, max_refine=max_refine)
    return d


def _random_rom(n, r, seed, F=6):
    rng = np.random.default_rng(seed)
    c = lambda s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    K = c((n, n)) + 4.0 * np.sqrt(n) * np.eye(n)
    return W.Rom(K=K, M=c((n, n)) * 0.1, D=c((n, n)) * 0.01, rhs=c((n, r)), omega=rng.uniform(0.1, 1.0, F))


# orders around the panel (32), tile-row (128) and tile-column (32) boundaries, up to the limit
@pytest.mark.parametrize("n", [1, 31, 32, 33, 63, 64, 65, 96, 97, 160, 161, 191, 255, 256, 300, 384, 449, 511, 512])
def test_tc_random_matches_oracle_without_fallback(handle, n):
    r = 3 if n < 300 else 2
    rom = _random_rom(n, r, 1000 + n)
    d = _sweep(handle, rom, rom.omega, TC, EVERY)
    xr = O.x_ref(rom.K, rom.M, rom.D, 0.0, rom.rhs, rom.omega)
    err = O.rel_err(d.solutions(), xr)
    assert err.max() <= 1e-10, err
    assert (d.info.cpu().numpy() == 0).all()
    steps_tc = d.steps.cpu().numpy()
    d32 = _sweep(handle, rom, rom.omega, FP32, EVERY)
    steps_32 = d32.steps.cpu().numpy()
    assert (steps_tc >= 0).all() and (steps_tc <= steps_32 + 1).all(), (steps_tc, steps_32)


@pytest.mark.parametrize("r", [1, 4, 5])
def test_tc_right_hand_side_counts_at_the_largest_order(handle, r):
    rom = _random_rom(512, r, 77 + r, F=3)
    d = _sweep(handle, rom, rom.omega, TC, EVERY)
    xr = O.x_ref(rom.K, rom.M, rom.D, 0.0, rom.rhs, rom.omega)
    assert O.rel_err(d.solutions(), xr).max() <= 1e-10
    assert (d.info.cpu().numpy() == 0).all()


def test_tc_plain_workload(handle):
    rom = W.plain_rom()
    d = _sweep(handle, rom, rom.omega, TC, FALLBACK | EVERY)
    xr = O.x_ref(rom.K, rom.M, rom.D, 0.0, rom.rhs, rom.omega)
    assert O.rel_err(d.solutions(), xr).max() <= 1e-10
    assert (d.steps.cpu().numpy() >= 1).all()  # refined, no fallback


def test_tc_precision_workload_near_resonance(handle):
    """n = 256, r = 8, 60 % of the frequencies within 0.1 % of an eigenfrequency: every 8th
    frequency (512 systems) against x_ref.  Near resonance the tensor-core factor (FP32
    accumulation in the tensor cores, U12 through the inverse of the panel's unit triangle)
    leaves somewhat more systems to the FP64 re-solve than the CUDA-core FP32 factor (measured
    25 against 14 of 512); the bound is twice the CUDA-core count, and the mean refinement
    steps of the converged systems within half a step of it."""
    rom = W.precision_rom()
    sel = rom.omega[::8]
    d = _sweep(handle, rom, sel, TC, FALLBACK)
    xr = O.x_ref(rom.K, rom.M, rom.D, 0.0, rom.rhs, sel)
    err = O.rel_err(d.solutions(), xr)
    assert err.max() <= 1e-10, (err.max(), int(np.argmax(err)))
    d32 = _sweep(handle, rom, sel, FP32, FALLBACK)
    fb_tc = int((d.steps.cpu().numpy() == -1).sum())
    fb_32 = int((d32.steps.cpu().numpy() == -1).sum())
    assert fb_tc <= max(2 * fb_32, 8), (fb_tc, fb_32)
    s_tc = d.steps.cpu().numpy()
    s_32 = d32.steps.cpu().numpy()
    ok = (s_tc >= 0) & (s_32 >= 0)
    assert s_tc[ok].mean() <= s_32[ok].mean() + 0.5, (s_tc[ok].mean(), s_32[ok].mean())


def test_tc_batching_roms_and_kernel_choice(handle):
    """Several ROMs of the batching workload in one call (orders 24..512, r in {1, 4}); the
    per-launch profile shows the tensor-core kernel ran."""
    roms = W.batching_roms()
    pick = [roms[i] for i in (0, 5, 17, 42, 60)]
    devs, refs = [], []
    for r in pick:
        sel = r.omega[:: max(1, r.F // 8)][:8]
        devs.append(DeviceRom.from_host(r.K, r.M, r.D, r.rhs, sel))
        refs.append(O.x_ref(r.K, r.M, r.D, 0.0, r.rhs, sel))
    handle.profile(True)
    handle.read_profile()
    sweep(handle, devs, precision=TC, flags=FALLBACK)
    recs, _ = handle.read_profile()
    handle.profile(False)
    assert "mixed_tc" in [rec[0] for rec in recs]
    for d, xr in zip(devs, refs):
        assert O.rel_err(d.solutions(), xr).max() <= 1e-10, d.n
        assert (d.steps.cpu().numpy() != -1).all()


def test_tc_zero_pivot_reported(handle):
    """A singular system (a zero column) reports LAPACK's info = first zero pivot column, as the
    CUDA-core mixed form does, instead of a converged solution."""
    n = 70
    rom = _random_rom(n, 1, 5, F=2)
    K = rom.K.copy()
    K[:, 40] = 0.0
    rom = W.Rom(K=K, M=np.zeros_like(K), D=None, rhs=rom.rhs, omega=np.array([0.5, 0.7]))
    d = _sweep(handle, rom, rom.omega, TC, EVERY, max_refine=2)
    d32 = _sweep(handle, rom, rom.omega, FP32, EVERY, max_refine=2)
    assert (d.info.cpu().numpy() == d32.info.cpu().numpy()).all()
    assert (d.info.cpu().numpy() == 41).all()


def test_tc_larger_orders_use_the_fp32_kernel(handle):
    """Above n = 512 the tensor-core precision falls back to the CUDA-core FP32 kernel."""
    rom = _random_rom(600, 1, 3, F=2)
    handle.profile(True)
    handle.read_profile()
    d = _sweep(handle, rom, rom.omega, TC, EVERY)
    recs, _ = handle.read_profile()
    handle.profile(False)
    names = [rec[0] for rec in recs]
    assert "mixed_global" in names and "mixed_tc" not in names
    xr = O.x_ref(rom.K, rom.M, rom.D, 0.0, rom.rhs, rom.omega)
    assert O.rel_err(d.solutions(), xr).max() <= 1e-10


def _kernels(h, fn):
    h.profile(True)
    h.read_profile()
    fn()
    recs, _ = h.read_profile()
    h.profile(False)
    return [rec[0] for rec in recs]


def test_auto_routes_each_system_to_its_kernel():
    """SROM_MIXED_AUTO without measurements: the tensor-core kernel from n = 320 up, the
    CUDA-core kernel below, both in one call; every system within 1e-10 of x_ref."""
    from staccato_b200 import _capi as CA

    h = CA.Handle(0)
    try:
        roms = [_random_rom(200, 2, 41, F=4), _random_rom(400, 3, 42, F=3), _random_rom(130, 1, 43, F=5)]
        devs = [DeviceRom.from_host(r.K, r.M, r.D, r.rhs, r.omega) for r in roms]
        names = _kernels(h, lambda: sweep(h, devs, precision=CA.SROM_MIXED_AUTO, flags=FALLBACK))
        assert "mixed_tc" in names and "mixed_global" in names, names
        for r, d in zip(roms, devs):
            xr = O.x_ref(r.K, r.M, r.D, 0.0, r.rhs, r.omega)
            assert O.rel_err(d.solutions(), xr).max() <= 1e-10
            assert (d.steps.cpu().numpy() >= 1).all()
    finally:
        h.close()


def test_auto_shared_fallback_is_the_fp64_solve():
    """With a tolerance no correction can meet, every system of both mixed kernels goes to the
    shared FP64 re-solve list: the results are the FP64 form's, bit for bit, steps = -1."""
    from staccato_b200 import _capi as CA

    h = CA.Handle(0)
    try:
        roms = [_random_rom(150, 2, 51, F=3), _random_rom(420, 2, 52, F=2)]
        devs = [DeviceRom.from_host(r.K, r.M, r.D, r.rhs, r.omega) for r in roms]
        names = _kernels(h, lambda: sweep(h, devs, precision=CA.SROM_MIXED_AUTO, max_refine=1, tol=1e-300,
                                          flags=FALLBACK))
        assert {"mixed_tc", "mixed_global", "fp64_fallback"} <= set(names), names
        for r, d in zip(roms, devs):
            Xo, _ = O.sweep(r.K, r.M, r.D, 0.0, r.rhs, r.omega)
            assert np.array_equal(np.ascontiguousarray(d.solutions()).view(np.uint64),
                                  np.ascontiguousarray(Xo).view(np.uint64))
            assert (d.steps.cpu().numpy() == -1).all()
    finally:
        h.close()


def test_auto_follows_the_tuner(tmp_path):
    """srom_tune records the faster mixed kernel per (n, r) (JSON entries of precision "auto")
    and SROM_MIXED_AUTO uses that choice."""
    import json

    from staccato_b200 import _capi as CA
    from staccato_b200.sweep import tune

    h = CA.Handle(0)
    try:
        cache = tmp_path / "tune.json"
        tune(h, [128, 448], r=2, cache_path=str(cache))
        auto = {e["n"]: e for e in json.loads(cache.read_text())["entries"] if e["precision"] == "auto"}
        assert set(auto) == {128, 448}
        for n, e in auto.items():
            assert e["kernel"] in ("tensor_core", "cuda_core") and e["ms_cuda_core"] > 0 and e["ms_tensor_core"] > 0
            assert (e["kernel"] == "tensor_core") == (e["ms_tensor_core"] < e["ms_cuda_core"])
            rom = _random_rom(n, 2, 60 + n, F=3)
            d = DeviceRom.from_host(rom.K, rom.M, rom.D, rom.rhs, rom.omega)
            names = _kernels(h, lambda: sweep(h, [d], precision=CA.SROM_MIXED_AUTO, flags=FALLBACK))
            assert ("mixed_tc" in names) == (e["kernel"] == "tensor_core"), (n, names)
            xr = O.x_ref(rom.K, rom.M, rom.D, 0.0, rom.rhs, rom.omega)
            assert O.rel_err(d.solutions(), xr).max() <= 1e-10
    finally:
        h.close()
