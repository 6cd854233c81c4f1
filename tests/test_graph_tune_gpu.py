"""Captured batched sweeps (CUDA graphs) and the kernel autotuner."""
import json

import numpy as np
import pytest

from oracle import oracle as O
from staccato_b200 import _capi, workloads as W
from staccato_b200.sweep import DeviceRom, Graph, sweep, tune

pytestmark = pytest.mark.gpu


def _roms():
    roms = W.batching_roms(count=6, n_lo=24, n_hi=300, F_lo=20, F_hi=60)
    return [DeviceRom.from_host(r.K, r.M, r.D, r.rhs, r.omega) for r in roms], roms


@pytest.mark.parametrize("precision,flags", [(_capi.SROM_FP64, 0),
                                             (_capi.SROM_MIXED_FP32, _capi.SROM_FLAG_FALLBACK_FP64)])
def test_graph_replays_equal_direct_sweep(handle, precision, flags):
    import torch

    devs, host = _roms()
    sweep(handle, devs, precision=precision, flags=flags)
    torch.cuda.synchronize()
    ref = [d.solutions().copy() for d in devs]
    g = Graph(handle, devs, precision=precision, flags=flags)
    for _ in range(2):
        for d in devs:
            d.X.fill_(float("nan"))
        g.launch(torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        for d, X in zip(devs, ref):
            assert np.array_equal(d.solutions().view(np.uint64), X.view(np.uint64))
    g.close()
    if precision == _capi.SROM_FP64:
        for d, r in zip(devs, host):
            Xo, _ = O.sweep(r.K, r.M, r.D, 0.0, r.rhs, r.omega)
            assert np.array_equal(d.solutions().view(np.uint64), Xo.view(np.uint64))


def test_tune_writes_cache_and_keeps_results_exact(handle, tmp_path):
    import torch

    cache = tmp_path / "tune.json"
    tune(handle, [24, 64, 100], r=1, cache_path=str(cache))
    data = json.loads(cache.read_text())
    fp64 = [e for e in data["entries"] if e["precision"] == "fp64"]
    mixed = [e for e in data["entries"] if e["precision"] == "mixed"]
    assert data["device"] and {e["n"] for e in fp64} >= {24, 64, 100}
    assert all(e["kernel"] in ("smem", "global") for e in fp64)
    # the mixed routing is measured wherever the FP64 choice is the shared-memory kernel
    smem_n = {e["n"] for e in fp64 if e["kernel"] == "smem"}
    assert {e["n"] for e in mixed} == smem_n
    assert all(e["kernel"] in ("fp64_smem", "mixed_global") and e["ms_fp64_smem"] > 0 and e["ms_mixed_global"] > 0
               for e in mixed)
    rom = W.plain_rom(F=30)
    d = DeviceRom.from_host(rom.K, rom.M, None, rom.rhs, rom.omega)
    sweep(handle, [d])
    torch.cuda.synchronize()
    Xo, _ = O.sweep(rom.K, rom.M, None, 0.0, rom.rhs, rom.omega)
    assert np.array_equal(d.solutions().view(np.uint64), Xo.view(np.uint64))
    # the mixed form follows the tuned routing and stays within 1e-10 of x_ref (n = 64)
    dm = DeviceRom.from_host(rom.K, rom.M, None, rom.rhs, rom.omega)
    sweep(handle, [dm], precision=_capi.SROM_MIXED_FP32, flags=_capi.SROM_FLAG_FALLBACK_FP64)
    steps = dm.steps.cpu().numpy()
    routed = {e["n"]: e["kernel"] for e in mixed}.get(64)
    if routed == "fp64_smem":
        assert (steps == 0).all()
    elif routed == "mixed_global":
        assert (steps != 0).all()
    xr = O.x_ref(rom.K, rom.M, None, 0.0, rom.rhs, rom.omega)
    assert O.rel_err(dm.solutions(), xr).max() <= 1e-10
    # a second tune call reads the cache instead of timing again
    tune(handle, [24, 64, 100], r=1, cache_path=str(cache))
