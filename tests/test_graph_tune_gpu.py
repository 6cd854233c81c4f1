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
    assert data["device"] and {e["n"] for e in data["entries"]} >= {24, 64, 100}
    assert all(e["kernel"] in ("smem", "global") for e in data["entries"])
    rom = W.plain_rom(F=30)
    d = DeviceRom.from_host(rom.K, rom.M, None, rom.rhs, rom.omega)
    sweep(handle, [d])
    torch.cuda.synchronize()
    Xo, _ = O.sweep(rom.K, rom.M, None, 0.0, rom.rhs, rom.omega)
    assert np.array_equal(d.solutions().view(np.uint64), Xo.view(np.uint64))
    # a second tune call reads the cache instead of timing again
    tune(handle, [24, 64, 100], r=1, cache_path=str(cache))
