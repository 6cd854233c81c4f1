#!/usr/bin/env python
"""Benchmark of the batched reduced-order frequency sweep on one (or N) B200.

Metric: frequency-solves per second at <= 1e-10 relative error, mixed precision + FP64
refinement versus plain FP64.  One "step" is one full sweep of the batching workload:
64 seeded ROMs, n ~ U[24, 512], F ~ U[1000, 4000] frequencies over 1..2000 Hz, 1 or 4
right-hand sides (164,933 systems, 12.8 TFLOP of complex LU + solve per step).  Inputs
(167 MB of ROM matrices) and outputs (1.6 GB of solutions) are larger than the 126 MB L2,
so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank sweeps its own batch of 64 ROMs drawn from the same distribution
(weak scaling, no collective on the data path); the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "freq-solves/s at <=1e-10 rel err: mixed+refine vs plain FP64, 1 B200"
WORKLOAD = ("batching: 64 ROMs, n~U[24,512], F~U[1000,4000] over 1-2000 Hz, r in {1,4}, "
            "hysteretic eta=0.02, seed 3")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--precision", choices=["both", "mixed", "mixed_tc", "mixed_fp32", "fp64"], default="both",
                   help="both: headline = mixed+refine with each system on the faster mixed kernel "
                        "(SROM_MIXED_AUTO), plain FP64, and the tensor-core and CUDA-core mixed "
                        "kernels on every system measured beside it")
    p.add_argument("--cpu-sample-stride", type=int, default=16,
                   help="CPU baseline sweeps every k-th frequency of every ROM")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the projection and adjoint side measurements")
    return p.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def workload_stats(roms):
    n = np.array([r.n for r in roms], dtype=np.float64)
    F = np.array([r.F for r in roms], dtype=np.float64)
    r = np.array([r.r for r in roms], dtype=np.float64)
    flops = float(((8.0 / 3.0) * n ** 3 + 8.0 * n ** 2 * r) @ F)
    return int(F.sum()), flops


# ----------------------------------------------------------------------------- clocks

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        rows = []
        for line in (getattr(self, "out", "") or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = np.array([r[0] for r in rows])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k, v in enumerate(r[2]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(r[1] for r in rows)),
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------------------- peaks

# DRAM bytes (read + write) per launch of the dominant kernel of a form on this bench's default
# workload (the 64-ROM batching draw of rank 0), keyed by (form, kernel).  The CUDA-core and FP64
# global kernels: a one-pass ncu capture of dram__bytes_read.sum + dram__bytes_write.sum over
# `bench.py --steps 1 --warmup 3 --no-cpu-baseline --no-e2e --no-extras` (mean of 4 launches;
# the CUDA-core kernel then took every system of the mixed form, as it does in mixed_fp32).
MEASURED_TRAFFIC = {("mixed_fp32", "mixed_global"): 574.5e9 + 460.1e9, ("fp64", "fp64_global"): 1757.4e9 + 1803.5e9}
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, one-pass capture of this "
                  "workload; compare with the bytes the matrices alone need (8 n^2 B per FP32 system, "
                  "16 n^2 B per FP64 system)")
# The tensor-core kernel of the headline (SROM_MIXED_AUTO) sweep: the same metrics captured on a
# small case, every 16th frequency of every ROM of the same batch (same n / r mix, autotuned the
# same way; one launch of 5,271 systems and 0.717 TFLOP), scaled to a full launch by its flops.
TC_SAMPLE_BYTES = 42724239616 + 42177227776
TC_SAMPLE_FLOPS = 716926045381.0
TC_TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the tensor-core launch on every 16th "
                     "frequency of the same batch (84.9 GB for 0.717 TFLOP), scaled to this launch by its flops; "
                     "compare with 8 n^2 B per FP32 system")


# DRAM bytes (read + write) of one projection of the Tet10 block (K and M, k = 96): transpose,
# SpMM, V^T Y and the partial reduction, from a one-pass ncu capture (dram__bytes_read.sum +
# dram__bytes_write.sum) of the third projection of three; filled in from the capture.
PROJ_TRAFFIC = 784.7e6
PROJ_TRAFFIC_SOURCE = "ncu dram__bytes_read.sum + dram__bytes_write.sum summed over the launches of one projection"


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return json.load(open(path))
    except (OSError, ValueError):
        return {}


def gemm_peak_tflops(torch, dev, dtype) -> float:
    """cuBLAS GEMM 8192^3 (DGEMM for float64; SGEMM with TF32 off for float32), best of 5
    (CUDA events): the FP64 / FP32-FMA denominators, measured in-run because only the HBM
    and bf16 rates are in the measured-peaks file."""
    n = 8192
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    a = torch.randn(n, n, dtype=dtype, device=dev)
    b = torch.randn(n, n, dtype=dtype, device=dev)
    torch.matmul(a, b)
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    torch.cuda.empty_cache()
    torch.backends.cuda.matmul.allow_tf32 = prev
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


# ----------------------------------------------------------------------------- CPU legs

def all_systems_error(torch, drom, x64):
    """Relative 2-norm difference (all right-hand sides of a system together) of every system's
    solution from the FP64 form's solution of the same system, computed on the device.  The FP64
    kernel is bit-identical to the oracle's zgetrf/zgetrs, so this compares the mixed form with
    the FP64 oracle on all systems of the step.  Returns the summary and the per-system errors."""
    errs = []
    for d, x in zip(drom, x64):
        a = d.X.view(d.F, d.r * d.n)
        b = x.view(d.F, d.r * d.n)
        errs.append(torch.linalg.vector_norm(a - b, dim=1) / torch.linalg.vector_norm(b, dim=1))
    e = torch.cat(errs)
    summary = {"systems": int(e.numel()), "max": float(e.max()), "median": float(e.median()),
               "above_1e-10": int((e > 1e-10).sum())}
    return {"summary": summary, "per_system": e.double().cpu().numpy()}


def _xref_group(task):
    """Worker: the oracle's long-double-refined solutions of one ROM at the given frequencies."""
    from oracle import oracle as O

    K, M, D, rhs, omega = task
    return O.x_ref(K, M, D, 0.0, rhs, omega)


def xref_worst(roms, drom, per_system, k_worst=32, seed=0):
    """The oracle's x_ref (FP64 LU + long-double residual refinement) for the k_worst systems that
    deviate most from the FP64 solution plus one random frequency of every ROM; returns the max
    and median relative error of the mixed form's solutions there.  Runs in a spawn pool over
    the host cores (the oracle is single-threaded)."""
    import multiprocessing as mp

    offs = np.cumsum([0] + [r.F for r in roms])
    worst = np.argsort(per_system)[::-1][:k_worst]
    rng = np.random.default_rng(seed)
    picks = {}
    for g in worst:
        i = int(np.searchsorted(offs, g, side="right") - 1)
        picks.setdefault(i, set()).add(int(g - offs[i]))
    for i, r in enumerate(roms):
        picks.setdefault(i, set()).add(int(rng.integers(r.F)))
    groups = sorted((i, sorted(fs)) for i, fs in picks.items())
    tasks = [(roms[i].K, roms[i].M, roms[i].D, roms[i].rhs, roms[i].omega[fs]) for i, fs in groups]
    procs = max(1, min(len(tasks), os.cpu_count() or 1))
    with mp.get_context("spawn").Pool(procs) as pool:
        refs = pool.map(_xref_group, tasks, chunksize=1)
    from oracle import oracle as O

    errs = []
    for (i, fs), xr in zip(groups, refs):
        X = drom[i].solutions()[fs]
        errs.append(O.rel_err(X, xr))
    e = np.concatenate(errs)
    return {"systems": int(e.size), "max": float(e.max()), "median": float(np.median(e)),
            "selection": f"the {k_worst} systems farthest from the FP64 solution and one random frequency per ROM",
            "gate_1e-10": bool(e.max() <= 1e-10)}


def cpu_sample(roms, stride):
    """Every stride-th frequency of every ROM (same n / r mix as the full workload)."""
    return [(i, np.arange(0, rom.F, stride)) for i, rom in enumerate(roms)]


def run_cpu_sweep(roms, sample, threads=0):
    from oracle import oracle as O

    t0 = time.perf_counter()
    total = 0
    outs = []
    for i, idx in sample:
        rom = roms[i]
        om = np.ascontiguousarray(rom.omega[idx])
        X = O.cpu_sweep(rom.K, rom.M, rom.D, 0.0, rom.rhs, om, 0, len(om), threads)
        outs.append(X)
        total += len(om)
    dt = time.perf_counter() - t0
    return total, dt, outs


def cpu_baseline_leg(roms, stride, gpu_solutions):
    """Time the CPU restatement on a bounded sample; check GPU accuracy on the same systems."""
    from oracle import oracle as O

    L = O.cpu_lib()
    cores = int(L.cpu_baseline_default_threads())
    sample = cpu_sample(roms, stride)
    total, dt, outs = run_cpu_sweep(roms, sample, threads=cores)
    kind = "port"
    lapack = "OpenBLAS LAPACKE zgetrf/zgetrs" if L.cpu_baseline_using_lapacke() else "restated unblocked zgetrf/zgetrs"
    base = {"value": total / dt, "unit": "freq-solves/s", "cores": cores, "kind": kind,
            "sample": f"every {stride}th frequency of all 64 ROMs ({total} systems, {dt:.1f} s), {lapack}, "
                      f"threaded over frequencies"}
    # the reference publishes a single-thread row beside the all-cores one: the same sweep on one
    # host thread, over every 4th frequency of this sample (same n / r mix)
    st_sample = cpu_sample(roms, stride * 4)
    t1, d1, _ = run_cpu_sweep(roms, st_sample, threads=1)
    base["single_thread"] = {"value": t1 / d1, "unit": "freq-solves/s", "cores": 1,
                             "sample": f"every {stride * 4}th frequency of all 64 ROMs ({t1} systems, {d1:.1f} s)"}
    acc = None
    if gpu_solutions is not None:
        errs_cpu, errs_ref = [], []
        rng = np.random.default_rng(0)
        for (i, idx), Xc in zip(sample, outs):
            Xg = gpu_solutions(i, idx)
            errs_cpu.append(O.rel_err(Xg, Xc))
            pick = rng.choice(len(idx), size=1, replace=False)
            rom = roms[i]
            xr = O.x_ref(rom.K, rom.M, rom.D, 0.0, rom.rhs, rom.omega[idx[pick]])
            errs_ref.append(O.rel_err(Xg[pick], xr))
        e_cpu = np.concatenate(errs_cpu)
        e_ref = np.concatenate(errs_ref)
        acc = {"vs_cpu_fp64_max": float(e_cpu.max()), "vs_xref_max": float(e_ref.max()),
               "vs_xref_median": float(np.median(e_ref)), "checked_systems": int(e_ref.size),
               "gate_1e-10": bool(e_ref.max() <= 1e-10)}
    return base, acc


# ----------------------------------------------------------------------------- side legs

def projection_leg(torch, dev, h, peaks, reps=5):
    """V^T K V and V^T M V on the 107,163-DOF Tet10 block (k = 96) and the FP64 Gram-Schmidt
    of the basis: device time and algorithmic HBM bytes (values + colind + rowptr + V once)."""
    from staccato_b200 import fe_tet10
    from staccato_b200.project import DeviceCsr, orthonormalize, project

    m = fe_tet10.clamped_block()
    k = 96
    V0 = fe_tet10.basis(m.n_dof, k, seed=1)
    Vt = torch.from_numpy(np.ascontiguousarray(V0.T)).to(dev)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    orthonormalize(h, Vt.clone(), passes=2)
    e0.record(stream)
    orthonormalize(h, Vt, passes=2)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    gs_ms = e0.elapsed_time(e1)
    csr = DeviceCsr.from_host(m.indptr, m.indices)
    Kv = torch.from_numpy(m.K).to(dev)
    Mv = torch.from_numpy(m.M).to(dev)
    project(h, csr, [Kv, Mv], Vt)
    torch.cuda.synchronize(dev)
    h.profile(True)
    h.read_profile()
    e0.record(stream)
    for _ in range(reps):
        project(h, csr, [Kv, Mv], Vt)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    h.profile(False)
    recs, _ = h.read_profile()
    ms = e0.elapsed_time(e1) / reps
    nnz, N = int(m.indices.shape[0]), m.n_dof
    alg_bytes = 2 * 8 * nnz + 4 * nnz + 8 * (N + 1) + 8 * N * k
    flops = 2 * (2 * nnz * k) + 2 * (2 * N * k * k)
    kms = {}
    for name, t, *_ in recs:
        kms[name] = kms.get(name, 0.0) + t / reps
    hbm = float(peaks.get("hbm_gbs", 0.0)) or None
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    # The arithmetic bound is the tighter one: 7.2 GFLOP of FP64 (SpMM on the CUDA cores, V^T Y
    # on the FP64 tensor cores) against 254 MB of algorithmic bytes, i.e. 28 FLOP/B, above the
    # machine balance of DGEMM-rate / copy-bandwidth (about 5.4 FLOP/B).
    p64 = gemm_peak_tflops(torch, dev, torch.float64)
    tf = flops / (ms * 1e-3) / 1e12
    spmm_fl, vty_fl = 2 * (2 * nnz * k), 2 * (2 * N * k * k)
    return {"workload": "Tet10 block 10x10x40, h=0.01 m, steel, z=0 clamped; N=107,163, nnz=%d; V 107,163 x 96 seeded N(0,1)" % nnz,
            "ms_per_projection": ms, "kernels_ms": kms, "gram_schmidt_ms": gs_ms,
            "roofline": {"bound": "fp64", "achieved": tf, "peak": p64, "unit": "TFLOP/s", "frac": tf / p64,
                         "traffic": PROJ_TRAFFIC, "traffic_source": PROJ_TRAFFIC_SOURCE,
                         "algorithmic_flops": flops,
                         "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 is not in MEASURED_PEAKS.json)",
                         "kernels_tflops": {"spmm": spmm_fl / (kms.get("spmm", 0.0) * 1e-3) / 1e12
                                            if kms.get("spmm") else None,
                                            "vty_dmma": vty_fl / (kms.get("vty_dmma", 0.0) * 1e-3) / 1e12
                                            if kms.get("vty_dmma") else None}},
            "roofline_hbm": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                             "frac": (achieved / hbm) if hbm else None, "algorithmic_bytes": alg_bytes,
                             "peak_source": "MEASURED_PEAKS.json hbm_gbs (copy bandwidth)"},
            "fp64_tflops": tf}


def adjoint_leg(torch, dev, h):
    """Forward FP64 sweep with kept factors + backward call on the differentiation workload
    (n = 128, 2000 frequencies, 16 stiffness scales + loss factor).  forward_ms includes the
    host-to-device copy of the ROM and J's evaluation; backward_ms is the backward call alone."""
    from staccato_b200 import workloads as W
    from staccato_b200.adjoint import backward, forward_J, modal_params

    prob = W.adjoint_rom()
    params = modal_params(prob, device=dev)
    J0, gbar, d = forward_J(h, prob, keep=True, device=dev)
    backward(h, d, gbar, params)
    torch.cuda.synchronize(dev)
    del d, gbar  # the timed call reuses their memory (kept factors: 2000 x 128^2 complex128)
    stream = torch.cuda.current_stream(dev)
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record(stream)
    J0, gbar, d = forward_J(h, prob, keep=True, device=dev)
    e1.record(stream)
    g = backward(h, d, gbar, params)
    e2.record(stream)
    torch.cuda.synchronize(dev)
    fwd, bwd = e0.elapsed_time(e1), e1.elapsed_time(e2)
    # central difference of J in p_0 and eta (relative step 1e-6) against the adjoint
    gh = g.cpu().numpy()
    hp = 1e-6
    pp, pm = prob.p.copy(), prob.p.copy()
    pp[0] += hp
    pm[0] -= hp
    fd0 = (forward_J(h, prob, p=pp, device=dev)[0] - forward_J(h, prob, p=pm, device=dev)[0]) / (2 * hp)
    return {"workload": "n=128, 2000 freq 1-1500 Hz, 16 stiffness scales + eta, J = sum |c^H x|^2",
            "forward_ms": fwd, "backward_ms": bwd, "backward_freq_per_s": prob.rom.F / (bwd * 1e-3),
            "grad_p0": float(gh[0]), "fd_p0": float(fd0), "rel_diff_p0": float(abs(gh[0] - fd0) / abs(fd0))}


def workloads_leg(torch, dev, h, reps=3):
    """Every form on the single-ROM workloads beside the batching one: plain (n = 64, 500
    frequencies, r = 1) and precision (n = 256, 4096 frequencies, 60 % within 0.1 % of an
    eigenfrequency, r = 8, damping D); mixed = SROM_MIXED_AUTO (untuned for these orders: the
    CUDA-core kernel below n = 320).  Device time per sweep (median of reps), freq-solves/s, and
    for the mixed forms the error against the oracle's refined x_ref on every 16th frequency."""
    from oracle import oracle as O
    from staccato_b200 import _capi, workloads as W
    from staccato_b200.sweep import DeviceRom, sweep

    stream = torch.cuda.current_stream(dev)
    out = {}
    for name, rom in (("plain_n64", W.plain_rom()), ("precision_n256", W.precision_rom())):
        d = DeviceRom.from_host(rom.K, rom.M, rom.D, rom.rhs, rom.omega, device=dev)
        res = {"n": rom.n, "F": rom.F, "r": int(rom.rhs.shape[1])}
        for form, prec, flags in (("fp64", _capi.SROM_FP64, 0),
                                  ("mixed_tc", _capi.SROM_MIXED_TC, _capi.SROM_FLAG_FALLBACK_FP64),
                                  ("mixed_fp32", _capi.SROM_MIXED_FP32, _capi.SROM_FLAG_FALLBACK_FP64),
                                  ("mixed", _capi.SROM_MIXED_AUTO, _capi.SROM_FLAG_FALLBACK_FP64)):
            sweep(h, [d], precision=prec, flags=flags)
            ts = []
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                sweep(h, [d], precision=prec, flags=flags)
                e1.record(stream)
                torch.cuda.synchronize(dev)
                ts.append(e0.elapsed_time(e1))
            ms = float(np.median(ts))
            res[form] = {"ms": ms, "freq_solves_per_s": rom.F / (ms * 1e-3)}
            if form != "fp64":
                sel = slice(None, None, 16)
                X = d.solutions()[sel]
                Xr = O.x_ref(rom.K, rom.M, rom.D, 0.0, rom.rhs, rom.omega[sel])
                err = O.rel_err(X, Xr)
                res[form]["max_rel_err"] = float(err.max())
                st = d.steps.cpu().numpy()
                res[form]["refine_steps_hist"] = {str(k): int(v) for k, v in zip(*np.unique(st, return_counts=True))}
        for form in ("mixed", "mixed_tc", "mixed_fp32"):
            res[form + "_vs_plain"] = res[form]["freq_solves_per_s"] / res["fp64"]["freq_solves_per_s"]
        out[name] = res
    return out


REFERENCE_PER_OMEGA_MS = {
    # test/krylovTestGPU/matrixInSingleLoop/timeMeasurements.txt:6 (GPU, sm_70) and :12 (MKL, 20 threads)
    21: {"gpu_sm70_ms": 0.380, "mkl_20thr_ms": 0.051},
    189: {"gpu_sm70_ms": 2.087, "mkl_20thr_ms": 40.6},
    2520: {"gpu_sm70_ms": 41.26, "mkl_20thr_ms": 230.1},
}


def reference_orders_leg(torch, dev, h, reps=2):
    """The reference's own dense ROM orders (r21, r189, r2520; 1 RHS; hysteretic eta = 0.02
    ROMs built like the plain workload): device time per frequency of the FP64 sweep (and of
    the mixed form, which at n = 2520 is the FP64 kernel), beside the reference's published
    per-frequency times.  n = 2520 runs 296 frequencies (two per SM); the others 1000.
    Accuracy at n = 2520: normwise backward error ||A x - b|| / (||A|| ||x|| + ||b||) of four
    frequencies, in FP64 with torch."""
    from staccato_b200 import _capi, workloads as W
    from staccato_b200.sweep import DeviceRom, sweep

    stream = torch.cuda.current_stream(dev)
    out = {}
    for n, F in ((21, 1000), (189, 1000), (2520, 296)):
        rom = W.plain_rom(seed=21 + n, n=n, F=F)
        d = DeviceRom.from_host(rom.K, rom.M, rom.D, rom.rhs, rom.omega, device=dev)
        res = {"n": n, "F": F, "r": 1, "reference": REFERENCE_PER_OMEGA_MS[n]}
        for form, prec, flags in (("fp64", _capi.SROM_FP64, 0),
                                  ("mixed", _capi.SROM_MIXED_AUTO, _capi.SROM_FLAG_FALLBACK_FP64)):
            sweep(h, [d], precision=prec, flags=flags)
            ts = []
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                sweep(h, [d], precision=prec, flags=flags)
                e1.record(stream)
                torch.cuda.synchronize(dev)
                ts.append(e0.elapsed_time(e1))
            ms = float(np.median(ts))
            res[form] = {"ms": ms, "ms_per_omega": ms / F, "freq_solves_per_s": F / (ms * 1e-3),
                         "tflops": (8.0 / 3.0 * n ** 3 + 8.0 * n * n) * F / (ms * 1e-3) / 1e12,
                         "vs_reference_gpu": REFERENCE_PER_OMEGA_MS[n]["gpu_sm70_ms"] / (ms / F)}
        if n == 2520:
            K = torch.from_numpy(rom.K).to(dev)
            M = torch.from_numpy(rom.M).to(dev)
            b = torch.from_numpy(np.ascontiguousarray(rom.rhs[:, 0])).to(dev)
            X = torch.from_numpy(np.ascontiguousarray(d.solutions())).to(dev)
            be = []
            for f in (0, 97, 201, F - 1):
                w = float(rom.omega[f])
                A = K - (w * w) * M
                x = X[f].reshape(-1)
                rr = torch.linalg.vector_norm(A @ x - b)
                den = torch.linalg.matrix_norm(A, ord=float("inf")) * torch.linalg.vector_norm(x, ord=float("inf")) \
                    + torch.linalg.vector_norm(b, ord=float("inf"))
                be.append(float(rr / den))
            res["backward_error_max"] = max(be)
            del K, M, b, X
        out[f"r{n}"] = res
        del d
        torch.cuda.empty_cache()
    return out


def krylov_leg(torch, dev, h):
    """Krylov basis generation (srom_krylov_basis) on the Tet10 block of the projection leg
    (10 x 10 x 40 hexes, z = 0 face clamped and removed, N = 105,840): D = 1e-5 K + 2 M, four
    unit-scaled point loads, one expansion point of order 1 and two points (100, 800 Hz) of
    order 4.  Wall time of the call (it synchronises: host ordering, band factorisation of K~
    per point, solves, re-orthogonalisation, pivoted QR) and the band factor's size.  The timed
    calls follow a warm-up call on the same pattern, whose full pattern and RCM order the handle
    keeps (`pattern_reused`); `first_call_s` is the warm-up call, which orders the pattern."""
    import scipy.sparse as sp

    from staccato_b200 import fe_tet10
    from staccato_b200.krylov import band_cache_report, band_order, krylov_basis
    from staccato_b200.project import DeviceCsr

    m = fe_tet10.clamped_block(10, 10, 40)
    keep = ~m.clamped
    K = sp.csr_matrix((m.K, m.indices, m.indptr), shape=(m.n_dof, m.n_dof))[keep][:, keep].tocsr()
    M = sp.csr_matrix((m.M, m.indices, m.indptr), shape=(m.n_dof, m.n_dof))[keep][:, keep].tocsr()
    K.sort_indices()
    M.sort_indices()
    n = K.shape[0]
    _, bw, band_b = band_order(K.indptr, K.indices)
    rng = np.random.default_rng(0)
    B = np.zeros((n, 4), dtype=np.complex128)
    B[rng.choice(n, 4, replace=False), np.arange(4)] = 1e9
    c = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.complex128)).to(dev)
    csr = DeviceCsr.from_host(K.indptr, K.indices, device=dev)
    Kd, Md, Dd, Bd = c(K.data), c(M.data), c(1e-5 * K.data + 2.0 * M.data), c(B.T)
    out = {"workload": "Tet10 block 10x10x40, N=%d, nnz=%d, 4 inputs" % (n, K.nnz), "bandwidth": bw,
           "band_gb": band_b / 1e9, "solver": "band LDL^T (RCM order), trailing and solve updates on the library's complex FP64 tensor-core GEMM"}
    for name, pts, order in (("one_point_order1", [100.0], 1), ("two_points_order4", [100.0, 800.0], 4)):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        krylov_basis(h, csr, Kd, Md, Dd, Bd, pts, order)  # warm-up
        torch.cuda.synchronize(dev)
        first = time.perf_counter() - t0
        t0 = time.perf_counter()
        V = krylov_basis(h, csr, Kd, Md, Dd, Bd, pts, order)
        torch.cuda.synchronize(dev)
        out[name] = {"s": time.perf_counter() - t0, "columns": int(V.shape[0]), "first_call_s": first,
                     "pattern_reused": band_cache_report(h)[0]}
    out["factor_tflop"] = 8.0 * n * bw * bw / 1e12
    # full-order direct sweep (performSolveFOM) at two frequencies, the four loads at once
    from staccato_b200.krylov import fom_sweep

    fom_sweep(h, csr, Kd, Md, Dd, Bd, [500.0])  # warm-up
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    fom_sweep(h, csr, Kd, Md, Dd, Bd, [300.0, 900.0])
    torch.cuda.synchronize(dev)
    out["fom_sweep_s_per_freq"] = (time.perf_counter() - t0) / 2
    return out


def coupling_leg(torch, dev, h):
    """Interface-Jacobian coupling of substructures (staccato_b200.ijcsa.couple; the reference's
    coupling program test/IJCSA/src/IJSA.cu): two substructures (n = 200 and 240, 12 interface
    DOFs, hysteretic damping 0.02, a unit load on the first) coupled by compatibility and
    equilibrium at 2000 frequencies: FP64 sweeps of the interface FRFs, the interface Jacobian
    and residual on the library's batched complex GEMM, the batched solve.  Wall time of the
    synchronised call after a warm-up and the largest residual norm."""
    from staccato_b200.ijcsa import SimulationModel, couple

    rng = np.random.default_rng(11)

    def spd(n, scale):
        A = rng.standard_normal((n, n))
        return scale * (A @ A.T / n + np.eye(n))

    n1, n2, p, nf = 200, 240, 12, 2000
    K1, M1, K2, M2 = spd(n1, 1e4), spd(n1, 1.0), spd(n2, 2e4), spd(n2, 1.5)
    B1 = np.zeros((n1, p))
    B1[n1 - p:, :] = np.eye(p)
    B2 = np.zeros((n2, p))
    B2[:p, :] = np.eye(p)
    load = np.zeros((n1, 1))
    load[2, 0] = 1.0
    s1 = SimulationModel(K=K1.astype(complex), M=M1.astype(complex), B_if=B1, C_if=B1.T, eta=0.02, B_load=load,
                         F=np.ones(1))
    s2 = SimulationModel(K=K2.astype(complex), M=M2.astype(complex), B_if=B2, C_if=B2.T, eta=0.02)
    I, Z = np.eye(p), np.zeros((p, p))
    dRdY = [np.vstack([I, Z]), np.vstack([-I, Z])]  # compatibility: Y1 - Y2 = 0
    dRdU = [np.vstack([Z, I]), np.vstack([Z, I])]   # equilibrium: U1 + U2 = 0
    freq = np.linspace(1.0, 400.0, nf)
    couple(h, [s1, s2], dRdY, dRdU, freq)  # warm-up
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    _, _, rn = couple(h, [s1, s2], dRdY, dRdU, freq)
    torch.cuda.synchronize(dev)
    sec = time.perf_counter() - t0
    return {"workload": "2 substructures (n = 200, 240), 12 interface DOFs, 2000 frequencies, FP64",
            "s": sec, "freq_per_s": nf / sec, "residual_norm_max": float(rn.abs().max().item())}


# ----------------------------------------------------------------------------- arms

def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from staccato_b200 import workloads as W

    roms = W.batching_roms()
    stride = args.cpu_sample_stride
    sample = cpu_sample(roms, stride)
    from oracle import oracle as O

    cores = int(O.cpu_lib().cpu_baseline_default_threads())
    for _ in range(args.warmup):
        run_cpu_sweep(roms, sample[:2], cores)
    times, total = [], 0
    for _ in range(args.steps):
        total, dt, _ = run_cpu_sweep(roms, sample, cores)
        times.append(dt)
    dt = float(np.mean(times))
    value = total / dt
    lapack = ("OpenBLAS LAPACKE zgetrf/zgetrs" if O.cpu_lib().cpu_baseline_using_lapacke()
              else "restated unblocked zgetrf/zgetrs")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "freq-solves/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "step": f"every {stride}th frequency of all 64 ROMs ({total} systems)"},
        "cpu_baseline": {"value": value, "unit": "freq-solves/s", "cores": cores, "kind": "port",
                         "sample": f"{total} systems per step; {lapack}; the reference's MKL build is not "
                                   f"available (no MKL), this is the C restatement of its host sweep"},
        "e2e": {"value": value, "unit": "freq-solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch

    rank, world, local = dist_env()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist

    from staccato_b200 import _capi, dist as D, workloads as W
    from staccato_b200.sweep import DeviceRom, HostRom, sweep, sweep_host, tune

    # weak scaling: every rank sweeps its own 64-ROM batch of the same distribution
    # (rank 0 is the named workload, seed 3); no collective touches the data path
    roms = W.batching_roms(seed=D.rank_seed(3, rank))
    systems, flops = workload_stats(roms)
    h = _capi.Handle(local)
    stream = torch.cuda.current_stream(dev)
    h.set_stream(stream.cuda_stream)
    drom = [DeviceRom.from_host(r.K, r.M, r.D, r.rhs, r.omega, device=dev) for r in roms]
    # the autotuned schedule: srom_tune measures the kernel choices of every (n, r) of the batch
    # (FP64 smem vs global kernel; the mixed form's FP64-outright vs mixed-kernel routing)
    t_tune = time.time()
    for rr in sorted({r.r for r in roms}):
        tune(h, sorted({r.n for r in roms if r.r == rr}), r=rr)
    tune_s = time.time() - t_tune
    FORMS = {"fp64": (_capi.SROM_FP64, 0),
             "mixed_tc": (_capi.SROM_MIXED_TC, _capi.SROM_FLAG_FALLBACK_FP64),
             "mixed_fp32": (_capi.SROM_MIXED_FP32, _capi.SROM_FLAG_FALLBACK_FP64),
             "mixed": (_capi.SROM_MIXED_AUTO, _capi.SROM_FLAG_FALLBACK_FP64)}
    forms = {"both": ["fp64", "mixed_tc", "mixed_fp32", "mixed"], "mixed": ["mixed"], "mixed_tc": ["mixed_tc"],
             "mixed_fp32": ["mixed_fp32"], "fp64": ["fp64"]}[args.precision]
    headline = forms[-1]
    x64 = None  # FP64 solutions of every system (device), the comparator of the mixed forms

    def barrier():
        if pg is not None:
            pg.barrier()

    results = {}
    clk = None
    nrec_total = 0
    for form in forms:
        precision, flags = FORMS[form]
        for _ in range(args.warmup):
            sweep(h, drom, precision=precision, flags=flags)
        torch.cuda.synchronize(dev)
        h.profile(True)
        h.read_profile()
        with ClockSampler(local) as c:
            barrier()
            torch.cuda.synchronize(dev)
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            for _ in range(args.steps):
                sweep(h, drom, precision=precision, flags=flags)
            t1.record(stream)
            torch.cuda.synchronize(dev)
            barrier()
        h.profile(False)
        ms = t0.elapsed_time(t1) / args.steps
        recs, nrec = h.read_profile()
        nrec_total += nrec
        if pg is not None:
            t = torch.tensor([ms], dtype=torch.float64, device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            ms = float(t.item())
        per = {}
        for name, kms, items, kfl, kby in recs:
            a = per.setdefault(name, [0.0, 0, 0.0, 0])
            a[0] += kms
            a[1] += items
            a[2] += kfl
            a[3] += 1
        steps_hist = None
        acc_all = None
        if form == "fp64":
            x64 = [d.X.clone() for d in drom]
        else:
            st = np.concatenate([d.steps.cpu().numpy() for d in drom])
            steps_hist = {str(k): int(v) for k, v in zip(*np.unique(st, return_counts=True))}
            if x64 is not None:
                acc_all = all_systems_error(torch, drom, x64)
        results[form] = {"ms": ms, "value": systems * world / (ms * 1e-3), "per": per, "steps": steps_hist,
                         "accuracy_all": acc_all}
        if form == headline:
            clk = c

    ms = results[headline]["ms"]
    value = results[headline]["value"]
    nrec = nrec_total

    def roofline(form, peak, peak_source):
        per = results[form]["per"]
        dom = max(per, key=lambda k: per[k][0])
        kms, kitems, kfl, kl = per[dom]
        achieved = kfl / (kms * 1e-3) / 1e12
        tot = sum(x[0] for x in per.values())
        traffic, tsource = MEASURED_TRAFFIC.get((form, dom)), TRAFFIC_SOURCE
        if form == "mixed" and dom == "mixed_tc" and kl > 0:
            traffic, tsource = TC_SAMPLE_BYTES * (kfl / kl) / TC_SAMPLE_FLOPS, TC_TRAFFIC_SOURCE
        return {"bound": "tensor", "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
                "traffic_source": tsource, "kernel": dom,
                "peak_source": peak_source,
                "algorithmic": "8/3 n^3 + 8 n^2 r real flops per system (LU + solve, both forms)",
                "kernels": {k: {"ms_per_launch": v[0] / v[3], "launches": v[3],
                                "tflops": (v[2] / (v[0] * 1e-3) / 1e12) if v[0] > 0 else 0.0,
                                "share": v[0] / tot if tot > 0 else 0.0} for k, v in per.items()}}

    info = {}
    if rank == 0:
        if "fp64" in results:
            p64 = gemm_peak_tflops(torch, dev, torch.float64)
            info["roofline_fp64"] = roofline("fp64", p64, "cuBLAS DGEMM 8192^3 measured in this run (FP64 is not in MEASURED_PEAKS.json)")
        bf16 = measured_peaks().get("bf16_tflops_sustained")
        tpeak, tsrc = ((float(bf16), "MEASURED_PEAKS.json bf16_tflops_sustained (dense bf16 tensor rate under "
                                     "the power cap)") if bf16 else
                       (1400.0, "fallback: 1.4 PFLOP/s sustained dense bf16 (no MEASURED_PEAKS.json)"))
        p32 = gemm_peak_tflops(torch, dev, torch.float32) if ("mixed" in results or "mixed_fp32" in results) else None
        for form in ("mixed", "mixed_fp32"):
            if form in results:
                # Against the GPU's compute ceiling (its tensor cores, sustained dense bf16: the
                # launch lasts over a second); the CUDA-core kernel's FP32 arithmetic is compared
                # with the FP32 rate (cuBLAS SGEMM measured in this run) as well.
                rm = roofline(form, tpeak, tsrc)
                rm["peak_fp32_cuda_cores"] = p32
                rm["frac_of_fp32_cuda_cores"] = rm["achieved"] / p32
                rm["peak_fp32_cuda_cores_source"] = "cuBLAS SGEMM 8192^3, TF32 off, measured in this run"
                info["roofline_" + form] = rm
        if "mixed_tc" in results:
            # Tensor-core form: Schur updates as tcgen05 MMAs; achieved counts algorithmic flops
            # (8/3 n^3 + 8 n^2 r), the tensor pipe executes six bf16 piece products per FP32
            # multiply-add of the Schur updates on top of them.
            rt = roofline("mixed_tc", tpeak, tsrc)
            rt["tensor_work_note"] = ("Schur updates run as six bf16 piece products per FP32 multiply-add "
                                      "(three-piece splits); panels, interchanges, solves and FP64 refinement "
                                      "on CUDA cores")
            info["roofline_mixed_tc"] = rt
        info["roofline"] = info.get("roofline_mixed") or info.get("roofline_fp64")
    precision = FORMS[headline][0]
    pflags = FORMS[headline][1]

    # the headline form replayed as one captured CUDA graph (srom_graph_create / _launch: the whole
    # batched sweep, all launches, no host work per step), timed the same way
    graph = None
    if not args.no_extras:
        from staccato_b200.sweep import Graph

        gph = Graph(h, drom, precision=FORMS[headline][0], flags=FORMS[headline][1])
        for _ in range(args.warmup):
            gph.launch(stream.cuda_stream)
        torch.cuda.synchronize(dev)
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(args.steps):
            gph.launch(stream.cuda_stream)
        g1.record(stream)
        torch.cuda.synchronize(dev)
        gms = g0.elapsed_time(g1) / args.steps
        gph.close()
        if pg is not None:  # every rank replays its own graph; the step is the slowest rank's
            t = torch.tensor([gms], dtype=torch.float64, device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            gms = float(t.item())
        graph = {"value": systems * world / (gms * 1e-3), "unit": "freq-solves/s", "ms_per_step": gms,
                 "api": "srom_graph_launch of the captured sweep (plan and metadata built once)"}

    # the oracle's x_ref on the systems farthest from the FP64 solution (and one per ROM)
    xref = None
    acc_all = results.get(headline, {}).get("accuracy_all")
    if rank == 0 and acc_all is not None and not args.no_cpu_baseline:
        xref = xref_worst(roms, drom, acc_all["per_system"])

    # end to end through the host-buffer C ABI call (pinned host memory)
    e2e = None
    if not args.no_e2e:
        def pinned(a):
            a = np.ascontiguousarray(a)
            t = torch.from_numpy(a.view(np.uint8).ravel()).pin_memory()
            return t.numpy().view(a.dtype).reshape(a.shape)

        hroms = []
        h2d = d2h = 0
        for r in roms:
            hr = HostRom(r.K, r.M, r.D, r.rhs, r.omega)
            for name in ("K", "M", "rhs", "omega", "X", "info", "steps", "berr"):
                setattr(hr, name, pinned(getattr(hr, name)))
            hroms.append(hr)
            h2d += hr.K.nbytes + hr.M.nbytes + hr.rhs.nbytes + hr.omega.nbytes
            d2h += hr.X.nbytes + hr.info.nbytes + hr.steps.nbytes + hr.berr.nbytes
        sweep_host(h, hroms, precision=precision, flags=pflags)
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            sweep_host(h, hroms, precision=precision, flags=pflags)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        ems = e0.elapsed_time(e1) / args.steps
        if pg is not None:
            t = torch.tensor([ems], dtype=torch.float64, device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            ems = float(t.item())
        e2e = {"value": systems * world / (ems * 1e-3), "unit": "freq-solves/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "api": "srom_sweep_host (host buffers in, host results out)"}

    extras = {}
    if rank == 0 and not args.no_extras:
        extras["projection"] = projection_leg(torch, dev, h, measured_peaks())
        extras["adjoint"] = adjoint_leg(torch, dev, h)
        extras["workloads"] = workloads_leg(torch, dev, h)
        extras["reference_orders"] = reference_orders_leg(torch, dev, h)
        extras["krylov"] = krylov_leg(torch, dev, h)
        try:
            extras["coupling"] = coupling_leg(torch, dev, h)
        except Exception as e:  # a side leg never takes the headline line down
            extras["coupling"] = {"error": ("%s: %s" % (type(e).__name__, e))[:300]}

    cpu = acc = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        def gpu_solutions(i, idx):
            return drom[i].solutions()[idx]

        cpu, acc = cpu_baseline_leg(roms, args.cpu_sample_stride, gpu_solutions)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "freq-solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": ({"mixed": "c64 LU (Schur updates on the tensor cores, bf16 piece splits, where that kernel is "
                                "the faster; CUDA-core FP32 elsewhere) + c128 refinement",
                      "mixed_fp32": "c64 LU + c128 refinement",
                      "mixed_tc": "c64 LU (tensor-core Schur updates on bf16 piece splits) + c128 refinement"}
                     .get(headline, "c128")),
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "systems_per_gpu": systems,
                       "tflop_per_step_per_gpu": flops / 1e12, "precision": headline,
                       "refine": "complex-FP32 LU, each system on the faster of the two mixed kernels for its (n, r) as the autotuner measured (SROM_MIXED_AUTO: the tensor-core kernel, Schur updates as tcgen05 MMAs on three-piece bf16 splits, or the CUDA-core kernel; each measured on every system beside it as mixed_tc and mixed_fp32), FP64 residuals, <=5 corrections, each right-hand side stopping once its predicted error rho*||d||/||x|| (2-norms) <= 2^-34 (or the system early once the measured contraction cannot reach it), correction solves streamed through a shared-memory strip ring, back substitution by reciprocals of diag(U), FP64 fallback; systems the FP64 shared-memory kernel holds are routed by the autotuner (FP64 outright or a mixed kernel)",
                       "l2": "inputs 167 MB + outputs 1.6 GB per step exceed L2; no flush",
                       "autotune": "srom_tune over every (n, r) of the batch before warm-up (%.1f s): FP64 smem/global "
                                   "kernel, the mixed form's FP64-outright/mixed-kernel routing of the orders the "
                                   "FP64 smem kernel holds, and tensor-core vs CUDA-core mixed kernel for n in "
                                   "96..512" % tune_s,
                       "parallelism": f"independent batch per GPU x{world} (seed 3 + 1000003*rank)"},
            "roofline": info.get("roofline"),
            "roofline_fp64": info.get("roofline_fp64"),
            "plain_fp64": ({"value": results["fp64"]["value"], "unit": "freq-solves/s",
                            "ms_per_step": results["fp64"]["ms"]} if "fp64" in results else None),
            "mixed_vs_plain": (results["mixed"]["value"] / results["fp64"]["value"]
                               if "mixed" in results and "fp64" in results else None),
            "refine_steps_hist": results.get("mixed", {}).get("steps"),
            **{form: ({"value": results[form]["value"], "unit": "freq-solves/s",
                       "ms_per_step": results[form]["ms"],
                       "vs_plain": (results[form]["value"] / results["fp64"]["value"]
                                    if "fp64" in results else None),
                       "refine_steps_hist": results[form]["steps"],
                       "accuracy_vs_fp64_all_systems": (results[form]["accuracy_all"] or {}).get("summary"),
                       "roofline": info.get("roofline_" + form)}
                      if form in results else None) for form in ("mixed_tc", "mixed_fp32")},
            "cpu_baseline": cpu,
            "accuracy": acc,
            "accuracy_vs_fp64_all_systems": (acc_all or {}).get("summary"),
            "accuracy_vs_xref": xref,
            "graph": graph,
            "e2e": e2e,
            "clocks": clk.summary(),
            "gpu_launches": int(nrec),
            "projection": extras.get("projection"),
            "adjoint": extras.get("adjoint"),
            "workloads": extras.get("workloads"),
            "reference_orders": extras.get("reference_orders"),
            "krylov": extras.get("krylov"),
            "coupling": extras.get("coupling"),
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()
    h.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
