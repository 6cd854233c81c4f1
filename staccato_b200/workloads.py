"""Seeded synthetic reduced-order models (ROMs) for the frequency sweep.

The reference ships no ROM files (its tests read ``KSM_*_r{21,189,2520}.mtx`` from
``/opt/software/examples/MOR/``, which are not part of the project), so every sweep input
here is generated from a seed.  The shapes follow the five workloads the sweep is measured on:

* ``plain_rom``       n=64, hysteretic damping eta=0.02, 500 frequencies 1..1000 Hz, 1 RHS.
* ``precision_rom``   n=256, eta=0.01 + Rayleigh damping D = 1e-5 K + 2 M, 4096 frequencies of
                      which 60 % lie within +-0.1 % of generalised eigenfrequencies, 8 RHS.
* ``batching_roms``   64 ROMs, n ~ U[24, 512], F ~ U[1000, 4000] over 1..2000 Hz, r in {1, 4}.
* ``adjoint_rom``     n=128, 16 stiffness-scaling parameters over disjoint 8-mode blocks,
                      eta=0.02, 2000 frequencies 1..1500 Hz, J = sum |c^H x|^2.

A ROM holds complex column-major K_r, M_r (and optionally D_r) exactly like the reference
members ``myKComplexReduced``, ``myMComplexReduced``, ``myDComplexReduced``
(src/analysis/KrylovROMSubstructure.h:210-221).  The hysteretic factor (1 + i eta) is folded
into K_r the way the reference builds ``KComplex`` (src/analysis/KrylovROMSubstructure.cpp:330-333).
Frequencies become omega = 2 pi f as in src/analysis/KrylovROMSubstructure.cpp:1408.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

TWO_PI = 2.0 * math.pi


@dataclasses.dataclass
class Rom:
    """One reduced-order model plus its sweep request.

    Matrices are complex128, Fortran (column-major) ordered, n x n.  ``rhs`` is n x r
    column-major.  ``omega`` holds angular frequencies (rad/s).
    """

    K: np.ndarray
    M: np.ndarray
    D: Optional[np.ndarray]
    rhs: np.ndarray
    omega: np.ndarray
    seed: int = 0
    meta: dict = dataclasses.field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.K.shape[0])

    @property
    def r(self) -> int:
        return int(self.rhs.shape[1])

    @property
    def F(self) -> int:
        return int(self.omega.shape[0])


def _orthogonal(rng: np.random.Generator, n: int) -> np.ndarray:
    """Random orthogonal Q: QR of an N(0,1) matrix with the signs of diag(R) fixed."""
    g = rng.standard_normal((n, n))
    q, r = np.linalg.qr(g)
    s = np.sign(np.diag(r))
    s[s == 0] = 1.0
    return q * s[None, :]


def _sym_noise(rng: np.random.Generator, n: int) -> np.ndarray:
    """Symmetric matrix with N(0,1) entries, scaled by 1/sqrt(n)."""
    g = rng.standard_normal((n, n))
    s = np.triu(g) + np.triu(g, 1).T
    return s / math.sqrt(n)


def modal_pair(rng: np.random.Generator, n: int, f_lo: float, f_hi: float):
    """K = Q diag((2 pi f_k)^2) Q^T with f_k log-uniform in [f_lo, f_hi]; M = I + 0.01 S."""
    q = _orthogonal(rng, n)
    f = np.exp(rng.uniform(math.log(f_lo), math.log(f_hi), size=n))
    lam = (TWO_PI * f) ** 2
    k = (q * lam[None, :]) @ q.T
    k = 0.5 * (k + k.T)
    m = np.eye(n) + 0.01 * _sym_noise(rng, n)
    return q, lam, k, m


def _as_complex_f(a: np.ndarray) -> np.ndarray:
    return np.asfortranarray(np.asarray(a, dtype=np.complex128))


def hysteretic(k: np.ndarray, eta: float) -> np.ndarray:
    """(1 + i eta) K with the same per-entry rounding as the reference's K(1+eta*i) build
    (real part = K, imaginary part = K * eta; src/analysis/KrylovROMSubstructure.cpp:330-333)."""
    out = np.empty(k.shape, dtype=np.complex128, order="F")
    out.real = k
    out.imag = k * eta
    return out


def plain_rom(seed: int = 0, n: int = 64, F: int = 500, eta: float = 0.02) -> Rom:
    """n=64 plain FP64 sweep: A = (1+0.02i)K_r - w^2 M_r, 500 freqs 1..1000 Hz, one real RHS."""
    rng = np.random.default_rng(seed)
    q, lam, k, m = modal_pair(rng, n, 20.0, 2000.0)
    rhs = np.asfortranarray(rng.standard_normal((n, 1)).astype(np.complex128))
    freq = np.linspace(1.0, 1000.0, F)
    return Rom(K=hysteretic(k, eta), M=_as_complex_f(m), D=None, rhs=rhs,
               omega=TWO_PI * freq, seed=seed,
               meta={"workload": "plain", "eta": eta, "f_band_hz": [1.0, 1000.0]})


def precision_rom(seed: int = 2, n: int = 256, F: int = 4096, r: int = 8,
                  eta: float = 0.01, near_frac: float = 0.6, rel_window: float = 1e-3) -> Rom:
    """n=256 near-resonance sweep with Rayleigh damping D = 1e-5 K + 2 M.

    60 % of the frequencies sit within +-0.1 % of a random half of the generalised
    eigenfrequencies of (K_r, M_r); the rest are uniform in the modal band 10..5000 Hz.
    """
    import scipy.linalg

    rng = np.random.default_rng(seed)
    q, lam, k, m = modal_pair(rng, n, 10.0, 5000.0)
    d = 1e-5 * k + 2.0 * m
    w2 = scipy.linalg.eigh(k, m, eigvals_only=True)
    f_eig = np.sqrt(np.maximum(w2, 0.0)) / TWO_PI
    subset = np.sort(rng.choice(n, size=n // 2, replace=False))
    n_near = int(round(near_frac * F))
    picks = rng.choice(subset, size=n_near, replace=True)
    f_near = f_eig[picks] * (1.0 + rng.uniform(-rel_window, rel_window, size=n_near))
    f_far = rng.uniform(10.0, 5000.0, size=F - n_near)
    freq = np.concatenate([f_near, f_far])
    rng.shuffle(freq)
    rhs = rng.standard_normal((n, r)) + 1j * rng.standard_normal((n, r))
    return Rom(K=hysteretic(k, eta), M=_as_complex_f(m), D=_as_complex_f(d),
               rhs=np.asfortranarray(rhs), omega=TWO_PI * freq, seed=seed,
               meta={"workload": "precision", "eta": eta, "eig_subset": subset.tolist(),
                     "n_near": n_near})


def batching_roms(seed: int = 3, count: int = 64, n_lo: int = 24, n_hi: int = 512,
                  F_lo: int = 1000, F_hi: int = 4000, eta: float = 0.02) -> List[Rom]:
    """64 ROMs of uneven order n ~ U[24,512] and frequency count F ~ U[1000,4000]
    over 1..2000 Hz, r in {1, 4}; each ROM is built like the n=64 plain ROM from its own seed."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_lo, n_hi + 1, size=count)
    Fs = rng.integers(F_lo, F_hi + 1, size=count)
    rs = rng.choice([1, 4], size=count)
    seeds = rng.integers(0, 2**31 - 1, size=count)
    roms = []
    for i in range(count):
        r_rng = np.random.default_rng(int(seeds[i]))
        n = int(ns[i])
        q, lam, k, m = modal_pair(r_rng, n, 20.0, 2000.0)
        r = int(rs[i])
        rhs = np.asfortranarray(r_rng.standard_normal((n, r)).astype(np.complex128))
        freq = np.linspace(1.0, 2000.0, int(Fs[i]))
        roms.append(Rom(K=hysteretic(k, eta), M=_as_complex_f(m), D=None, rhs=rhs,
                        omega=TWO_PI * freq, seed=int(seeds[i]),
                        meta={"workload": "batching", "index": i, "eta": eta}))
    return roms


@dataclasses.dataclass
class AdjointProblem:
    """ROM with 16 stiffness-scaling parameters and the loss factor eta.

    K(p) = Q diag(lam * s(p)) Q^T with s_k = p_j for the j-th block of 8 modes;
    A(w) = (1 + i eta) K(p) - w^2 M.  J = sum_w |c^H x(w)|^2.
    """

    rom: Rom
    Q: np.ndarray
    lam: np.ndarray
    Mreal: np.ndarray
    p: np.ndarray
    eta: float
    c: np.ndarray
    block: int = 8

    def stiffness(self, p: Optional[np.ndarray] = None) -> np.ndarray:
        p = self.p if p is None else p
        s = np.repeat(p, self.block)
        k = (self.Q * (self.lam * s)[None, :]) @ self.Q.T
        return 0.5 * (k + k.T)

    def rom_at(self, p: Optional[np.ndarray] = None, eta: Optional[float] = None) -> Rom:
        eta = self.eta if eta is None else eta
        k = self.stiffness(p)
        return dataclasses.replace(self.rom, K=hysteretic(k, eta))


def adjoint_rom(seed: int = 4, n: int = 128, F: int = 2000, n_params: int = 16,
                eta: float = 0.02) -> AdjointProblem:
    rng = np.random.default_rng(seed)
    q, lam, _k, m = modal_pair(rng, n, 20.0, 2000.0)
    order = np.argsort(lam)
    q = q[:, order]
    lam = lam[order]
    block = n // n_params
    assert block * n_params == n
    rhs = np.asfortranarray(rng.standard_normal((n, 1)).astype(np.complex128))
    c = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    freq = np.linspace(1.0, 1500.0, F)
    p = np.ones(n_params)
    k = (q * lam[None, :]) @ q.T
    k = 0.5 * (k + k.T)
    rom = Rom(K=hysteretic(k, eta), M=_as_complex_f(m), D=None, rhs=rhs,
              omega=TWO_PI * freq, seed=seed, meta={"workload": "adjoint", "eta": eta})
    return AdjointProblem(rom=rom, Q=q, lam=lam, Mreal=m, p=p, eta=eta, c=c, block=block)
