"""KrylovROMSubstructure: generate_rom + back_transform_kmor end to end (the reference's
ROM interface), against the oracle."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from staccato_b200 import _capi, fe_tet10, workloads as W
from staccato_b200.project import DeviceCsr
from staccato_b200.rom import KrylovROMSubstructure

pytestmark = pytest.mark.gpu


def test_back_transform_matches_oracle_with_output_projection(handle):
    rom = W.plain_rom(F=40)
    n = rom.n
    rng = np.random.default_rng(0)
    B = rng.standard_normal((n, 2))
    C = rng.standard_normal((3, n))
    load = rng.standard_normal((2, 1))
    s = KrylovROMSubstructure(handle=handle)
    s.set_reduced(rom.K, rom.M, None, B, C)
    freq = rom.omega / (2 * math.pi)
    Y, info = s.back_transform_kmor(freq, load)
    rhs = B @ load
    X, _ = O.sweep(rom.K, rom.M, None, 0.0, rhs, 2 * math.pi * freq)
    ref = np.einsum("on,fnr->for", C, X)
    Yh = Y.cpu().numpy()
    assert np.abs(Yh - ref).max() <= 1e-12 * np.abs(ref).max()
    assert (info.cpu().numpy() == 0).all()


def test_generate_rom_then_sweep_small_block(handle):
    import torch

    m = fe_tet10.clamped_block(2, 2, 6)
    V = O.mgs(fe_tet10.basis(m.n_dof, 24, seed=5), passes=2)
    s = KrylovROMSubstructure(handle=handle)
    csr = DeviceCsr.from_host(m.indptr, m.indices)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    s.generate_rom(csr, dev(m.K), dev(m.M), dev(np.ascontiguousarray(V.T)), eta=0.02)
    Kr = O.project(m.indptr, m.indices, m.K, V)
    Mr = O.project(m.indptr, m.indices, m.M, V)
    assert np.abs(s.K_r.cpu().numpy() - Kr).max() <= 1e-12 * np.abs(Kr).max()
    freq = np.linspace(10.0, 5000.0, 16)
    load = np.ones(24)
    Y, info = s.back_transform_kmor(freq, load)
    X, _ = O.sweep(Kr.astype(complex), Mr.astype(complex), None, 0.02, load[:, None].astype(complex),
                   2 * math.pi * freq)
    assert np.abs(Y.cpu().numpy() - X).max() <= 1e-9 * np.abs(X).max()


def test_generate_rom_complex_basis_then_sweep(handle):
    """Complex basis (and hysteretic complex stiffness values): generate_rom takes the complex
    projection, and the swept ROM matches the oracle on the same reduced operators."""
    import torch

    m = fe_tet10.clamped_block(2, 2, 6)
    n, k = m.n_dof, 20
    rng = np.random.default_rng(6)
    V = np.linalg.qr(rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k)))[0]
    s = KrylovROMSubstructure(handle=handle)
    csr = DeviceCsr.from_host(m.indptr, m.indices)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    Kc = m.K * (1 + 0.02j)
    B = np.zeros((n, 1))
    B[n - 1, 0] = 1.0
    s.generate_rom(csr, dev(Kc), dev(m.M), dev(V.T), B=B, C=B.T)
    import scipy.sparse as sp

    Ka = sp.csr_matrix((Kc, m.indices, m.indptr), shape=(n, n))
    Ma = sp.csr_matrix((m.M, m.indices, m.indptr), shape=(n, n))
    Kr, Mr = V.conj().T @ (Ka @ V), V.conj().T @ (Ma @ V)
    assert np.abs(s.K_r.cpu().numpy() - Kr).max() <= 1e-12 * np.abs(Kr).max()
    freq = np.linspace(10.0, 3000.0, 12)
    Y, info = s.back_transform_kmor(freq, np.ones(1))
    X, _ = O.sweep(s.K_r.cpu().numpy(), s.M_r.cpu().numpy(), None, 0.0, s.B_r.cpu().numpy(), 2 * math.pi * freq)
    ref = np.einsum("on,fnr->for", s.C_r.cpu().numpy(), X)
    assert np.abs(Y.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()
