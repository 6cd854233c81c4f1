"""Interface-Jacobian coupling (staccato_b200.ijcsa) against a monolithic solve: two
substructures sharing p interface DOFs are coupled by compatibility (equal interface
displacements) and equilibrium (interface forces summing to zero); the coupled interface
displacements must equal those of the primal assembly of both substructures solved directly
(oracle zgetrf/zgetrs on the assembled system)."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from staccato_b200 import _capi
from staccato_b200.ijcsa import ExperimentalModel, SimulationModel, couple, interface_frfs

pytestmark = pytest.mark.gpu


def _spd(rng, n, scale):
    A = rng.standard_normal((n, n))
    return scale * (A @ A.T / n + np.eye(n))


def _two_substructures(seed=0, n1=30, n2=40, p=6):
    rng = np.random.default_rng(seed)
    # substructure 1 DOFs: [internal (n1 - p), interface (p)]; substructure 2: [interface (p), internal]
    K1, M1 = _spd(rng, n1, 1e4), _spd(rng, n1, 1.0)
    K2, M2 = _spd(rng, n2, 2e4), _spd(rng, n2, 1.5)
    N = n1 + n2 - p
    Kg = np.zeros((N, N))
    Mg = np.zeros((N, N))
    idx1 = np.arange(n1)
    idx2 = np.arange(n1 - p, N)
    Kg[np.ix_(idx1, idx1)] += K1
    Mg[np.ix_(idx1, idx1)] += M1
    Kg[np.ix_(idx2, idx2)] += K2
    Mg[np.ix_(idx2, idx2)] += M2
    B1 = np.zeros((n1, p))
    B1[n1 - p:, :] = np.eye(p)
    B2 = np.zeros((n2, p))
    B2[:p, :] = np.eye(p)
    load = np.zeros((n1, 1))
    load[2, 0] = 1.0  # unit force on an internal DOF of substructure 1
    eta = 0.02
    s1 = SimulationModel(K=K1.astype(complex), M=M1.astype(complex), B_if=B1, C_if=B1.T, eta=eta,
                         B_load=load, F=np.ones(1))
    s2 = SimulationModel(K=K2.astype(complex), M=M2.astype(complex), B_if=B2, C_if=B2.T, eta=eta)
    I, Z = np.eye(p), np.zeros((p, p))
    dRdY = [np.vstack([I, Z]), np.vstack([-I, Z])]  # compatibility: Y1 - Y2 = 0
    dRdU = [np.vstack([Z, I]), np.vstack([Z, I])]   # equilibrium: U1 + U2 = 0
    Fg = np.zeros((N, 1), dtype=complex)
    Fg[2, 0] = 1.0
    return s1, s2, dRdY, dRdU, Kg, Mg, Fg, eta, n1, p


@pytest.mark.parametrize("precision", [_capi.SROM_FP64, _capi.SROM_MIXED_FP32], ids=["fp64", "mixed"])
def test_two_substructures_match_monolithic_solve(handle, precision):
    s1, s2, dRdY, dRdU, Kg, Mg, Fg, eta, n1, p = _two_substructures()
    freq = np.linspace(1.0, 40.0, 25)
    U, Y, rn = couple(handle, [s1, s2], dRdY, dRdU, freq, precision=precision)
    Xg = O.x_ref(Kg.astype(complex), Mg.astype(complex), None, eta, Fg, 2 * math.pi * freq)[:, :, 0]
    ref_if = Xg[:, n1 - p:n1]  # displacements of the shared interface DOFs
    Y1, Y2 = Y[0].cpu().numpy(), Y[1].cpu().numpy()
    err = np.linalg.norm(Y1 - ref_if, axis=1) / np.linalg.norm(ref_if, axis=1)
    assert err.max() <= (1e-9 if precision == _capi.SROM_FP64 else 1e-8)
    assert np.abs(Y1 - Y2).max() <= 1e-9 * np.abs(ref_if).max()
    assert np.abs(U[0].cpu().numpy() + U[1].cpu().numpy()).max() <= 1e-9 * np.abs(U[0].cpu().numpy()).max()
    assert rn.cpu().numpy().max() <= 1e-9 * np.abs(ref_if).max() * 1e4


def test_measured_frfs_in_place_of_a_simulation_model(handle):
    """An experimental model (interface FRFs given as data) couples like a simulated one."""
    s1, s2, dRdY, dRdU, Kg, Mg, Fg, eta, n1, p = _two_substructures(seed=1)
    freq = np.linspace(2.0, 30.0, 11)
    H2, _ = interface_frfs(handle, s2, freq)
    e2 = ExperimentalModel(H=H2.cpu().numpy())
    U, Y, _ = couple(handle, [s1, e2], dRdY, dRdU, freq)
    U_ref, Y_ref, _ = couple(handle, [s1, s2], dRdY, dRdU, freq)
    assert np.allclose(Y[0].cpu().numpy(), Y_ref[0].cpu().numpy(), rtol=1e-12, atol=0)
