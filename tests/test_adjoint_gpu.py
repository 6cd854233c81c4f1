"""Adjoint sweep: gradient against the FP64 CPU adjoint (oracle) and central finite
differences (relative step 1e-6); tolerance 1e-6 relative, as the differentiation workload
specifies."""
import numpy as np
import pytest

from oracle import oracle as O
from staccato_b200 import _capi, workloads as W
from staccato_b200.adjoint import Param, backward, forward_J, modal_params, objective_and_cotangent
from staccato_b200.sweep import DeviceRom, sweep

pytestmark = pytest.mark.gpu


def _t(a):
    import torch

    return torch.from_numpy(np.asarray(a)).cuda()


def test_adjoint_random_params_vs_cpu_adjoint(handle):
    import torch

    rng = np.random.default_rng(11)
    n, r, F = 37, 2, 9
    c = lambda s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    K, M, D = c((n, n)) + 6 * np.eye(n), c((n, n)), c((n, n))
    rhs = c((n, r))
    omega = rng.uniform(0.2, 1.5, F)
    d = DeviceRom.from_host(K, M, D, rhs, omega, keep_factors=True)
    sweep(handle, [d], flags=_capi.SROM_FLAG_KEEP_FACTORS)
    X = d.X.reshape(F, r, n).transpose(1, 2)
    gb = c((F, n, r))
    U, Wm, s, G = c((n, 3)), c((n, 3)), rng.uniform(0.5, 2, 3), c((n, n))
    flat = lambda a: _t(np.asfortranarray(a).ravel(order="F").astype(np.complex128))
    params = [Param(U=flat(U), W=flat(Wm), s=_t(s), rank=3, c0=0.3 + 0.1j, c1=0.7, c2=-0.2j),
              Param(G=flat(G), c0=1j, c1=0.5 - 0.5j),
              Param(U=flat(U), s=None, rank=3, c2=1.0)]
    g = backward(handle, d, _t(gb), params).cpu().numpy()

    def dA(j, w):
        coef = lambda p: p.c0 + p.c1 * (1j * w) + p.c2 * (-w * w)
        if j == 0:
            return coef(params[0]) * (U * s) @ Wm.T
        if j == 1:
            return coef(params[1]) * G
        return coef(params[2]) * U @ U.T

    class Terms:
        count = 3

        def __call__(self, j, w):
            return dA(j, w)

    ref = O.adjoint_gradient(K, M, D, 0.0, rhs, omega, gb, Terms())
    assert np.abs(g - ref).max() <= 1e-10 * max(np.abs(ref).max(), 1.0)


def _J_exact(prob, omega, p=None, eta=None):
    """Objective from the oracle's long-double-refined solutions (noise ~1e-16 J), so that a
    central difference with a 1e-6 relative step resolves the gradient to ~1e-8."""
    rom = prob.rom
    e = prob.eta if eta is None else eta
    X = O.x_ref(prob.stiffness(p).astype(complex), rom.M, None, e, rom.rhs, omega)
    y = np.einsum("i,fir->fr", prob.c.conj(), X)
    return float((np.abs(y) ** 2).sum())


def test_adjoint_modal_workload_vs_fd_and_cpu(handle):
    import torch

    prob = W.adjoint_rom()
    rom = prob.rom
    sub = np.arange(0, rom.F, 50)  # 40 of the 2000 frequencies, spread over 1-1500 Hz
    om = rom.omega[sub]
    K = prob.stiffness()
    d = DeviceRom.from_host(K.astype(np.complex128), rom.M, None, rom.rhs, om, eta=prob.eta, keep_factors=True)
    sweep(handle, [d], flags=_capi.SROM_FLAG_KEEP_FACTORS)
    X = d.X.reshape(d.F, d.r, d.n).transpose(1, 2)
    J0, gbar = objective_and_cotangent(X, prob.c)
    params = modal_params(prob)
    g = backward(handle, d, gbar, params).cpu().numpy()
    # central finite differences of the exact objective, relative step 1e-6
    fd = np.zeros(len(params))
    for j in range(len(prob.p)):
        h = 1e-6 * prob.p[j]
        pp, pm = prob.p.copy(), prob.p.copy()
        pp[j] += h
        pm[j] -= h
        fd[j] = (_J_exact(prob, om, p=pp) - _J_exact(prob, om, p=pm)) / (2 * h)
    h = 1e-6 * prob.eta
    fd[-1] = (_J_exact(prob, om, eta=prob.eta + h) - _J_exact(prob, om, eta=prob.eta - h)) / (2 * h)
    assert np.abs(g - fd).max() <= 1e-6 * np.abs(fd).max(), (g, fd)
    # per component: 1e-6 relative, with a floor of 1e-8 of the largest component for the
    # tiny ones (a central difference of J cannot resolve them below that)
    floor = 1e-8 * np.abs(fd).max()
    assert (np.abs(g - fd) <= 1e-6 * np.abs(fd) + floor).all(), (g, fd)
    # FP64 CPU adjoint on the same frequencies (dense derivative matrices)

    class Terms:
        count = len(params)

        def __call__(self, j, w):
            if j < len(prob.p):
                b = prob.block
                Qj = prob.Q[:, j * b:(j + 1) * b]
                return (1 + 1j * prob.eta) * (Qj * prob.lam[j * b:(j + 1) * b]) @ Qj.T
            return 1j * K

    ref = O.adjoint_gradient(K.astype(complex), rom.M, None, prob.eta, rom.rhs, om, gbar.cpu().numpy(), Terms())
    assert np.abs(g - ref).max() <= 1e-10 * np.abs(ref).max()


def test_adjoint_full_workload_runs(handle):
    prob = W.adjoint_rom()
    J0, gbar, d = forward_J(handle, prob, keep=True)
    g = backward(handle, d, gbar, modal_params(prob)).cpu().numpy()
    assert np.isfinite(g).all() and np.abs(g).max() > 0


def test_backward_requires_kept_factors(handle):
    rom = W.plain_rom(F=4)
    d = DeviceRom.from_host(rom.K, rom.M, None, rom.rhs, rom.omega)
    sweep(handle, [d])
    import torch

    gb = torch.zeros((4, rom.n, 1), dtype=torch.complex128, device="cuda")
    with pytest.raises(_capi.SromError) as e:
        backward(handle, d, gb, [Param(G=torch.zeros(rom.n * rom.n, dtype=torch.complex128, device="cuda"))])
    assert e.value.status == _capi.SROM_ERR_INVALID
