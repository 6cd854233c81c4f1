"""Backward (adjoint) sweep through ``srom_sweep_backward``, and the objective of the
differentiation workload: J = sum_w |c^H x(w)|^2 for a modal ROM with stiffness-scaling
parameters p_j (each scaling a disjoint block of modes) and the loss factor eta.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence

import numpy as np

from . import _capi
from ._capi import Complex, DParam, check
from .sweep import DeviceRom, sweep


class Param:
    """dA/dp(w) = (c0 + c1 (i w) + c2 (-w^2)) G with G = U diag(s) W^T or dense G
    (device tensors; U, W, G complex128 column-major flattened, s float64)."""

    def __init__(self, U=None, s=None, W=None, G=None, rank=0, c0=1.0, c1=0.0, c2=0.0):
        self.U, self.s, self.W, self.G, self.rank = U, s, W, G, rank
        self.c0, self.c1, self.c2 = complex(c0), complex(c1), complex(c2)

    def struct(self) -> DParam:
        p = lambda t: None if t is None else C.c_void_p(t.data_ptr())
        kind = _capi.SROM_DPARAM_DENSE if self.G is not None else _capi.SROM_DPARAM_LOWRANK
        cx = lambda z: Complex(z.real, z.imag)
        return DParam(kind=kind, rank=self.rank, U=p(self.U), W=p(self.W), s=p(self.s), G=p(self.G),
                      c0=cx(self.c0), c1=cx(self.c1), c2=cx(self.c2))


def backward(handle: _capi.Handle, rom: DeviceRom, gbar, params: Sequence[Param], want_lambda=False):
    """dJ/dp for every parameter (torch float64 tensor); gbar: (F, n, r) complex tensor of
    cotangents 2 dJ/d conj(x).  rom must hold the kept factors of a forward FP64 sweep."""
    import torch

    g = gbar.transpose(1, 2).contiguous()  # per frequency: n x r column-major
    out = torch.empty(len(params), dtype=torch.float64, device=g.device)
    lam = torch.empty(rom.F * rom.n * rom.r, dtype=torch.complex128, device=g.device) if want_lambda else None
    arr = (DParam * max(len(params), 1))(*[q.struct() for q in params])
    d = rom.desc()
    check(handle.ptr, _capi.lib().srom_sweep_backward(
        handle.ptr, C.byref(d), C.c_void_p(g.data_ptr()), rom.n, arr, len(params),
        C.c_void_p(out.data_ptr()), None if lam is None else C.c_void_p(lam.data_ptr())))
    if want_lambda:
        return out, lam.reshape(rom.F, rom.r, rom.n).transpose(1, 2)
    return out


def modal_params(prob, device="cuda") -> List[Param]:
    """Parameters of the differentiation workload: p_j scales modes [8j, 8j+8) of K
    (dA/dp_j = (1 + i eta) Q_j diag(lam_j) Q_j^T), then eta (dA/deta = i K)."""
    import torch

    out = []
    b = prob.block
    for j in range(len(prob.p)):
        Qj = prob.Q[:, j * b:(j + 1) * b]
        U = torch.from_numpy(np.asfortranarray(Qj).ravel(order="F").astype(np.complex128)).to(device)
        s = torch.from_numpy((prob.lam[j * b:(j + 1) * b] * 1.0).astype(np.float64)).to(device)
        out.append(Param(U=U, s=s, rank=b, c0=complex(1.0, prob.eta)))
    K = prob.stiffness()
    G = torch.from_numpy(np.asfortranarray(K).ravel(order="F").astype(np.complex128)).to(device)
    out.append(Param(G=G, c0=1j))
    return out


def objective_and_cotangent(X, c):
    """J = sum_f sum_r |c^H x_f|^2 and gbar_f = 2 c (c^H x_f) for X of shape (F, n, r)."""
    import torch

    ct = torch.as_tensor(c, dtype=torch.complex128, device=X.device)
    y = torch.einsum("i,fir->fr", ct.conj(), X)  # c^H x
    J = float((y.abs() ** 2).sum())
    gbar = 2.0 * ct[None, :, None] * y[:, None, :]
    return J, gbar


def forward_J(handle, prob, p=None, eta=None, keep=False, device="cuda"):
    """Forward FP64 sweep of the differentiation workload at parameters (p, eta)."""
    rom = prob.rom
    K = prob.stiffness(p)
    e = prob.eta if eta is None else eta
    d = DeviceRom.from_host(K.astype(np.complex128), rom.M, None, rom.rhs, rom.omega, eta=e, device=device,
                            keep_factors=keep)
    sweep(handle, [d], precision=_capi.SROM_FP64, flags=_capi.SROM_FLAG_KEEP_FACTORS if keep else 0)
    X = d.X.reshape(d.F, d.r, d.n).transpose(1, 2)
    J, gbar = objective_and_cotangent(X, prob.c)
    return J, gbar, d
