"""Interface-Jacobian coupling of substructures (IJCSA) on the sweep kernels.

Restates the simulation-model part of the reference's coupling program
(test/IJCSA/src/IJSA.cu): per substructure s and frequency w,

* the interface transfer functions H_s = C_if A_s(w)^-1 B_if and the loaded response
  y_s = C_if A_s(w)^-1 B_load F (IJSA.cu:826-919: batched assembly, getrf, getrs, GEMMs) --
  here one sweep per substructure, right-hand sides [B_if, B_load F], with the back-projection
  C_if fused after the solve;
* the interface outputs Y_s = H_s U_s + y_s for the current interface inputs U_s (:921-945);
* the residual R = sum_s dR/dY_s Y_s + dR/dU_s U_s (:947-969) and the interface Jacobian,
  whose column block s is dR/dY_s H_s + dR/dU_s (:971-983);
* the correction dU = J^-1 R by a batched LU solve over the frequencies (:1198-1207) --
  here ``solve_batched`` (partial pivoting; the reference's cuBLAS call pivots nothing);
* the update U_s <- U_s - dU_s and the outputs Y_s again (:1348-1410).

The coupling conditions are linear in (U, Y), so one step from any start solves them exactly
(up to rounding); ``steps`` > 1 repeats the update from the new residual.  The reference's
experimental models (measured FRFs in place of H_s) enter the same way: pass ``H`` and ``y``
directly through ``ExperimentalModel``.  A_s(w) follows the sweep's convention
(1 + i eta) K - w^2 M + i w D with w = 2 pi f; the reference's coupling program scales M by
4 pi^2 and D by f instead, which is the same matrix.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence, Union

import numpy as np

from . import _capi
from .linalg import OP_N, OP_T, zgemm
from .sweep import DeviceRom, solve_batched, sweep


@dataclasses.dataclass
class SimulationModel:
    """A substructure given by its (reduced) operators.  B_if: n x p inputs at the interface
    DOFs (interface forces), C_if: p x n outputs there (displacements), B_load: n x q with
    load amplitudes F (q,)."""

    K: np.ndarray
    M: Optional[np.ndarray]
    B_if: np.ndarray
    C_if: np.ndarray
    D: Optional[np.ndarray] = None
    eta: float = 0.0
    B_load: Optional[np.ndarray] = None
    F: Optional[np.ndarray] = None


@dataclasses.dataclass
class ExperimentalModel:
    """A substructure given by measured interface FRFs: H (nf, p, p) and the loaded
    response y (nf, p) at the same frequencies (zeros when unloaded)."""

    H: np.ndarray
    y: Optional[np.ndarray] = None


Model = Union[SimulationModel, ExperimentalModel]


def _torch():
    import torch

    return torch


def interface_frfs(handle: _capi.Handle, model: SimulationModel, freq_hz, precision: int = _capi.SROM_FP64):
    """(H, y): H (nf, p, p) = C_if A^-1 B_if and y (nf, p) = C_if A^-1 B_load F per frequency."""
    torch = _torch()
    omega = 2.0 * math.pi * np.asarray(freq_hz, dtype=np.float64)
    p = int(model.B_if.shape[1])
    rhs = np.asarray(model.B_if, dtype=np.complex128)
    loaded = model.B_load is not None and model.F is not None
    if loaded:
        f = np.asarray(model.B_load, dtype=np.complex128) @ np.asarray(model.F, dtype=np.complex128).reshape(-1)
        rhs = np.concatenate([rhs, f[:, None]], axis=1)
    rom = DeviceRom.from_host(model.K, model.M, model.D, rhs, omega, eta=model.eta,
                              device=torch.device("cuda", handle.device), C=model.C_if)
    sweep(handle, [rom], precision=precision, flags=_capi.SROM_FLAG_FALLBACK_FP64)
    Y = rom.Y.reshape(rom.F, rom.r, rom.n_out).transpose(1, 2)  # (nf, p, r)
    H = Y[:, :, :p]
    y = Y[:, :, p] if loaded else torch.zeros((rom.F, p), dtype=torch.complex128, device=Y.device)
    return H, y


def couple(handle: _capi.Handle, models: Sequence[Model], dRdY: Sequence[np.ndarray], dRdU: Sequence[np.ndarray],
           freq_hz, U0: Optional[Sequence[np.ndarray]] = None, steps: int = 1,
           precision: int = _capi.SROM_FP64):
    """Coupled interface inputs and outputs of all substructures at every frequency.

    dRdY[s], dRdU[s]: G x p_s derivatives of the G coupling conditions with respect to the
    outputs and inputs of substructure s (G = sum_s p_s).  Returns (U, Y, residual_norm):
    U[s], Y[s] of shape (nf, p_s) and the 2-norm of the residual per frequency after the
    last step (device tensors)."""
    torch = _torch()
    dev = torch.device("cuda", handle.device)
    freq = np.asarray(freq_hz, dtype=np.float64)
    nf = len(freq)
    Hs, ys = [], []
    for m in models:
        if isinstance(m, SimulationModel):
            H, y = interface_frfs(handle, m, freq, precision)
        else:
            H = torch.as_tensor(m.H, dtype=torch.complex128, device=dev)
            y = (torch.zeros(H.shape[:2], dtype=torch.complex128, device=dev) if m.y is None
                 else torch.as_tensor(m.y, dtype=torch.complex128, device=dev))
        Hs.append(H)
        ys.append(y)
    ps = [int(H.shape[1]) for H in Hs]
    G = sum(ps)
    dY = [torch.as_tensor(a, dtype=torch.complex128, device=dev).contiguous() for a in dRdY]
    dU = [torch.as_tensor(a, dtype=torch.complex128, device=dev).contiguous() for a in dRdU]
    Hs = [H.contiguous() for H in Hs]
    ys = [y.contiguous() for y in ys]
    for s, p in enumerate(ps):
        if tuple(dY[s].shape) != (G, p) or tuple(dU[s].shape) != (G, p):
            raise ValueError(f"dRdY[{s}] and dRdU[{s}] must be {G} x {p}")
    U = [torch.zeros((nf, p), dtype=torch.complex128, device=dev) if U0 is None
         else torch.as_tensor(U0[s], dtype=torch.complex128, device=dev).expand(nf, p).clone()
         for s, p in enumerate(ps)]
    offs = np.cumsum([0] + ps)
    # Products on the library's batched complex GEMM, in column-major terms (a row-major
    # (a, b) tensor is the column-major b x a matrix, its transpose).
    # Interface Jacobian J (nf, G, G), column block s = dR/dY_s H_s + dR/dU_s (constant in U):
    # J_s^T = H_s^T dY_s^T + dU_s^T per frequency.
    J = torch.empty((nf, G, G), dtype=torch.complex128, device=dev)
    for s, p in enumerate(ps):
        J[:, :, offs[s]:offs[s + 1]] = dU[s]
        zgemm(handle, OP_N, OP_N, p, G, p, Hs[s], p, p * p, dY[s], p, 0, J[:, :, offs[s]:], G, G * G,
              batch=nf, beta=1.0)

    def outputs_and_residual():
        # Y_s[f] = H_s[f] U_s[f] + y_s[f]   (y^T = U^T H^T: op T on the column-major H^T)
        Y = []
        for s, p in enumerate(ps):
            Ys = ys[s].clone()
            zgemm(handle, OP_T, OP_N, p, 1, p, Hs[s], p, p * p, U[s], p, p, Ys, p, p, batch=nf, beta=1.0)
            Y.append(Ys)
        # R[f] = sum_s dY_s Y_s[f] + dU_s U_s[f], all frequencies at once: R^T = dY_s Y_s^T + ...
        R = torch.empty((nf, G), dtype=torch.complex128, device=dev)
        first = True
        for s, p in enumerate(ps):
            for Dm, X in ((dY[s], Y[s]), (dU[s], U[s])):
                zgemm(handle, OP_T, OP_N, G, nf, p, Dm, p, 0, X.contiguous(), p, 0, R, G, 0,
                      beta=0.0 if first else 1.0)
                first = False
        return Y, R

    Y, R = outputs_and_residual()
    for _ in range(max(steps, 1)):
        dUall, info = solve_batched(handle, J, R[:, :, None], precision=_capi.SROM_FP64)
        if (info != 0).any():
            raise RuntimeError("singular interface Jacobian at some frequency")
        for s in range(len(ps)):
            U[s] = U[s] - dUall[:, offs[s]:offs[s + 1], 0]
        Y, R = outputs_and_residual()
    return U, Y, torch.linalg.vector_norm(R, dim=1)
