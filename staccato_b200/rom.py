"""``KrylovROMSubstructure``: the reference's ROM interface on the B200 kernels.

Mirrors the members of STACCATO's ``KrylovROMSubstructure`` that form the hot path
(src/analysis/KrylovROMSubstructure.h:156, .cpp:709-765 and :1393-1460) and the basis
generation before it (.cpp:367-569):

* ``add_krylov_modes_for_expansion_point(...)`` -- the Krylov basis V for the given expansion
  points and order (block Arnoldi with deflation; the shifted FE matrix factored on the GPU);
* ``generate_rom(K, M, V, D=None, B=None, C=None)`` -- project the sparse FE operators onto
  the basis: K_r = V^T K V, M_r = V^T M V (D_r = V^T D V), B_r = V^T B, C_r = C V;
* ``back_transform_kmor(freq_hz, input_load)`` -- for every frequency assemble
  A(w) = K_r - w^2 M_r + i w D_r (w = 2 pi f), solve A x = B_r F and return
  y = C_r x stacked per frequency, like the reference's results vector.

Matrices are torch tensors on the handle's device; results stay on the device.  The
reduced operators are complex128 like the reference's ``myKComplexReduced`` etc.
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np

from . import _capi
from .project import DeviceCsr, orthonormalize, project, project_complex
from .sweep import DeviceRom, sweep


class KrylovROMSubstructure:
    def __init__(self, device: int = 0, handle: Optional[_capi.Handle] = None):
        self.handle = handle or _capi.Handle(device)
        self.device = device
        self.K_r = self.M_r = self.D_r = self.B_r = self.C_r = None
        self.V = None
        self.eta = 0.0

    # --------------------------------------------------------------- reduced operators
    def set_reduced(self, K_r, M_r, D_r=None, B_r=None, C_r=None, eta: float = 0.0):
        """Install reduced operators (numpy or torch, n x n complex) directly."""
        import torch

        dev = torch.device("cuda", self.device)
        c = lambda a: None if a is None else torch.as_tensor(a, dtype=torch.complex128, device=dev)
        self.K_r, self.M_r, self.D_r, self.B_r, self.C_r = c(K_r), c(M_r), c(D_r), c(B_r), c(C_r)
        self.eta = float(eta)

    def add_krylov_modes_for_expansion_point(self, csr: DeviceCsr, K_vals, M_vals, B, exp_points_hz, krylov_order: int,
                                             D_vals=None, tol: float = 1e-8):
        """The basis of addKrylovModesForExpansionPoint (KrylovROMSubstructure.cpp:367-569) on the
        GPU (``srom_krylov_basis``), kept as ``self.V`` ((k, n) complex128 = n x k column-major,
        ready for ``generate_rom``).  B: n x n_in (numpy or torch)."""
        import torch

        from .krylov import krylov_basis

        dev = torch.device("cuda", self.device)
        c = lambda a: None if a is None else torch.as_tensor(a, dtype=torch.complex128, device=dev).contiguous()
        Bt = torch.as_tensor(B, dtype=torch.complex128, device=dev).t().contiguous()
        self.V = krylov_basis(self.handle, csr, c(K_vals), c(M_vals), c(D_vals), Bt, exp_points_hz, krylov_order, tol)
        return self.V

    def generate_rom(self, csr: DeviceCsr, K_vals, M_vals, V, D_vals=None, B=None, C=None, eta: float = 0.0):
        """Projection of the FE operators (sharing the CSR pattern) onto V, as generateROM
        (KrylovROMSubstructure.cpp:709-765): K_r = V^H K V, M_r = V^H M V, D_r = V^H D V,
        B_r = V^H B, C_r = C V.

        V: (k, n) tensor = n x k column-major basis, float64 (real form, k <= 4096) or
        complex128 (complex form, k <= 2048; complex values are used as given, real values are
        promoted).  B: n x n_in, C: n_out x n."""
        import torch

        mats = [K_vals, M_vals] + ([D_vals] if D_vals is not None else [])
        complex_form = V.dtype == torch.complex128 or any(torch.as_tensor(a).is_complex() for a in mats)
        if complex_form:
            Vc = V.to(torch.complex128).contiguous()
            R = project_complex(self.handle, csr,
                                [torch.as_tensor(a).to(device=V.device, dtype=torch.complex128).contiguous()
                                 for a in mats], Vc)
            to_c = lambda r: r
        else:
            Vc = V
            R = project(self.handle, csr, [torch.as_tensor(a).to(device=V.device) for a in mats], V)
            to_c = lambda r: r.to(torch.complex128)
        self.K_r, self.M_r = to_c(R[0]), to_c(R[1])
        self.D_r = to_c(R[2]) if D_vals is not None else None
        Vcm = Vc.t().to(torch.complex128)  # n x k
        self.B_r = None if B is None else (Vcm.conj().t() @ torch.as_tensor(B, device=V.device).to(torch.complex128))
        self.C_r = None if C is None else (torch.as_tensor(C, device=V.device).to(torch.complex128) @ Vcm)
        self.eta = float(eta)
        return R

    # --------------------------------------------------------------- frequency sweep
    def _device_rom(self, rhs, omega, with_c: bool) -> DeviceRom:
        import torch

        n, r = int(rhs.shape[0]), int(rhs.shape[1])
        cm = lambda a: a.t().contiguous().reshape(-1)  # column-major flat copy
        rom = DeviceRom(n=n, r=r, F=len(omega), K=cm(self.K_r), M=cm(self.M_r),
                        D=None if self.D_r is None else cm(self.D_r), rhs=cm(rhs),
                        omega=torch.as_tensor(omega, device=self.K_r.device), eta=self.eta)
        if with_c and self.C_r is not None:
            rom.C, rom.n_out = cm(self.C_r), int(self.C_r.shape[0])
        rom.allocate_outputs(self.K_r.device)
        return rom

    def back_transform_kmor(self, freq_hz, input_load, precision: int = _capi.SROM_FP64,
                            flags: int = _capi.SROM_FLAG_FALLBACK_FP64, max_refine: int = 5):
        """y(w) = C_r A(w)^-1 B_r F per frequency; returns (Y, info) with Y of shape
        (F, n_out, r) (x itself when C_r is None).  The back-projection y = C_r x runs on the
        device right after the sweep (srom_rom_desc.C / .Y)."""
        import torch

        freq = np.asarray(freq_hz, dtype=np.float64)
        omega = 2.0 * math.pi * freq
        F_load = torch.as_tensor(input_load, dtype=torch.complex128, device=self.K_r.device)
        if F_load.ndim == 1:
            F_load = F_load[:, None]
        rhs = F_load if self.B_r is None else self.B_r @ F_load
        rom = self._device_rom(rhs, omega, with_c=True)
        sweep(self.handle, [rom], precision=precision, flags=flags, max_refine=max_refine)
        if rom.n_out > 0:
            Y = rom.Y.reshape(rom.F, rom.r, rom.n_out).transpose(1, 2)  # (F, n_out, r)
        else:
            Y = rom.X.reshape(rom.F, rom.r, rom.n).transpose(1, 2)  # (F, n, r)
        return Y, rom.info

    def transfer_functions(self, freq_hz, precision: int = _capi.SROM_FP64,
                           flags: int = _capi.SROM_FLAG_FALLBACK_FP64, max_refine: int = 5):
        """H_R(w) = C_r A(w)^-1 B_r per frequency (KrylovROMSubstructure.cpp:1433-1441): the
        sweep with B_r as right-hand sides and C_r as output matrix.  Returns (H, info) with H
        of shape (F, n_out, n_in) (A^-1 B_r when C_r is None)."""
        if self.B_r is None:
            raise ValueError("transfer functions need B_r")
        omega = 2.0 * math.pi * np.asarray(freq_hz, dtype=np.float64)
        rom = self._device_rom(self.B_r, omega, with_c=True)
        sweep(self.handle, [rom], precision=precision, flags=flags, max_refine=max_refine)
        if rom.n_out > 0:
            H = rom.Y.reshape(rom.F, rom.r, rom.n_out).transpose(1, 2)
        else:
            H = rom.X.reshape(rom.F, rom.r, rom.n).transpose(1, 2)
        return H, rom.info
