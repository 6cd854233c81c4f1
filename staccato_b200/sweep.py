"""Python front end of the batched frequency sweep (device-resident torch buffers).

``sweep()`` packs one or many ROMs into ``srom_rom_desc`` records and calls ``srom_sweep``
on the handle's stream; ``sweep_host()`` does the same through ``srom_sweep_host`` with
host (numpy) buffers, which is the end-to-end form of the reference's backTransformKMOR.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import List, Optional, Sequence

import numpy as np

from . import _capi
from ._capi import RomDesc, SweepOpts, check


def _torch():
    import torch

    return torch


def colmajor(a) -> np.ndarray:
    """Column-major complex128 data of a matrix as a flat array."""
    return np.asarray(a, dtype=np.complex128).ravel(order="F")


@dataclasses.dataclass
class DeviceRom:
    """One ROM with its inputs and outputs in device memory (flat column-major tensors)."""

    n: int
    r: int
    F: int
    K: "object"
    M: "object"
    D: Optional["object"]
    rhs: "object"
    omega: "object"
    eta: float = 0.0
    X: Optional["object"] = None
    info: Optional["object"] = None
    steps: Optional["object"] = None
    berr: Optional["object"] = None
    LU: Optional["object"] = None
    ipiv: Optional["object"] = None
    C: Optional["object"] = None      # n_out x n output matrix (flat column-major) or None
    Y: Optional["object"] = None      # F blocks of n_out x r: y(w) = C x(w)
    n_out: int = 0

    @classmethod
    def from_host(cls, K, M, D, rhs, omega, eta: float = 0.0, device="cuda",
                  keep_factors: bool = False, C=None) -> "DeviceRom":
        torch = _torch()
        K = np.asarray(K)
        n = int(K.shape[0])
        rhs = np.asarray(rhs, dtype=np.complex128)
        if rhs.ndim == 1:
            rhs = rhs[:, None]
        r = int(rhs.shape[1])
        omega = np.ascontiguousarray(omega, dtype=np.float64)
        F = int(omega.shape[0])
        t = lambda a: torch.from_numpy(colmajor(a)).to(device)
        rom = cls(n=n, r=r, F=F, K=t(K), M=None if M is None else t(M), D=None if D is None else t(D), rhs=t(rhs),
                  omega=torch.from_numpy(omega).to(device), eta=float(eta))
        if C is not None:
            C = np.asarray(C)
            rom.C, rom.n_out = t(C), int(C.shape[0])
        rom.allocate_outputs(device, keep_factors)
        return rom

    def allocate_outputs(self, device="cuda", keep_factors: bool = False) -> None:
        torch = _torch()
        self.X = torch.empty(self.F * self.n * self.r, dtype=torch.complex128, device=device)
        self.info = torch.empty(self.F, dtype=torch.int32, device=device)
        self.steps = torch.empty(self.F, dtype=torch.int32, device=device)
        self.berr = torch.empty(self.F, dtype=torch.float64, device=device)
        if keep_factors:
            self.LU = torch.empty(self.F * self.n * self.n, dtype=torch.complex128, device=device)
            self.ipiv = torch.empty(self.F * self.n, dtype=torch.int32, device=device)
        if self.n_out > 0:
            self.Y = torch.empty(self.F * self.n_out * self.r, dtype=torch.complex128, device=device)

    def desc(self) -> RomDesc:
        def p(t):
            if t is None:
                return None
            if not t.is_cuda:
                raise ValueError("DeviceRom arrays must be CUDA tensors (the C ABI takes device pointers)")
            return C.c_void_p(t.data_ptr())

        return RomDesc(n=self.n, r=self.r, F=self.F, ldk=self.n, K=p(self.K), M=p(self.M),
                       D=p(self.D), eta=self.eta, rhs=p(self.rhs), ldb=self.n,
                       omega=p(self.omega), X=p(self.X), info=p(self.info), steps=p(self.steps),
                       berr=p(self.berr), LU=p(self.LU), ipiv=p(self.ipiv),
                       n_out=self.n_out, ldc=max(self.n_out, 1), C=p(self.C), Y=p(self.Y))

    def solutions(self) -> np.ndarray:
        """X as a numpy array of shape (F, n, r)."""
        x = self.X.cpu().numpy().reshape(self.F, self.r, self.n)
        return np.ascontiguousarray(x.transpose(0, 2, 1))

    def outputs(self) -> np.ndarray:
        """Y = C X as a numpy array of shape (F, n_out, r)."""
        y = self.Y.cpu().numpy().reshape(self.F, self.r, self.n_out)
        return np.ascontiguousarray(y.transpose(0, 2, 1))


def opts(precision: int = _capi.SROM_FP64, max_refine: int = 5, tol: float = 0.0,
         flags: int = 0) -> SweepOpts:
    return SweepOpts(precision=precision, max_refine=max_refine, tol=tol, flags=flags)


def sweep(handle: _capi.Handle, roms: Sequence[DeviceRom], precision: int = _capi.SROM_FP64,
          max_refine: int = 5, tol: float = 0.0, flags: int = 0) -> None:
    """Asynchronous batched sweep of every ROM on the handle's stream."""
    arr = (RomDesc * max(len(roms), 1))(*[r.desc() for r in roms])
    o = opts(precision, max_refine, tol, flags)
    check(handle.ptr, _capi.lib().srom_sweep(handle.ptr, arr, len(roms), C.byref(o)))


def solve_batched(handle: _capi.Handle, A, B, precision: int = _capi.SROM_FP64,
                  flags: int = _capi.SROM_FLAG_FALLBACK_FP64, max_refine: int = 5):
    """Solve A_i X_i = B_i for a batch of given complex matrices: the batched
    getrf + getrs of the reference's coupling and batched-LU programs
    (test/IJCSA/src/IJSA.cu:1198-1206, test/krylovMidsizeTest/gpu/concurrent/batchedLU/
    src/main.cu:254-259, cublasZgetrfBatched / cublasZgetrsBatched, there without pivoting).

    Each matrix goes through the sweep kernels as a one-frequency system with K = A_i and no
    mass or damping term (M = D = NULL), so it is factored with partial pivoting exactly like a
    swept system.  A: (count, n, n) and B: (count, n, r) or (n, r), numpy or torch (any
    device).  Returns (X, info) as device tensors of shape (count, n, r) and (count,)."""
    torch = _torch()
    dev = torch.device("cuda", handle.device)
    A = torch.as_tensor(A, dtype=torch.complex128)
    if A.ndim != 3 or A.shape[1] != A.shape[2]:
        raise ValueError("A must have shape (count, n, n)")
    count, n = int(A.shape[0]), int(A.shape[1])
    B = torch.as_tensor(B, dtype=torch.complex128)
    if B.ndim == 1:
        B = B[:, None]
    if B.ndim == 2:
        B = B.unsqueeze(0).expand(count, -1, -1)
    r = int(B.shape[2])
    Acm = A.transpose(1, 2).contiguous().to(dev)  # column-major blocks
    Bcm = B.transpose(1, 2).contiguous().to(dev)
    X = torch.empty((count, r, n), dtype=torch.complex128, device=dev)
    info = torch.empty(count, dtype=torch.int32, device=dev)
    omega = torch.zeros(1, dtype=torch.float64, device=dev)
    zb = 16  # bytes per complex128
    descs = []
    for i in range(count):
        descs.append(RomDesc(n=n, r=r, F=1, ldk=n, K=C.c_void_p(Acm.data_ptr() + i * n * n * zb), M=None, D=None,
                             eta=0.0, rhs=C.c_void_p(Bcm.data_ptr() + i * n * r * zb), ldb=n,
                             omega=C.c_void_p(omega.data_ptr()), X=C.c_void_p(X.data_ptr() + i * n * r * zb),
                             info=C.c_void_p(info.data_ptr() + 4 * i), steps=None, berr=None, LU=None, ipiv=None))
    arr = (RomDesc * max(count, 1))(*descs)
    o = opts(precision, max_refine, 0.0, flags)
    check(handle.ptr, _capi.lib().srom_sweep(handle.ptr, arr, count, C.byref(o)))
    torch.cuda.synchronize(dev)  # the staged copies above must outlive the kernels
    return X.transpose(1, 2), info


@dataclasses.dataclass
class HostRom:
    """Host (numpy) buffers for ``sweep_host``; outputs are filled in place."""

    K: np.ndarray
    M: np.ndarray
    D: Optional[np.ndarray]
    rhs: np.ndarray
    omega: np.ndarray
    eta: float = 0.0
    X: Optional[np.ndarray] = None
    info: Optional[np.ndarray] = None
    steps: Optional[np.ndarray] = None
    berr: Optional[np.ndarray] = None
    C: Optional[np.ndarray] = None
    Y: Optional[np.ndarray] = None

    def __post_init__(self):
        self.K = colmajor(self.K)
        self.M = None if self.M is None else colmajor(self.M)
        self.D = None if self.D is None else colmajor(self.D)
        rhs = np.asarray(self.rhs, dtype=np.complex128)
        if rhs.ndim == 1:
            rhs = rhs[:, None]
        self.n = int(rhs.shape[0])
        self.r = int(rhs.shape[1])
        self.rhs = colmajor(rhs)
        self.omega = np.ascontiguousarray(self.omega, dtype=np.float64)
        self.F = int(self.omega.shape[0])
        if self.X is None:
            self.X = np.empty(self.F * self.n * self.r, dtype=np.complex128)
        if self.info is None:
            self.info = np.empty(self.F, dtype=np.int32)
        if self.steps is None:
            self.steps = np.empty(self.F, dtype=np.int32)
        if self.berr is None:
            self.berr = np.empty(self.F, dtype=np.float64)
        self.n_out = 0
        if self.C is not None:
            self.n_out = int(np.asarray(self.C).shape[0])
            self.C = colmajor(self.C)
            if self.Y is None:
                self.Y = np.empty(self.F * self.n_out * self.r, dtype=np.complex128)

    def desc(self) -> RomDesc:
        p = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
        return RomDesc(n=self.n, r=self.r, F=self.F, ldk=self.n, K=p(self.K), M=p(self.M),
                       D=p(self.D), eta=self.eta, rhs=p(self.rhs), ldb=self.n,
                       omega=p(self.omega), X=p(self.X), info=p(self.info), steps=p(self.steps),
                       berr=p(self.berr), LU=None, ipiv=None,
                       n_out=self.n_out, ldc=max(self.n_out, 1), C=p(self.C), Y=p(self.Y))

    def solutions(self) -> np.ndarray:
        return np.ascontiguousarray(self.X.reshape(self.F, self.r, self.n).transpose(0, 2, 1))

    def outputs(self) -> np.ndarray:
        return np.ascontiguousarray(self.Y.reshape(self.F, self.r, self.n_out).transpose(0, 2, 1))


def sweep_host(handle: _capi.Handle, roms: Sequence[HostRom], precision: int = _capi.SROM_FP64,
               max_refine: int = 5, tol: float = 0.0, flags: int = 0) -> None:
    """Synchronous sweep with host buffers (copies in, sweeps, copies out)."""
    arr = (RomDesc * max(len(roms), 1))(*[r.desc() for r in roms])
    o = opts(precision, max_refine, tol, flags)
    check(handle.ptr, _capi.lib().srom_sweep_host(handle.ptr, arr, len(roms), C.byref(o)))


class Graph:
    """A planned batched sweep captured as a CUDA graph (``srom_graph_create``)."""

    def __init__(self, handle: _capi.Handle, roms: Sequence[DeviceRom], precision: int = _capi.SROM_FP64,
                 max_refine: int = 5, tol: float = 0.0, flags: int = 0):
        self.handle = handle
        self._g = C.c_void_p()
        self._roms = list(roms)  # keep the buffers alive
        arr = (RomDesc * max(len(roms), 1))(*[r.desc() for r in roms])
        o = opts(precision, max_refine, tol, flags)
        check(handle.ptr, _capi.lib().srom_graph_create(handle.ptr, arr, len(roms), C.byref(o), C.byref(self._g)))

    def launch(self, stream_ptr: int = 0) -> None:
        check(self.handle.ptr, _capi.lib().srom_graph_launch(self._g, C.c_void_p(stream_ptr)))

    def close(self) -> None:
        if self._g:
            _capi.lib().srom_graph_destroy(self._g)
            self._g = C.c_void_p()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


def tune(handle: _capi.Handle, n_values, r: int = 1, cache_path: Optional[str] = None) -> None:
    """Autotune the FP64 kernel choice per order n (``srom_tune``), optionally with a JSON cache."""
    ns = (C.c_int * max(len(n_values), 1))(*[int(v) for v in n_values])
    check(handle.ptr, _capi.lib().srom_tune(handle.ptr, ns, len(n_values), int(r),
                                            None if cache_path is None else cache_path.encode()))
