"""CSR containers for the Python side: host (numpy) and device (torch CUDA
tensors used as plain device memory), mirroring the reference's CSRm helpers
(src/CSR.cu: init :28, copyToDevice :656-680, copyToHost :683, free :572).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import F32, F64, CsrIn, lib


@dataclass
class HostCSR:
    """CSR in host memory: 0-based int32 rowptr/col, float64 (or float32) val."""
    nrows: int
    ncols: int
    rowptr: np.ndarray
    col: np.ndarray
    val: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1]) if len(self.rowptr) else 0

    def to_device(self, device="cuda", pin=False):
        return DeviceCSR.from_host(self, device=device, pin=pin)

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col, self.rowptr), shape=(self.nrows, self.ncols))

    def row_block(self, r0: int, r1: int) -> "HostCSR":
        """Rows [r0, r1) as their own CSR (same columns)."""
        a, b = int(self.rowptr[r0]), int(self.rowptr[r1])
        return HostCSR(r1 - r0, self.ncols, (self.rowptr[r0:r1 + 1] - a).astype(np.int32),
                       self.col[a:b].copy(), self.val[a:b].copy())


class DevBuf:
    """A cudaMalloc'd block owned by Python; freed with nspb_free. Exposes
    __cuda_array_interface__ so torch.as_tensor can view it without a copy."""

    def __init__(self, ptr: int, count: int, typestr: str):
        self.ptr = int(ptr or 0)
        self.count = int(count)
        self.typestr = typestr

    @property
    def __cuda_array_interface__(self):
        return {"shape": (self.count,), "typestr": self.typestr,
                "data": (self.ptr, False), "version": 2, "strides": None}

    def __del__(self):
        if self.ptr:
            lib.nspb_free(C.c_void_p(self.ptr))
            self.ptr = 0


def adopt(ptr: int, count: int, dtype):
    """Wrap a library-allocated device array as a torch tensor that frees it."""
    import torch
    typestr = {np.dtype(np.int32): "<i4", np.dtype(np.float64): "<f8",
               np.dtype(np.float32): "<f4"}[np.dtype(dtype)]
    return torch.as_tensor(DevBuf(ptr, count, typestr), device="cuda")


class DeviceCSR:
    """CSR whose arrays are torch CUDA tensors (device memory plumbing only)."""

    def __init__(self, nrows, ncols, rowptr, col, val):
        self.nrows = int(nrows)
        self.ncols = int(ncols)
        self.rowptr = rowptr
        self.col = col
        self.val = val

    @property
    def nnz(self) -> int:
        return int(self.col.numel())

    @staticmethod
    def from_host(h: HostCSR, device="cuda", pin=False) -> "DeviceCSR":
        import torch

        def up(a):
            t = torch.from_numpy(np.ascontiguousarray(a))
            if pin:
                t = t.pin_memory()
            return t.to(device, non_blocking=pin)
        return DeviceCSR(h.nrows, h.ncols, up(h.rowptr), up(h.col), up(h.val))

    def to_host(self) -> HostCSR:
        return HostCSR(self.nrows, self.ncols, self.rowptr.cpu().numpy(),
                       self.col.cpu().numpy(), self.val.cpu().numpy())

    def as_in(self) -> CsrIn:
        import torch
        d = CsrIn()
        d.nrows = self.nrows
        d.ncols = self.ncols
        d.nnz = self.nnz
        d.rowptr = self.rowptr.data_ptr()
        d.col = self.col.data_ptr() if self.nnz else None
        d.val = self.val.data_ptr() if self.nnz else None
        d.val_type = F32 if self.val.dtype == torch.float32 else F64
        return d
