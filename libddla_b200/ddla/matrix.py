"""Block-cyclic matrix on a handle -- mirror of the reference's python/ddla/matrix.py.

On the 1x1 grid the local partition is the whole matrix, column-major with
leading dimension LLD_, in device memory (ddla_c_malloc).  Besides the
reference's constructors, `wrap` views device memory the caller owns (for
example a torch CUDA tensor) without copying.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import numpy as np

from . import _c_api as C
from .backend import Handle

DTYPE_TO_CHAR = {
    np.dtype(np.float32): "s",
    np.dtype(np.float64): "d",
    np.dtype(np.complex64): "c",
    np.dtype(np.complex128): "z",
}
CHAR_TO_DTYPE = {v: k.type for k, v in DTYPE_TO_CHAR.items()}


class DistributedMatrix:
    def __init__(self, handle: Handle, m: int, n: int, mb: int = 64, nb: int = 64, dtype=np.float64,
                 irsrc: int = 0, icsrc: int = 0, lld: int = -1, data: Optional[np.ndarray] = None,
                 device_ptr: Optional[int] = None):
        self.handle = handle
        self.m, self.n, self.mb, self.nb = int(m), int(n), int(mb), int(nb)
        self.irsrc, self.icsrc = int(irsrc), int(icsrc)
        self.dtype = np.dtype(dtype)
        if self.dtype not in DTYPE_TO_CHAR:
            raise TypeError(f"Unsupported dtype: {self.dtype}. Supported: float32, float64, complex64, complex128")
        self.type_char = DTYPE_TO_CHAR[self.dtype]
        nprows, npcols = handle.grid_dims
        myprow, mypcol = handle.grid_coords
        self.m_loc = handle.numloc(self.m, self.mb, myprow, self.irsrc, nprows)
        self.n_loc = handle.numloc(self.n, self.nb, mypcol, self.icsrc, npcols)
        self.desc = np.zeros(C.DLEN_, dtype=np.int32)
        handle.descinit(self.desc, self.m, self.n, self.mb, self.nb, self.irsrc, self.icsrc, lld)
        self.lld = int(self.desc[C.LLD_])
        self.nbytes = self.lld * max(1, self.n_loc) * self.dtype.itemsize
        self._owned = device_ptr is None
        self._device_ptr = handle.malloc(self.nbytes) if device_ptr is None else int(device_ptr)
        self.data_ptr = self._device_ptr
        self.data = None
        if data is not None:
            self.from_host(data)

    @classmethod
    def wrap(cls, handle: Handle, device_ptr: int, m: int, n: int, lld: int, dtype, mb: int = 64, nb: int = 64):
        """View caller-owned device memory (column-major, leading dimension lld) as a matrix."""
        return cls(handle, m, n, mb=mb, nb=nb, dtype=dtype, lld=lld, device_ptr=device_ptr)

    def __del__(self):
        if getattr(self, "_owned", False) and self._device_ptr:
            try:
                self.handle.free(self._device_ptr)
            except Exception:
                pass
            self._device_ptr = 0

    @property
    def shape(self) -> Tuple[int, int]:
        return (self.m, self.n)

    @property
    def local_shape(self) -> Tuple[int, int]:
        return (self.m_loc, self.n_loc)

    def to_host(self, full_lld: bool = False) -> np.ndarray:
        """Copy the local partition (or, with full_lld, all lld rows) to a Fortran-ordered array."""
        rows = self.lld if full_lld else self.m_loc
        out = np.empty((rows, self.n_loc), dtype=self.dtype, order="F")
        es = self.dtype.itemsize
        if rows and self.n_loc:
            C.check_status(C.ddla_c_memcpy2d(self.handle.ptr, out.ctypes.data, rows * es, self._device_ptr,
                                             self.lld * es, rows * es, self.n_loc), "ddla_c_memcpy2d (to_host)")
            self.handle.synchronize()
        return out

    def from_host(self, arr: np.ndarray, full_lld: bool = False) -> None:
        rows = self.lld if full_lld else self.m_loc
        if arr.shape != (rows, self.n_loc):
            raise ValueError(f"Shape {arr.shape} != local shape ({rows}, {self.n_loc})")
        a = np.asfortranarray(arr, dtype=self.dtype)
        es = self.dtype.itemsize
        if rows and self.n_loc:
            C.check_status(C.ddla_c_memcpy2d(self.handle.ptr, self._device_ptr, self.lld * es, a.ctypes.data,
                                             rows * es, rows * es, self.n_loc), "ddla_c_memcpy2d (from_host)")
            self.handle.synchronize()

    def to_global_matrix(self, root: int = 0) -> Optional[np.ndarray]:
        out = np.zeros((self.m, self.n), dtype=self.dtype, order="F")
        f = getattr(C.lib, f"ddla_{self.type_char}_gather")
        C.check_status(f(self.handle.ptr, self.m, self.n, self._device_ptr, 1, 1, self.desc.ctypes.data, root,
                         out.ctypes.data, max(1, self.m)), f"ddla_{self.type_char}_gather")
        return out

    @classmethod
    def from_global_matrix(cls, handle: Handle, global_arr: np.ndarray, mb: int = 64, nb: int = 64, root: int = 0,
                           lld: int = -1):
        m, n = global_arr.shape
        A = cls(handle, m, n, mb=mb, nb=nb, dtype=global_arr.dtype, lld=lld)
        arr = np.asfortranarray(global_arr, dtype=A.dtype)
        f = getattr(C.lib, f"ddla_{A.type_char}_scatter")
        C.check_status(f(handle.ptr, m, n, A._device_ptr, 1, 1, A.desc.ctypes.data, root, arr.ctypes.data,
                         max(1, m)), f"ddla_{A.type_char}_scatter")
        return A
