"""Handle lifecycle -- mirror of the reference's python/ddla/backend.py."""
from __future__ import annotations

import ctypes
import enum
from typing import Optional

import numpy as np

from . import _c_api as C
from .layout import ProcessorLayout


class Backend(enum.IntEnum):
    CPU = C.BACKEND_CPU
    GPU = C.BACKEND_GPU


class Communication(enum.IntEnum):
    MPI = C.COMMUNICATION_MPI
    HOST_STAGED_MPI = C.COMMUNICATION_HOST_STAGED_MPI
    CCL = C.COMMUNICATION_CCL


class Handle:
    """Owns one ddla handle: backend, process grid and the CUDA stream.

    The grid is 1x1 by default.  A grid of several ranks (one rank per GPU, this
    handle's current device) is joined with `local_group` (a grid.LocalGroup: the
    ranks are threads of this process) or `nccl_id` (the 128-byte clique id from
    grid.nccl_unique_id on rank 0: the ranks are processes), with `rank` and
    `nprows` x `npcols`."""

    def __init__(self, backend: Backend, layout: Optional[ProcessorLayout] = None, comm=None,
                 nprows: Optional[int] = None, npcols: Optional[int] = None, major: str = "R",
                 local_group=None, nccl_id: Optional[bytes] = None, rank: int = 0):
        self._handle = ctypes.c_void_p()
        if backend is None:
            raise TypeError("backend must explicitly select CPU or GPU")
        C.check_status(C.ddla_c_init_backend(ctypes.byref(self._handle), int(backend)), "ddla_c_init_backend")
        if local_group is not None or nccl_id is not None:
            if nprows is None or npcols is None:
                self.destroy()
                raise ValueError("a grid of several ranks needs nprows and npcols")
            self.layout = None
            if local_group is not None:
                st = C.ddla_c_set_local_group(self._handle, local_group.ptr, int(rank), int(nprows), int(npcols),
                                              major.encode())
                what = "ddla_c_set_local_group"
            else:
                idbuf = ctypes.create_string_buffer(bytes(nccl_id), 128)
                st = C.ddla_c_set_nccl(self._handle, idbuf, int(nprows) * int(npcols), int(rank), int(nprows),
                                       int(npcols), major.encode())
                what = "ddla_c_set_nccl"
            if st != C.STATUS_SUCCESS:
                self.destroy()
            C.check_status(st, what)
            return
        if layout is None:
            layout = ProcessorLayout(comm=comm, np_rows=nprows, np_cols=npcols, major=major)
        self.layout = layout
        st = C.ddla_c_set(self._handle, layout.comm_f, layout.np_rows, layout.np_cols, layout.major.encode())
        if st != C.STATUS_SUCCESS:
            self.destroy()
        C.check_status(st, "ddla_c_set")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def destroy(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value is not None:
            C.ddla_c_destroy(ctypes.byref(h))
            self._handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    @property
    def ptr(self) -> ctypes.c_void_p:
        return self._handle

    @property
    def backend(self) -> Backend:
        return Backend(C.ddla_c_get_backend(self._handle))

    @staticmethod
    def is_backend_available(backend: Backend) -> bool:
        return bool(C.ddla_c_backend_available(int(backend)))

    @property
    def communication(self) -> Communication:
        v = ctypes.c_int()
        C.check_status(C.ddla_c_get_communication(self._handle, ctypes.byref(v)), "ddla_c_get_communication")
        return Communication(v.value)

    def set_communication(self, mode: Communication) -> None:
        C.check_status(C.ddla_c_set_communication(self._handle, int(mode)), "ddla_c_set_communication")

    @property
    def grid_dims(self):
        r, c = ctypes.c_int(), ctypes.c_int()
        C.check_status(C.ddla_c_grid_dims(self._handle, ctypes.byref(r), ctypes.byref(c)), "ddla_c_grid_dims")
        return r.value, c.value

    @property
    def grid_coords(self):
        r, c = ctypes.c_int(), ctypes.c_int()
        C.check_status(C.ddla_c_grid_coords(self._handle, ctypes.byref(r), ctypes.byref(c)), "ddla_c_grid_coords")
        return r.value, c.value

    @property
    def rank(self) -> int:
        return C.ddla_c_rank(self._handle)

    @property
    def size(self) -> int:
        return C.ddla_c_size(self._handle)

    def numloc(self, n, nb, iproc, srcproc, nprocs) -> int:
        return C.ddla_c_numloc(int(n), int(nb), int(iproc), int(srcproc), int(nprocs))

    def descinit(self, desc: np.ndarray, m, n, mb, nb, irsrc=0, icsrc=0, lld=-1) -> None:
        if desc.dtype != np.int32 or desc.size < C.DLEN_:
            raise ValueError("descriptor must be an int32 array of length 9")
        C.check_status(C.ddla_c_descinit(desc.ctypes.data, self._handle, int(m), int(n), int(mb), int(nb),
                                         int(irsrc), int(icsrc), int(lld)), "ddla_c_descinit")

    def malloc(self, nbytes: int) -> int:
        p = ctypes.c_void_p()
        C.check_status(C.ddla_c_malloc(self._handle, ctypes.byref(p), int(nbytes)), "ddla_c_malloc")
        return p.value or 0

    def free(self, ptr: int) -> None:
        C.check_status(C.ddla_c_free(self._handle, ptr), "ddla_c_free")

    def memcpy(self, dst: int, src: int, nbytes: int) -> None:
        C.check_status(C.ddla_c_memcpy(self._handle, dst, src, int(nbytes)), "ddla_c_memcpy")

    def memset(self, ptr: int, value: int, nbytes: int) -> None:
        C.check_status(C.ddla_c_memset(self._handle, ptr, int(value), int(nbytes)), "ddla_c_memset")

    def synchronize(self) -> None:
        C.check_status(C.ddla_c_synchronize(self._handle), "ddla_c_synchronize")
