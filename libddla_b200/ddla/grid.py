"""Process grids of several ranks, one rank per GPU.

A grid handle is a `Handle(Backend.GPU, local_group=..., rank=r, nprows=P,
npcols=Q)` (the ranks are threads of this process: `LocalGroup`) or
`Handle(Backend.GPU, nccl_id=..., rank=r, nprows=P, npcols=Q)` (the ranks are
processes: `nccl_unique_id` on rank 0, distributed by the caller, e.g. through
torch.distributed).  Every rank then calls ppotrf / ppotrs (side 'L') / pposv
(side 'L') / pdiag_logdet with its local block-cyclic piece and the common
descriptor, as with the reference on an MPI grid.

`local_piece` / `assemble` convert between a global matrix and the ranks'
ScaLAPACK block-cyclic pieces on the host (column-major, leading dimension =
the local row count), and `run_ranks` runs one function per rank on threads
(the native calls release the GIL), re-raising the first exception.
"""
from __future__ import annotations

import ctypes
import threading
from typing import Callable, List, Optional, Sequence

import numpy as np

from . import _c_api as C


class LocalGroup:
    """The shared state of `nranks` ranks that are threads of this process.  A
    collective whose members do not all arrive within `timeout_s` seconds raises
    on the ranks that wait; the group is then unusable."""

    def __init__(self, nranks: int, timeout_s: float = 120.0):
        self._g = ctypes.c_void_p()
        C.check_status(C.ddla_c_local_group_create(ctypes.byref(self._g), int(nranks), float(timeout_s)),
                       "ddla_c_local_group_create")
        self.nranks = int(nranks)

    @property
    def ptr(self) -> ctypes.c_void_p:
        return self._g

    def close(self) -> None:
        if self._g is not None and self._g.value is not None:
            C.ddla_c_local_group_destroy(self._g)
            self._g = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def nccl_available() -> bool:
    return bool(C.ddla_c_nccl_available())


def nccl_unique_id() -> bytes:
    buf = ctypes.create_string_buffer(128)
    C.check_status(C.ddla_c_nccl_unique_id(buf), "ddla_c_nccl_unique_id")
    return buf.raw


def rank_to_rc(rank: int, nprows: int, npcols: int, major: str = "R"):
    return (rank % nprows, rank // nprows) if major == "C" else (rank // npcols, rank % npcols)


def _indices(n: int, nb: int, coord: int, src: int, nprocs: int) -> np.ndarray:
    """Global indices held by process coordinate `coord`, in local order."""
    g = np.arange(n)
    return g[((g // nb) + src) % nprocs == coord] if n else g


def local_piece(A: np.ndarray, mb: int, nb: int, nprows: int, npcols: int, row: int, col: int, rsrc: int = 0,
                csrc: int = 0) -> np.ndarray:
    """The block-cyclic local piece of the global matrix A held by grid coordinate (row, col)."""
    ri = _indices(A.shape[0], mb, row, rsrc, nprows)
    ci = _indices(A.shape[1], nb, col, csrc, npcols)
    return np.asfortranarray(A[np.ix_(ri, ci)])


def assemble(pieces: Sequence[np.ndarray], m: int, n: int, mb: int, nb: int, nprows: int, npcols: int,
             rsrc: int = 0, csrc: int = 0, major: str = "R") -> np.ndarray:
    """The global m x n matrix from every rank's local piece (pieces[rank])."""
    out = np.zeros((m, n), dtype=pieces[0].dtype)
    for rank, p in enumerate(pieces):
        row, col = rank_to_rc(rank, nprows, npcols, major)
        ri = _indices(m, mb, row, rsrc, nprows)
        ci = _indices(n, nb, col, csrc, npcols)
        out[np.ix_(ri, ci)] = p[: len(ri), : len(ci)]
    return out


def run_ranks(nranks: int, fn: Callable[[int], object]) -> List[object]:
    """fn(rank) on one thread per rank; the results in rank order.  The first exception
    (by rank) is re-raised after every thread has ended."""
    results: List[Optional[object]] = [None] * nranks
    errors: List[Optional[BaseException]] = [None] * nranks

    def body(r: int) -> None:
        try:
            results[r] = fn(r)
        except BaseException as e:  # noqa: BLE001 - re-raised below
            errors[r] = e

    threads = [threading.Thread(target=body, args=(r,), daemon=True) for r in range(nranks)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for e in errors:
        if e is not None:
            raise e
    return results


def exchange_nccl_id(group=None) -> bytes:
    """The NCCL clique id of a torch.distributed group: made by the group's first rank and
    broadcast to every rank (torch.distributed.broadcast_object_list)."""
    import torch.distributed as dist

    src = dist.get_global_rank(group, 0) if group is not None else 0
    obj = [nccl_unique_id() if dist.get_rank(group) == 0 else None]
    dist.broadcast_object_list(obj, src=src, group=group)
    return obj[0]


def nccl_grid_handle(nprows: int, npcols: int, major: str = "R", group=None):
    """This process's handle on an nprows x npcols grid formed by the ranks of a torch.distributed
    group (one process per GPU, the current CUDA device): the clique id is exchanged through the
    group, then every rank joins the NCCL clique with its group rank."""
    import torch.distributed as dist

    from .backend import Backend, Handle

    world = dist.get_world_size(group)
    if nprows * npcols != world:
        raise ValueError(f"a {nprows} x {npcols} grid needs {nprows * npcols} ranks, the group has {world}")
    uid = exchange_nccl_id(group)
    return Handle(Backend.GPU, nccl_id=uid, rank=dist.get_rank(group), nprows=nprows, npcols=npcols, major=major)
