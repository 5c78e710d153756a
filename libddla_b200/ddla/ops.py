"""Cholesky-path routines -- mirror of ppotrf / ppotrs / pposv in the reference's
python/ddla/ops.py:113-143, plus potrf, potrf_bottom_right / ppotrf_bottom_right,
diag_logdet / pdiag_logdet and pposv_mixed."""
from __future__ import annotations

import ctypes
from typing import Tuple, Union

import numpy as np

from . import _c_api as C
from .matrix import DistributedMatrix


def _ch(c: Union[str, bytes]) -> bytes:
    if isinstance(c, bytes):
        return c.upper()
    return c.upper().encode("ascii")


def ppotrf(A: DistributedMatrix, uplo: str = "L") -> Tuple[DistributedMatrix, int]:
    """Cholesky factorization in place; returns (A, info)."""
    info = ctypes.c_int(0)
    f = getattr(C.lib, f"ddla_{A.type_char}_ppotrf")
    C.check_status(f(A.handle.ptr, _ch(uplo), A.n, A.data_ptr, 1, 1, A.desc.ctypes.data, ctypes.byref(info)),
                   f"ddla_{A.type_char}_ppotrf")
    return A, info.value


def ppotrs(A: DistributedMatrix, B: DistributedMatrix, uplo: str = "L", side: str = "L",
           trans: str = "N") -> DistributedMatrix:
    """Solve A X = B (side 'L') or X A = B (side 'R') with the factor from ppotrf; X overwrites B."""
    s = _ch(side)
    nrhs = B.n if s == b"L" else B.m
    f = getattr(C.lib, f"ddla_{A.type_char}_ppotrs")
    C.check_status(f(A.handle.ptr, s, _ch(uplo), _ch(trans), A.n, nrhs, A.data_ptr, A.desc.ctypes.data,
                     B.data_ptr, B.desc.ctypes.data), f"ddla_{A.type_char}_ppotrs")
    return B


def pposv(A: DistributedMatrix, B: DistributedMatrix, uplo: str = "L", side: str = "L",
          trans: str = "N") -> Tuple[DistributedMatrix, int]:
    """Factor and solve in one native call (ddla::pposv); returns (B, info), B untouched when info != 0."""
    s = _ch(side)
    nrhs = B.n if s == b"L" else B.m
    info = ctypes.c_int(0)
    f = getattr(C.lib, f"ddla_{A.type_char}_pposv")
    C.check_status(f(A.handle.ptr, s, _ch(uplo), _ch(trans), A.n, nrhs, A.data_ptr, 1, 1, A.desc.ctypes.data,
                     B.data_ptr, 1, 1, B.desc.ctypes.data, ctypes.byref(info)), f"ddla_{A.type_char}_pposv")
    return B, info.value


def potrf(handle, type_char: str, uplo: str, n: int, A_ptr: int, lda: int, dinfo_ptr: int) -> None:
    """LAPACK-style potrf with a DEVICE info pointer (asynchronous on the handle's stream)."""
    f = getattr(C.lib, f"ddla_{type_char}_potrf")
    C.check_status(f(handle.ptr, _ch(uplo), int(n), A_ptr, int(lda), dinfo_ptr), f"ddla_{type_char}_potrf")


def potrf_bottom_right(handle, type_char: str, uplo: str, n: int, A_ptr: int, lda: int) -> int:
    """Cholesky from the bottom-right corner in place (A = U U^H for 'U', L^H L for 'L');
    returns info (0, or the index of the failed pivot).  The binding of
    ddla_?_potrf_bottom_right (the reference's fortran/ddla_c_api.cpp:1191-1225)."""
    info = ctypes.c_int(0)
    f = getattr(C.lib, f"ddla_{type_char}_potrf_bottom_right")
    C.check_status(f(handle.ptr, _ch(uplo), int(n), A_ptr, int(lda), ctypes.byref(info)),
                   f"ddla_{type_char}_potrf_bottom_right")
    return info.value


def ppotrf_bottom_right(A: DistributedMatrix, uplo: str = "U") -> Tuple[DistributedMatrix, int]:
    """Bottom-right Cholesky of a descriptor-described matrix in place; returns (A, info)."""
    info = ctypes.c_int(0)
    f = getattr(C.lib, f"ddla_{A.type_char}_ppotrf_bottom_right")
    C.check_status(f(A.handle.ptr, _ch(uplo), A.n, A.data_ptr, A.desc.ctypes.data, ctypes.byref(info)),
                   f"ddla_{A.type_char}_ppotrf_bottom_right")
    return A, info.value


def pdiag_logdet(A: DistributedMatrix, n: int = -1) -> complex:
    """diag_logdet through A's descriptor (ddla_?_pdiag_logdet; the reference's
    src/PBLAS/pdiag_logdet.cpp on a 1x1 grid)."""
    n = A.n if n < 0 else n
    out = np.zeros(2, dtype=np.float32 if A.type_char in "sc" else np.float64)
    f = getattr(C.lib, f"ddla_{A.type_char}_pdiag_logdet")
    C.check_status(f(A.handle.ptr, int(n), A.data_ptr, A.desc.ctypes.data, out.ctypes.data),
                   f"ddla_{A.type_char}_pdiag_logdet")
    return complex(float(out[0]), float(out[1]))


def pdiag_logdet_local(handle, type_char: str, n: int, a_ptr: int, desc, grid) -> np.ndarray:
    """This rank's pdiag_logdet state {magnitude, phase, zero, negative parity, nonfinite} over the
    diagonal entries its local matrix (device pointer a_ptr, int[9] descriptor desc) holds, for rank
    (row, col) of a pr x pc grid, grid = (pr, pc, row, col) (ddla_?_pdiag_logdet_local)."""
    pr, pc, row, col = (int(v) for v in grid)
    d = np.ascontiguousarray(desc, dtype=np.int32)
    state = np.zeros(5, dtype=np.float64)
    f = getattr(C.lib, f"ddla_{type_char}_pdiag_logdet_local")
    C.check_status(f(handle.ptr, int(n), a_ptr, d.ctypes.data, pr, pc, row, col, state.ctypes.data),
                   f"ddla_{type_char}_pdiag_logdet_local")
    return state


def pdiag_logdet_finish(total, single: bool = False) -> complex:
    """log det from the states summed over every rank (ddla_c_pdiag_logdet_finish); raises on every
    rank when any rank saw a nonfinite diagonal entry."""
    t = np.ascontiguousarray(total, dtype=np.float64)
    if t.shape != (5,):
        raise ValueError("pdiag_logdet_finish: five summed doubles expected")
    out = np.zeros(2, dtype=np.float32 if single else np.float64)
    C.check_status(C.ddla_c_pdiag_logdet_finish(t.ctypes.data, int(bool(single)), out.ctypes.data),
                   "ddla_c_pdiag_logdet_finish")
    return complex(float(out[0]), float(out[1]))


def pdiag_logdet_grid(handle, type_char: str, n: int, a_ptr: int, desc, grid, group=None,
                      local_state=None) -> complex:
    """pdiag_logdet of a matrix distributed block-cyclically over the ranks of a torch.distributed
    group arranged as a pr x pc grid: this rank's state (ddla_?_pdiag_logdet_local, or `local_state`
    when the caller already has it), ONE all-reduce (sum) of its five doubles -- the reference's
    MPI_Allreduce of src/PBLAS/pdiag_logdet.cpp:45 -- and the finish.  Every rank of the group must
    call it; all get the same result (or all raise)."""
    import torch
    import torch.distributed as dist

    state = local_state if local_state is not None else pdiag_logdet_local(handle, type_char, n, a_ptr, desc, grid)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.as_tensor(np.asarray(state, dtype=np.float64), device=dev).clone()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return pdiag_logdet_finish(t.cpu().numpy(), single=type_char in "sc")


def phegst(A: DistributedMatrix, F: DistributedMatrix, uplo: str = "L", n: int = -1) -> DistributedMatrix:
    """A <- L^-1 A L^-H in place with F holding the Cholesky factor of B (ddla_?_phegst;
    the reference's phegst on a 1x1 grid).  Returns A."""
    n = A.n if n < 0 else n
    f = getattr(C.lib, f"ddla_{A.type_char}_phegst")
    C.check_status(f(A.handle.ptr, _ch(uplo), int(n), A.data_ptr, A.desc.ctypes.data, F.data_ptr,
                     F.desc.ctypes.data), f"ddla_{A.type_char}_phegst")
    return A


def diag_logdet(A: DistributedMatrix, n: int = -1) -> complex:
    """Principal log of the product of the diagonal of the leading n x n of A."""
    n = A.n if n < 0 else n
    out = np.zeros(2, dtype=np.float32 if A.type_char in "sc" else np.float64)
    f = getattr(C.lib, f"ddla_{A.type_char}_diag_logdet")
    C.check_status(f(A.handle.ptr, int(n), A.data_ptr, A.lld, out.ctypes.data), f"ddla_{A.type_char}_diag_logdet")
    return complex(float(out[0]), float(out[1]))


def pposv_mixed(A: DistributedMatrix, B: DistributedMatrix, X: DistributedMatrix, precision: str = "B",
                uplo: str = "L"):
    """FP64-accurate solve from a low-precision tensor-core factor plus refinement.

    Returns (X, info, report) with report = {iter, gmres, shift, backward_error}; A is left
    unchanged unless the routine fell back to the FP64 factorization (iter < 0)."""
    if A.type_char != "d":
        raise TypeError("pposv_mixed takes float64 matrices")
    info = ctypes.c_int(0)
    rep = (ctypes.c_double * 4)()
    C.check_status(C.ddla_d_pposv_mixed(A.handle.ptr, _ch(uplo), _ch(precision), A.n, B.n, A.data_ptr,
                                        A.desc.ctypes.data, B.data_ptr, B.desc.ctypes.data, X.data_ptr,
                                        X.desc.ctypes.data, ctypes.byref(info), rep), "ddla_d_pposv_mixed")
    report = {"iter": int(rep[0]), "gmres": int(rep[1]), "shift": float(rep[2]), "backward_error": float(rep[3])}
    return X, info.value, report


def pposv_mixed_host(handle, A, B, precision: str = "T", uplo: str = "L", X=None):
    """pposv_mixed on host arrays (ddla_d_pposv_mixed_host): A (n x n) and B (n x nrhs) float64 in
    host memory, column-major; only A's lower triangle is read.  A streams to the device by column
    panels while the arrived panels are factored; with pinned arrays (for instance the .numpy() view
    of a torch tensor made with pin_memory=True) the copy overlaps the factorization.  Returns
    (X, info, report); X is a new Fortran-ordered array unless one is given."""
    import numpy as np

    A = np.asarray(A)
    B = np.asarray(B)
    if A.dtype != np.float64 or B.dtype != np.float64:
        raise TypeError("pposv_mixed_host takes float64 arrays")
    A = np.asfortranarray(A)
    B = np.asfortranarray(B if B.ndim == 2 else B[:, None])
    n, nrhs = A.shape[0], B.shape[1]
    if X is None:
        X = np.empty((n, nrhs), dtype=np.float64, order="F")
    info = ctypes.c_int(0)
    rep = (ctypes.c_double * 4)()
    C.check_status(C.ddla_d_pposv_mixed_host(handle.ptr, _ch(uplo), _ch(precision), n, nrhs, A.ctypes.data,
                                             max(1, A.shape[0]), B.ctypes.data, max(1, B.shape[0]), X.ctypes.data,
                                             max(1, X.shape[0]), ctypes.byref(info), rep),
                   "ddla_d_pposv_mixed_host")
    report = {"iter": int(rep[0]), "gmres": int(rep[1]), "shift": float(rep[2]), "backward_error": float(rep[3])}
    return X, info.value, report


def gather(A: DistributedMatrix, root: int = 0):
    return A.to_global_matrix(root)


def scatter(handle, arr, mb: int = 64, nb: int = 64, root: int = 0):
    return DistributedMatrix.from_global_matrix(handle, arr, mb=mb, nb=nb, root=root)
