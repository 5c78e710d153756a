"""The reference's 1x1 CPU arm through real LAPACK (TEST AND CPU-BASELINE INFRASTRUCTURE ONLY).

On a CPU handle with a 1x1 grid the reference's pposv is exactly
    ?potrf_(uplo, n, A, LLD, info)                    src/Cholesky/potrf.cpp:41-59
    ?trsm_(side, uplo, first,  'N', m, n, 1, A, ...)  src/BLAS/trsm.cpp:137-144
    ?trsm_(side, uplo, second, 'N', m, n, 1, A, ...)  first/second: src/Cholesky/ppotrs.cpp:44-48
against the CPU BLAS/LAPACK it was linked with.  Here that library is the
OpenBLAS bundled with scipy (threadpool_info() reports version and core type),
reached through scipy.linalg.lapack / scipy.linalg.blas.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg.blas as blas
import scipy.linalg.lapack as lapack

_P = {np.dtype(np.float32): "s", np.dtype(np.float64): "d", np.dtype(np.complex64): "c",
      np.dtype(np.complex128): "z"}


def blas_info() -> dict:
    try:
        from threadpoolctl import threadpool_info

        for d in threadpool_info():
            if d.get("internal_api") == "openblas" and "scipy.libs" in d.get("filepath", ""):
                return {"library": "OpenBLAS", "version": d.get("version"), "core": d.get("architecture"),
                        "threads": d.get("num_threads")}
        for d in threadpool_info():
            if d.get("user_api") == "blas":
                return {"library": d.get("internal_api"), "version": d.get("version"),
                        "core": d.get("architecture"), "threads": d.get("num_threads")}
    except Exception:
        pass
    return {"library": "unknown"}


def potrf(a: np.ndarray, uplo: str = "L", overwrite: bool = False):
    p = _P[a.dtype]
    f = getattr(lapack, f"{p}potrf")
    c, info = f(a, lower=(uplo == "L"), clean=False, overwrite_a=overwrite)
    return c, int(info)


def ppotrs(c: np.ndarray, b: np.ndarray, uplo: str = "L", overwrite: bool = False):
    """Side 'L': the two ?trsm_ calls of ppotrs_run (uplo 'L': L then L^H; 'U': U^H then U)."""
    p = _P[c.dtype]
    trsm = getattr(blas, f"{p}trsm")
    lower = uplo == "L"
    first = 0 if lower else 2   # 'N' for L, 'C' for U (left side)
    second = 2 if lower else 0
    y = trsm(1.0, c, b, side=0, lower=lower, trans_a=first, diag=0, overwrite_b=overwrite)
    return trsm(1.0, c, y, side=0, lower=lower, trans_a=second, diag=0, overwrite_b=True)


def pposv(a: np.ndarray, b: np.ndarray, uplo: str = "L", overwrite: bool = False):
    c, info = potrf(a, uplo, overwrite=overwrite)
    if info != 0:
        return c, b, info
    return c, ppotrs(c, b, uplo, overwrite=overwrite), 0
