"""Analytic fixtures of the reference's own Cholesky tests, restated in NumPy.

The reference ships no golden data files; its tests build known answers from
closed-form generators, which are restated here (same formulas, same
accumulation order) so that the committed fixtures and the tests can use them:

  kat_factor / kat_matrix   tests/test_ppotrf_grids.cpp:11-26 (factor<T>(i,j),
                            matrix<T>(i,j) = sum_k factor(i,k) conj(factor(j,k)))
  spd_value / x_value_real  tests/test_ppotrf_real.cpp:10-23
  hpd_value / x_value       tests/api_grid_test_common.h:490-537
  logdet cases              tests/test_diag_logdet.cpp:76-111 (+ the long-double
                            reference of lines 21-30)
  python cases              python/tests/test_cholesky.py:12-92 (legacy NumPy seeds)
"""
from __future__ import annotations

import math

import numpy as np

REAL = {np.dtype(np.float32): np.float32, np.dtype(np.float64): np.float64,
        np.dtype(np.complex64): np.float32, np.dtype(np.complex128): np.float64}
DTYPES = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}


def _scalar(dtype, re, im=0.0):
    dt = np.dtype(dtype)
    if np.issubdtype(dt, np.complexfloating):
        return dt.type(complex(re, im))
    return dt.type(re)


def kat_factor(n: int, dtype) -> np.ndarray:
    """factor<T>(i,j) for i >= j, zero above (test_ppotrf_grids.cpp:17-20)."""
    dt = np.dtype(dtype)
    L = np.zeros((n, n), dtype=dt)
    for i in range(n):
        for j in range(i + 1):
            if i == j:
                L[i, j] = _scalar(dt, 2 + .01 * i)
            else:
                L[i, j] = _scalar(dt, .003 * (1 + (i + j) % 5), .002 * (i - j))
    return L


def kat_matrix(n: int, dtype) -> np.ndarray:
    """matrix<T>(i,j) = sum_{k <= min(i,j)} factor(i,k) * conj(factor(j,k)), accumulated in T in k order."""
    L = kat_factor(n, dtype)
    A = np.zeros((n, n), dtype=L.dtype)
    Lc = np.conj(L)
    for k in range(n):
        # term k contributes to all (i,j) with i,j >= k; factor(i,k) = 0 for i < k
        A += np.outer(L[:, k], Lc[:, k]).astype(L.dtype)
    return A


def spd_value(n: int, dtype) -> np.ndarray:
    i = np.arange(n)[:, None]
    j = np.arange(n)[None, :]
    lo, hi = np.minimum(i, j), np.maximum(i, j)
    A = 0.01 * ((lo + 2 * hi) % 5 - 2).astype(np.float64)
    A[np.arange(n), np.arange(n)] = 6.0 + 0.05 * np.arange(n)
    return A.astype(dtype)


def x_value_real(n: int, nrhs: int, dtype) -> np.ndarray:
    i = np.arange(n)[:, None]
    j = np.arange(nrhs)[None, :]
    return (0.2 + 0.03 * i - 0.02 * j).astype(dtype)


def hpd_value(n: int) -> np.ndarray:
    i = np.arange(n)[:, None]
    j = np.arange(n)[None, :]
    lo, hi = np.minimum(i, j), np.maximum(i, j)
    val = 0.01 * ((lo + 2 * hi) % 5 - 2) + 1j * 0.006 * ((3 * lo + hi) % 7 - 3)
    A = np.where(i < j, val, np.conj(val))
    A[np.arange(n), np.arange(n)] = 5.0 + 0.2 * n + 0.05 * np.arange(n)
    return A.astype(np.complex128)


def x_value(n: int, nrhs: int) -> np.ndarray:
    i = np.arange(n)[:, None]
    j = np.arange(nrhs)[None, :]
    return (0.2 + 0.03 * i - 0.02 * j) + 1j * (0.04 * (i + 1) + 0.01 * j)


def rhs_sequential(A: np.ndarray, X: np.ndarray) -> np.ndarray:
    """B(i,j) = sum_l A(i,l) X(l,j) accumulated in l order in A's dtype (build_rhs)."""
    B = np.zeros((A.shape[0], X.shape[1]), dtype=A.dtype)
    X = X.astype(A.dtype)
    for l in range(A.shape[1]):
        B += np.outer(A[:, l], X[l, :]).astype(A.dtype)
    return B


def logdet_reference(diag) -> complex | None:
    """test_diag_logdet.cpp:21-30: sum log|z| and atan2, remainder of the phase by 2 pi;
    None for a nonfinite entry (the routine throws)."""
    mag = 0.0
    phase = 0.0
    zero = False
    for z in diag:
        z = complex(z)
        if not (math.isfinite(z.real) and math.isfinite(z.imag)):
            return None
        hi = max(abs(z.real), abs(z.imag))
        lo = min(abs(z.real), abs(z.imag))
        if hi == 0:
            zero = True
        else:
            # log|z| without forming |z| (hypot(DBL_MAX, DBL_MAX) overflows in double;
            # the reference evaluates it in long double)
            mag += math.log(hi) + 0.5 * math.log1p((lo / hi) ** 2)
            phase += math.atan2(z.imag, z.real)
    if zero:
        return complex(-math.inf, 0.0)
    return complex(mag, math.remainder(phase, 2 * math.pi))


def logdet_cases(dtype) -> list:
    """The diagonals exercised by test_diag_logdet.cpp:78-95 for one scalar type."""
    dt = np.dtype(dtype)
    R = REAL[dt]
    fi = np.finfo(R)
    cplx = np.issubdtype(dt, np.complexfloating)

    def v(x, y=0.0):
        return _scalar(dt, x, y if cplx else 0.0)

    cases = [
        [],
        [v(2), v(3), v(5)],
        [v(-2), v(3), v(5)],
        [v(-2), v(-3), v(5)],
        [v(0), v(-3), v(5)],
        [v(fi.max, fi.max), v(fi.smallest_subnormal, -fi.smallest_subnormal)],
    ]
    if cplx:
        z = np.exp(1j * R(.8) * R(np.pi)).astype(dt)
        cases.append([z, z, z])
    cases.append([v(1), v(np.inf)])
    cases.append([v(1), v(np.nan)])
    cases.append([v(1 + i % 3) for i in range(11)])
    return cases


def python_cases():
    """The seeded cases of python/tests/test_cholesky.py (legacy global RandomState)."""
    out = {}
    np.random.seed(55)
    M = np.random.randn(32, 32)
    out["ppotrf_ppotrs"] = (M @ M.T + np.eye(32) * 10.0, np.random.randn(32, 4))
    np.random.seed(56)
    M = np.random.randn(24, 24)
    out["pposv"] = (M @ M.T + np.eye(24) * 5.0, np.random.randn(24, 2))
    rng = np.random.RandomState(57)
    n = 15
    typed = []
    for dtype in (np.float32, np.float64, np.complex64, np.complex128):
        for uplo in ("L", "U"):
            M = rng.randn(n, n)
            X = rng.randn(n, 2)
            if np.issubdtype(dtype, np.complexfloating):
                M = M + 1j * rng.randn(n, n)
                X = X + 1j * rng.randn(n, 2)
            M = M.astype(dtype)
            X = X.astype(dtype)
            A = (M @ M.conj().T + np.eye(n, dtype=dtype) * 10).astype(dtype)
            typed.append((np.dtype(dtype).char, uplo, A, X, (A @ X).astype(dtype)))
    out["typed"] = typed
    return out
