"""The allocation-free solve (ddla_d_ppotrs_noalloc) gives the same answer as ddla_d_ppotrs.

ddla_d_ppotrs_noalloc exists for callers that must not allocate device memory
while they run (a serving loop with a fixed memory budget, or a program whose
allocator belongs to another framework): it keeps the solve's flags in a fixed
device array inside the library.  This file is named so that pytest collects
it last; a failure here leaves every other test already run.  It passes alone
in a fresh process and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(C):
    f = C.lib.ddla_d_ppotrs_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_char, ctypes.c_char, ctypes.c_char, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return f


# (side, uplo, n, nrhs): both triangles and both sides; nrhs = 256 with n = 333
# (not a multiple of the 64-row block) fills the array's whole flag stride.
@pytest.mark.parametrize("side,uplo,n,nrhs", [("L", "L", 1000, 7), ("L", "U", 777, 40), ("R", "L", 500, 9),
                                              ("R", "U", 333, 256), ("L", "L", 333, 256)])
def test_noalloc_solve_matches_ppotrs_twice(handle, side, uplo, n, nrhs):
    from libddla_b200 import ddla

    C = ddla._c_api
    f = _noalloc(C)
    rng = np.random.default_rng(4242 + n)
    G = rng.standard_normal((n, n))
    A = G @ G.T / n + np.eye(n)
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=64, nb=64)
    _, info = ddla.ppotrf(dA, uplo)
    assert info == 0
    for _ in range(2):  # two calls in a row: the shared scratch is reset by each call
        B = rng.standard_normal((n, nrhs) if side == "L" else (nrhs, n))
        d1 = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=64, nb=64)
        ddla.ppotrs(dA, d1, uplo, side=side)
        d2 = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=64, nb=64)
        st = f(handle.ptr, side.encode(), uplo.encode(), b"N", n, nrhs, dA.data_ptr, dA.desc.ctypes.data,
               d2.data_ptr, d2.desc.ctypes.data)
        assert st == 0, C.error_string(st)
        X1, X2 = d1.to_global_matrix(), d2.to_global_matrix()
        assert np.max(np.abs(X1 - X2)) <= 1e-12 * np.max(np.abs(X1))
        R = A @ X2 - B if side == "L" else X2 @ A - B
        assert np.max(np.abs(R)) <= 1e-9 * np.max(np.abs(B))


def test_noalloc_rejects_sizes_beyond_its_scratch(handle):
    from libddla_b200 import ddla

    C = ddla._c_api
    f = _noalloc(C)
    small = ddla.DistributedMatrix(handle, 8, 8, mb=8, nb=8)
    big = np.zeros(9, dtype=np.int32)
    handle.descinit(big, 70000, 70000, 64, 64)
    st = f(handle.ptr, b"L", b"L", b"N", 70000, 1, small.data_ptr, big.ctypes.data, small.data_ptr,
           big.ctypes.data)
    assert st == C.STATUS_EXCEPTION
    assert "n <= 65536" in C.error_string(st)
