"""Variable-size batched GEMM (gemmVbatched; ddla_?_gemm_vbatched through the C ABI).

The cases follow the reference's own test (tests/test_gemm_vbatched.cpp): its
standard case (three entries of sizes 2..5 with padded leading dimensions, the
ten transpose pairs, beta in {0, 1, other} with NaN in C when beta is 0, the
padding rows checked unchanged bit for bit), its zero-product cases (k = 0 and
alpha = 0 with null A and B arrays), its tolerances (1e-5 for FP32, 1e-12 for
FP64, absolute), an empty batch with null arrays, a null handle; plus entries
larger than one 64 x 64 tile, m / n / k of 0, null entries, more than 65535
entries, and every argument error with the reference's message.

The CPU tests pin the oracle's restatement against a loop port of the reference
test's reference_gemm on the same generated inputs.
"""
import ctypes

import numpy as np
import pytest

from oracle import restated

DT = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}
TOL = {"s": 1e-5, "d": 1e-12, "c": 1e-5, "z": 1e-12}
OPS = [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T"), ("C", "N"), ("N", "C"), ("C", "C"), ("T", "C"),
       ("C", "T"), ("n", "t")]


def _value(p, index):
    """The reference test's input generator (tests/test_gemm_vbatched.cpp:28-44)."""
    if p in "cz":
        return complex(((index % 13) - 6) / 7.0, ((index % 9) - 4) / 11.0)
    return ((index % 13) - 6) / 7.0


def _matrix(p, ld, cols, seed):
    return np.array([_value(p, seed + i) for i in range(ld * cols)], dtype=DT[p])


def _rows(op, m, k):
    return m if op in "Nn" else k


def _cols(op, m, k):
    return k if op in "Nn" else m


def _standard_inputs(p, ta, tb):
    m, n, k = [2, 4, 3], [3, 2, 5], [4, 3, 2]
    lda = [_rows(ta, m[b], k[b]) + 1 for b in range(3)]
    ldb = [_rows(tb, k[b], n[b]) + 2 for b in range(3)]
    ldc = [m[b] + 1 for b in range(3)]
    A = [_matrix(p, lda[b], _cols(ta, m[b], k[b]), 101 * b + 1) for b in range(3)]
    B = [_matrix(p, ldb[b], _cols(tb, k[b], n[b]), 101 * b + 29) for b in range(3)]
    C = [_matrix(p, ldc[b], n[b], 101 * b + 53) for b in range(3)]
    alpha = DT[p](1 + _value(p, 19))
    return m, n, k, lda, ldb, ldc, A, B, C, alpha


def _loop_gemm(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
    """Loop port of the reference test's reference_gemm (tests/test_gemm_vbatched.cpp:56-90)."""
    def el(X, ld, r, c, op):
        if op in "Nn":
            return X[r + c * ld]
        v = X[c + r * ld]
        return np.conj(v) if op in "Cc" else v

    C = C.copy()
    for j in range(n):
        for i in range(m):
            s = 0
            if alpha != 0:
                for l in range(k):
                    s += el(A, lda, i, l, ta) * el(B, ldb, l, j, tb)
            prod = alpha * s
            C[i + j * ldc] = prod if beta == 0 else prod + beta * C[i + j * ldc]
    return C


# ---- CPU: the oracle against the reference test's own reference product -------------

@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("ta,tb", OPS)
def test_oracle_matches_reference_test_loop(p, ta, tb):
    m, n, k, lda, ldb, ldc, A, B, C, alpha = _standard_inputs(p, ta, tb)
    for beta in (DT[p](0), DT[p](1), DT[p](_value(p, 23))):
        got = restated.gemm_vbatched(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc)
        for b in range(3):
            ref = _loop_gemm(ta, tb, m[b], n[b], k[b], complex(alpha) if p in "cz" else float(alpha),
                             A[b].astype(np.complex128 if p in "cz" else np.float64), lda[b],
                             B[b].astype(np.complex128 if p in "cz" else np.float64), ldb[b],
                             complex(beta) if p in "cz" else float(beta),
                             C[b].astype(np.complex128 if p in "cz" else np.float64), ldc[b])
            assert np.max(np.abs(got[b] - ref)) <= TOL[p]


def test_oracle_edge_rules():
    C0 = np.arange(12, dtype=np.float64)
    nan = np.full(12, np.nan)
    # k == 0 and alpha == 0 scale by beta without reading A / B (None here)
    for k, alpha in ((0, 1.0), (3, 0.0)):
        out = restated.gemm_vbatched("N", "N", [3], [4], [k], alpha, [None], [3], [None], [3], 2.0, [C0], [3])
        assert np.array_equal(out[0], 2.0 * C0)
        out = restated.gemm_vbatched("N", "N", [3], [4], [k], alpha, [None], [3], [None], [3], 0.0, [nan], [3])
        assert np.array_equal(out[0], np.zeros(12))
        out = restated.gemm_vbatched("N", "N", [3], [4], [k], alpha, [None], [3], [None], [3], 1.0, [nan], [3])
        assert np.isnan(out[0]).all()
    # null entries and empty sizes leave C
    out = restated.gemm_vbatched("N", "N", [3, 0], [4, 4], [2, 2], 1.0, [None, C0], [3, 1], [C0, C0], [2, 2], 0.5,
                                 [C0, C0], [3, 1])
    assert np.array_equal(out[0], C0) and np.array_equal(out[1], C0)


# ---- GPU ----------------------------------------------------------------------------

def _torch():
    import torch
    return torch


def _dev(x):
    torch = _torch()
    return None if x is None else torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _run(handle, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
    from libddla_b200.ddla import batched
    dA, dB, dC = [_dev(a) for a in A], [_dev(b) for b in B], [_dev(c) for c in C]
    # null entries still need a typed tensor somewhere to fix the routine's type
    if all(t is None for t in dA + dB + dC):
        raise ValueError("test needs at least one matrix")
    batched.gemm_vbatched(handle, ta, tb, m, n, k, alpha, dA, lda, dB, ldb, beta, dC, ldc)
    return [None if t is None else t.cpu().numpy() for t in dC]


@pytest.mark.gpu
@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("ta,tb", OPS)
def test_standard_case_matches_oracle(handle, p, ta, tb):
    m, n, k, lda, ldb, ldc, A, B, C, alpha = _standard_inputs(p, ta, tb)
    for beta in (DT[p](0), DT[p](1), DT[p](_value(p, 23))):
        inp = [c.copy() for c in C]
        if beta == 0:
            for b in range(3):
                inp[b].reshape(n[b], ldc[b]).T[:m[b]] = np.nan
        want = restated.gemm_vbatched(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, inp, ldc)
        got = _run(handle, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, inp, ldc)
        for b in range(3):
            g = got[b].reshape(n[b], ldc[b]).T
            x = inp[b].reshape(n[b], ldc[b]).T
            assert g[m[b]:].tobytes() == x[m[b]:].tobytes(), "padding rows modified"
            assert np.all(np.isfinite(got[b]))
            assert np.max(np.abs(got[b] - want[b])) <= TOL[p], (p, ta, tb, beta, b)


@pytest.mark.gpu
@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "C"), ("C", "N")])
@pytest.mark.parametrize("zero_alpha", [False, True])
def test_zero_product_scales_c_without_reading_inputs(handle, p, ta, tb, zero_alpha):
    m, n = [2, 33, 65], [3, 17, 67]
    k = [5, 7, 9] if zero_alpha else [0, 0, 0]
    lda = [_rows(ta, m[b], k[b]) + 1 for b in range(3)]
    ldb = [_rows(tb, k[b], n[b]) + 2 for b in range(3)]
    ldc = [m[b] + 3 for b in range(3)]
    C = [_matrix(p, ldc[b], n[b], 31 * b + 7) for b in range(3)]
    alpha = DT[p](0 if zero_alpha else 1)
    for beta in (DT[p](0), DT[p](1), DT[p](_value(p, 23))):
        inp = [c.copy() for c in C]
        if beta == 0:
            for b in range(3):
                inp[b].reshape(n[b], ldc[b]).T[:m[b]] = np.nan
        want = restated.gemm_vbatched(ta, tb, m, n, k, alpha, [None] * 3, lda, [None] * 3, ldb, beta, inp, ldc)
        got = _run(handle, ta, tb, m, n, k, alpha, [None] * 3, lda, [None] * 3, ldb, beta, inp, ldc)
        for b in range(3):
            g = got[b].reshape(n[b], ldc[b]).T
            x = inp[b].reshape(n[b], ldc[b]).T
            assert g[m[b]:].tobytes() == x[m[b]:].tobytes()
            if beta == 1:
                assert got[b].tobytes() == inp[b].tobytes()
            assert np.max(np.abs(got[b] - want[b])) <= TOL[p]


def _random(p, rng, size):
    x = rng.standard_normal(size)
    if p in "cz":
        x = x + 1j * rng.standard_normal(size)
    return x.astype(DT[p])


@pytest.mark.gpu
@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("C", "C"), ("T", "C")])
def test_uneven_batch_matches_oracle(handle, p, ta, tb):
    rng = np.random.default_rng(7 + ord(p) + 3 * ord(ta) + ord(tb))
    nb = 24
    m = rng.integers(0, 200, nb)
    n = rng.integers(0, 200, nb)
    k = rng.integers(0, 300, nb)
    m[:4], n[:4], k[:4] = [64, 65, 1, 0], [64, 129, 1, 5], [16, 17, 1, 9]
    k[5] = 0
    lda = [max(1, _rows(ta, m[b], k[b])) + int(rng.integers(0, 3)) for b in range(nb)]
    ldb = [max(1, _rows(tb, k[b], n[b])) + int(rng.integers(0, 3)) for b in range(nb)]
    ldc = [max(1, int(m[b])) + int(rng.integers(0, 3)) for b in range(nb)]
    A = [_random(p, rng, lda[b] * max(1, _cols(ta, m[b], k[b]))) for b in range(nb)]
    B = [_random(p, rng, ldb[b] * max(1, _cols(tb, k[b], n[b]))) for b in range(nb)]
    C = [_random(p, rng, ldc[b] * max(1, int(n[b]))) for b in range(nb)]
    A[6], B[7], C[8] = None, None, None  # null entries are skipped
    alpha = DT[p](0.75 - 0.5j) if p in "cz" else DT[p](0.75)
    beta = DT[p](-1.25 + 0.25j) if p in "cz" else DT[p](-1.25)
    hi = np.complex128 if p in "cz" else np.float64
    up = [[None if x is None else x.astype(hi) for x in X] for X in (A, B, C)]
    ab = [[None if x is None else np.abs(x).astype(np.float64) for x in X] for X in (A, B, C)]
    want = restated.gemm_vbatched(ta, tb, m, n, k, hi(alpha), up[0], lda, up[1], ldb, hi(beta), up[2], ldc)
    # forward-error bound of a k-term dot product: gamma_(k+2) (|alpha| |op(A)| |op(B)| + |beta| |C|)
    bound = restated.gemm_vbatched(ta, tb, m, n, k, abs(alpha), ab[0], lda, ab[1], ldb, abs(beta), ab[2], ldc)
    got = _run(handle, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc)
    u = 2.0 ** -24 if p in "sc" else 2.0 ** -53
    for b in range(nb):
        if C[b] is None:
            assert got[b] is None
            continue
        tol = 4 * (int(k[b]) + 2) * u * bound[b] + 1e-30
        err = np.abs(got[b] - want[b])
        assert np.all(err <= tol), (p, ta, tb, b, int(m[b]), int(n[b]), int(k[b]), float(np.max(err - tol)))
        if (A[b] is None or B[b] is None) and int(k[b]) != 0:
            assert got[b].tobytes() == C[b].tobytes()


@pytest.mark.gpu
def test_more_than_65535_entries(handle):
    torch = _torch()
    from libddla_b200.ddla import _c_api as Cc
    nb = 70000
    data = torch.empty(4 * nb, dtype=torch.float64, device="cuda")
    i = torch.arange(nb, device="cuda", dtype=torch.float64)
    data[:nb] = i % 7 + 1
    data[nb:2 * nb] = 2.0
    data[2 * nb:3 * nb] = 1.0
    es = 8
    base = data.data_ptr()
    idx = np.arange(nb, dtype=np.int64)
    pa = torch.from_numpy(base + idx * es).cuda()
    pb = torch.from_numpy(base + (nb + idx) * es).cuda()
    pc = torch.from_numpy(base + (2 * nb + idx) * es).cuda()
    ones = torch.ones(nb, dtype=torch.int32, device="cuda")
    al, be = ctypes.c_double(3.0), ctypes.c_double(0.5)
    torch.cuda.synchronize()
    Cc.check_status(Cc.ddla_d_gemm_vbatched(handle.ptr, b"N", b"N", ones.data_ptr(), ones.data_ptr(), ones.data_ptr(),
                                            ctypes.addressof(al), pa.data_ptr(), ones.data_ptr(), pb.data_ptr(),
                                            ones.data_ptr(), ctypes.addressof(be), pc.data_ptr(), ones.data_ptr(), nb),
                    "gemm_vbatched")
    Cc.check_status(Cc.ddla_c_synchronize(handle.ptr), "sync")
    out = data[2 * nb:3 * nb].cpu().numpy()
    want = 3.0 * 2.0 * (np.arange(nb) % 7 + 1) + 0.5
    assert np.max(np.abs(out - want)) <= 1e-12


@pytest.mark.gpu
def test_argument_errors(handle):
    torch = _torch()
    from libddla_b200.ddla import _c_api as Cc
    f = Cc.ddla_d_gemm_vbatched
    one = ctypes.c_double(1.0)
    a1 = ctypes.addressof(one)
    # an empty batch is a no-op whatever the pointers are
    Cc.check_status(f(handle.ptr, b"N", b"N", None, None, None, a1, None, None, None, None, a1, None, None, 0), "empty")
    # invalid transpose with an empty batch is not looked at (the check comes after the empty-batch return)
    Cc.check_status(f(handle.ptr, b"X", b"N", None, None, None, a1, None, None, None, None, a1, None, None, 0), "empty")
    assert f(None, b"N", b"N", None, None, None, a1, None, None, None, None, a1, None, None, 0) == Cc.STATUS_INVALID_HANDLE
    x = torch.zeros(16, dtype=torch.float64, device="cuda")
    ptrs = torch.tensor([x.data_ptr(), x.data_ptr()], dtype=torch.int64, device="cuda")
    dims = torch.tensor([2, 2], dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    P, D = ptrs.data_ptr(), dims.data_ptr()
    with pytest.raises(Cc.DdlaError, match="gemmVbatched: negative batch count"):
        Cc.check_status(f(handle.ptr, b"N", b"N", D, D, D, a1, P, D, P, D, a1, P, D, -1), "neg")
    with pytest.raises(Cc.DdlaError, match="gemmVbatched: null matrix pointer array"):
        Cc.check_status(f(handle.ptr, b"N", b"N", D, D, D, a1, None, D, P, D, a1, P, D, 2), "null A")
    with pytest.raises(Cc.DdlaError, match="gemmVbatched: null matrix pointer array"):
        Cc.check_status(f(handle.ptr, b"N", b"N", D, D, D, a1, P, D, P, D, a1, None, D, 2), "null C")
    with pytest.raises(Cc.DdlaError, match="gemmVbatched: invalid transpose operation"):
        Cc.check_status(f(handle.ptr, b"N", b"X", D, D, D, a1, P, D, P, D, a1, P, D, 2), "trans")
    with pytest.raises(Cc.DdlaError, match="gemmVbatched: null dimension array"):
        Cc.check_status(f(handle.ptr, b"N", b"N", D, None, D, a1, P, D, P, D, a1, P, D, 2), "null n")
    with pytest.raises(Cc.DdlaError, match="gemmVbatched: null dimension array"):
        Cc.check_status(f(handle.ptr, b"N", b"N", D, D, D, a1, P, D, P, D, a1, P, None, 2), "null ldc")
    # invalid entries found on the device: a negative size, a leading dimension too small
    for bad_m, bad_lda, trans, want in (([2, -1], [2, 2], b"N", 1), ([2, 2], [1, 2], b"N", 0),
                                        ([2, 2], [2, 1], b"T", 1)):
        dm = torch.tensor(bad_m, dtype=torch.int32, device="cuda")
        dl = torch.tensor(bad_lda, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        with pytest.raises(Cc.DdlaError, match=f"gemmVbatched: invalid dimensions at batch {want}$"):
            Cc.check_status(f(handle.ptr, trans, b"N", dm.data_ptr(), D, D, a1, P, dl.data_ptr(), P, D, a1, P, D, 2),
                            "dims")
    # nothing was written by the rejected calls
    assert float(x.abs().sum()) == 0.0
