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


# ---- two stages (gemmVbatched2s) ----------------------------------------------------

def _two_stage_inputs(p, left):
    """The reference test's two-stage case (tests/test_gemm_vbatched.cpp:375-447)."""
    m0, n0, k0 = [2, 3, 2, 5], [3, 2, 4, 2], [4, 2, 3, 2]
    lda0, ldb0, ldc0 = list(m0), list(k0), list(m0)
    A0 = [_matrix(p, lda0[b], k0[b], 71 * b + 1) for b in range(4)]
    B0 = [_matrix(p, ldb0[b], n0[b], 71 * b + 19) for b in range(4)]
    if left:
        m1, n1, k1 = list(m0), [2, 3, 1, 1], list(n0)
    else:
        m1, n1, k1 = [3, 2, 4, 4], list(n0), list(m0)
    lda1, ldb1, ldc1 = list(m1), list(k1), [m + 1 for m in m1]
    AB1 = [_matrix(p, ldb1[b], n1[b], 71 * b + 37) if left else _matrix(p, lda1[b], k1[b], 71 * b + 37)
           for b in range(4)]
    C1 = [_matrix(p, ldc1[b], n1[b], 71 * b + 53) for b in range(4)]
    alphas = (DT[p](_value(p, 17)), DT[p](_value(p, 21)), DT[p](_value(p, 25)))
    offsets = [0, 6, 0, 8]  # the segments {2, 2} reuse one 18-element temporary buffer
    return (m0, n0, k0, lda0, ldb0, ldc0, A0, B0, m1, n1, k1, lda1, ldb1, ldc1, AB1, C1, alphas, offsets)


def _two_stage_loop(p, left, inp):
    m0, n0, k0, lda0, ldb0, ldc0, A0, B0, m1, n1, k1, lda1, ldb1, ldc1, AB1, C1, (a0, a1, b1), _ = inp
    hi = np.complex128 if p in "cz" else np.float64
    cast = complex if p in "cz" else float
    out = []
    for b in range(4):
        tmp = _loop_gemm("N", "N", m0[b], n0[b], k0[b], cast(a0), A0[b].astype(hi), lda0[b], B0[b].astype(hi),
                         ldb0[b], 0.0, np.zeros(ldc0[b] * n0[b], dtype=hi), ldc0[b])
        x, y = (tmp, AB1[b].astype(hi)) if left else (AB1[b].astype(hi), tmp)
        out.append(_loop_gemm("N", "N", m1[b], n1[b], k1[b], cast(a1), x, lda1[b], y, ldb1[b], cast(b1),
                              C1[b].astype(hi), ldc1[b]))
    return out


@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("left", [True, False])
def test_oracle_two_stage_matches_reference_test_loop(p, left):
    inp = _two_stage_inputs(p, left)
    m0, n0, k0, lda0, ldb0, ldc0, A0, B0, m1, n1, k1, lda1, ldb1, ldc1, AB1, C1, (a0, a1, b1), offs = inp
    buf = np.full(18, np.nan, dtype=DT[p])
    got = restated.gemm_vbatched2s("NN", m0, n0, k0, a0, A0, lda0, B0, ldb0, [(buf, o) for o in offs], ldc0,
                                   "NN", m1, n1, k1, a1, AB1, lda1, ldb1, b1, C1, ldc1, left, [2, 2])
    want = _two_stage_loop(p, left, inp)
    for b in range(4):
        g = got[b].reshape(n1[b], ldc1[b]).T[:m1[b]]
        w = want[b].reshape(n1[b], ldc1[b]).T[:m1[b]]
        assert np.max(np.abs(g - w)) <= TOL[p]


@pytest.mark.gpu
@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("left", [True, False])
def test_two_stage_shared_temporaries(handle, p, left):
    torch = _torch()
    from libddla_b200.ddla import batched
    inp = _two_stage_inputs(p, left)
    m0, n0, k0, lda0, ldb0, ldc0, A0, B0, m1, n1, k1, lda1, ldb1, ldc1, AB1, C1, (a0, a1, b1), offs = inp
    tdt = {"s": torch.float32, "d": torch.float64, "c": torch.complex64, "z": torch.complex128}[p]
    temp = torch.full((18,), float("nan"), dtype=tdt, device="cuda")
    es = temp.element_size()
    dC1 = [_dev(c) for c in C1]
    batched.gemm_vbatched2s(handle, "NN", m0, n0, k0, a0, [_dev(a) for a in A0], lda0, [_dev(b) for b in B0], ldb0,
                            [temp.data_ptr() + o * es for o in offs], ldc0, "NN", m1, n1, k1, a1,
                            [_dev(x) for x in AB1], lda1, ldb1, b1, dC1, ldc1, left, [2, 2], tdt)
    want = _two_stage_loop(p, left, inp)
    for b in range(4):
        got = dC1[b].cpu().numpy().reshape(n1[b], ldc1[b]).T
        w = want[b].reshape(n1[b], ldc1[b]).T
        assert np.max(np.abs(got[:m1[b]] - w[:m1[b]])) <= TOL[p], (p, left, b)
        assert got[m1[b]:].tobytes() == C1[b].reshape(n1[b], ldc1[b]).T[m1[b]:].tobytes()


def _two_stage_call(handle, beta0=0.0, segments=(2, 2), batch=4, **over):
    from libddla_b200.ddla import batched
    inp = _two_stage_inputs("d", True)
    m0, n0, k0, lda0, ldb0, ldc0, A0, B0, m1, n1, k1, lda1, ldb1, ldc1, AB1, C1, (a0, a1, b1), offs = inp
    torch = _torch()
    temp = torch.zeros(18, dtype=torch.float64, device="cuda")
    args = dict(ops0="NN", m0=m0, n0=n0, k0=k0, alpha0=a0, A0=[_dev(a) for a in A0], lda0=lda0,
                B0=[_dev(b) for b in B0], ldb0=ldb0, C0=[temp.data_ptr() + o * 8 for o in offs], ldc0=ldc0,
                ops1="NN", m1=m1, n1=n1, k1=k1, alpha1=a1, AB1=[_dev(x) for x in AB1], lda1=lda1, ldb1=ldb1,
                beta1=b1, C1=[_dev(c) for c in C1], ldc1=ldc1, c0_left=True, segments=list(segments),
                dtype=torch.float64, beta0=beta0)
    args.update(over)
    batched.gemm_vbatched2s(handle, **args)


@pytest.mark.gpu
def test_two_stage_argument_errors(handle):
    from libddla_b200.ddla import _c_api as Cc
    for segs in ([0, 4], [-1, 5]):
        with pytest.raises(Cc.DdlaError, match="gemmVbatched2s: segment sizes must be positive"):
            _two_stage_call(handle, segments=segs)
    with pytest.raises(Cc.DdlaError, match="gemmVbatched2s: segment total does not match batch count"):
        _two_stage_call(handle, segments=[1, 1])
    with pytest.raises(Cc.DdlaError, match="gemmVbatched2s: missing segment sizes"):
        _two_stage_call(handle, segments=[])
    with pytest.raises(Cc.DdlaError, match="gemmVbatched2s: stage-zero beta must be zero"):
        _two_stage_call(handle, beta0=1.0)
    with pytest.raises(Cc.DdlaError, match="gemmVbatched: invalid transpose operation"):
        _two_stage_call(handle, ops1="NX")
    with pytest.raises(Cc.DdlaError, match="gemmVbatched: invalid dimensions at batch 2"):
        _two_stage_call(handle, ldc1=[3, 4, 1, 5])
    _two_stage_call(handle)  # the valid call still works after the rejected ones
    # an empty batch is a no-op whatever the pointers are; a null pointer array is rejected
    f = Cc.ddla_d_gemm_vbatched2s
    one = ctypes.c_double(1.0)
    zero = ctypes.c_double(0.0)
    a1, z0 = ctypes.addressof(one), ctypes.addressof(zero)
    nulls = [None] * 3
    Cc.check_status(f(handle.ptr, b"N", b"N", *nulls, a1, None, None, None, None, z0, None, None, b"N", b"N", *nulls,
                      a1, None, None, None, a1, None, None, 0, 0, None, 0), "empty")
    assert f(None, b"N", b"N", *nulls, a1, None, None, None, None, z0, None, None, b"N", b"N", *nulls,
             a1, None, None, None, a1, None, None, 0, 0, None, 0) == Cc.STATUS_INVALID_HANDLE
    seg = (ctypes.c_int * 1)(1)
    with pytest.raises(Cc.DdlaError, match="gemmVbatched2s: null matrix pointer array"):
        Cc.check_status(f(handle.ptr, b"N", b"N", *nulls, a1, None, None, None, None, z0, None, None, b"N", b"N",
                          *nulls, a1, None, None, None, a1, None, None, 0, 1, seg, 1), "null arrays")
    with pytest.raises(Cc.DdlaError, match="gemmVbatched2s: negative batch count"):
        Cc.check_status(f(handle.ptr, b"N", b"N", *nulls, a1, None, None, None, None, z0, None, None, b"N", b"N",
                          *nulls, a1, None, None, None, a1, None, None, 0, -1, seg, 1), "negative")


@pytest.mark.gpu
def test_two_stage_segment_above_grid_limit(handle):
    """One segment of 70000 1x1x1 entries (tests/test_gemm_vbatched.cpp:562-607):
    C1 = alpha1 (A0 B0) AB1 + beta1 C1 with the temporaries on the left."""
    torch = _torch()
    from libddla_b200.ddla import _c_api as Cc
    nb = 70000
    data = torch.empty(5 * nb, dtype=torch.float64, device="cuda")
    i = torch.arange(nb, device="cuda", dtype=torch.float64)
    data[:nb] = i % 7 + 1
    data[nb:2 * nb] = 2.0
    data[2 * nb:3 * nb] = 0.0
    data[3 * nb:4 * nb] = 3.0
    data[4 * nb:] = 1.0
    base = data.data_ptr()
    idx = np.arange(nb, dtype=np.int64)
    ptrs = [torch.from_numpy(base + (s * nb + idx) * 8).cuda() for s in range(5)]
    ones = torch.ones(nb, dtype=torch.int32, device="cuda")
    o = ones.data_ptr()
    one, zero, half = ctypes.c_double(1.0), ctypes.c_double(0.0), ctypes.c_double(0.5)
    seg = (ctypes.c_int * 1)(nb)
    torch.cuda.synchronize()
    Cc.check_status(Cc.ddla_d_gemm_vbatched2s(
        handle.ptr, b"N", b"N", o, o, o, ctypes.addressof(one), ptrs[0].data_ptr(), o, ptrs[1].data_ptr(), o,
        ctypes.addressof(zero), ptrs[2].data_ptr(), o, b"N", b"N", o, o, o, ctypes.addressof(one),
        ptrs[3].data_ptr(), o, o, ctypes.addressof(half), ptrs[4].data_ptr(), o, 1, nb, seg, 1), "2s large")
    Cc.check_status(Cc.ddla_c_synchronize(handle.ptr), "sync")
    out = data[4 * nb:].cpu().numpy()
    want = 6.0 * (np.arange(nb) % 7 + 1) + 0.5
    assert np.max(np.abs(out - want)) <= 1e-12


def test_two_stage_helper_marshalling(monkeypatch):
    """The Python helper hands ddla_?_gemm_vbatched2s its arrays in the C
    signature's order (host tensors and a stub in place of the library call)."""
    torch = _torch()
    from libddla_b200.ddla import _c_api as Cc
    from libddla_b200.ddla import batched
    seen = {}

    def ints(addr, n, kind=ctypes.c_int):
        return list((kind * n).from_address(addr)) if addr else None

    def stub(h, ta0, tb0, m0, n0, k0, al0, A0, lda0, B0, ldb0, be0, C0, ldc0, ta1, tb1, m1, n1, k1, al1, AB1, lda1,
             ldb1, be1, C1, ldc1, left, batch, seg, nseg):
        ll = ctypes.c_longlong
        seen.update(ops=(ta0, tb0, ta1, tb1), dims0=[ints(x, batch) for x in (m0, n0, k0, lda0, ldb0, ldc0)],
                    dims1=[ints(x, batch) for x in (m1, n1, k1, lda1, ldb1, ldc1)],
                    ptrs=[ints(x, batch, ll) for x in (A0, B0, C0, AB1, C1)],
                    scal=[ctypes.c_double.from_address(x).value for x in (al0, be0, al1, be1)],
                    left=left, batch=batch, seg=ints(seg, nseg), nseg=nseg, h=h)
        return 0

    monkeypatch.setattr(Cc, "ddla_d_gemm_vbatched2s", stub)
    monkeypatch.setattr(Cc, "ddla_c_synchronize", lambda h: 0)

    class _H:
        ptr = 77

    mats = [torch.zeros(4, dtype=torch.float64) for _ in range(6)]
    batched.gemm_vbatched2s(_H(), "nT", [1, 2], [3, 4], [5, 6], 1.5, mats[:2], [7, 8], mats[2:4], [9, 10],
                            [1000, 2000], [11, 12], "CN", [13, 14], [15, 16], [17, 18], 2.5, [mats[4], None],
                            [19, 20], [21, 22], -0.5, [None, mats[5]], [23, 24], False, [1, 1], torch.float64)
    assert seen["h"] == 77 and seen["batch"] == 2 and seen["left"] == 0
    assert seen["ops"] == (b"n", b"T", b"C", b"N")
    assert seen["dims0"] == [[1, 2], [3, 4], [5, 6], [7, 8], [9, 10], [11, 12]]
    assert seen["dims1"] == [[13, 14], [15, 16], [17, 18], [19, 20], [21, 22], [23, 24]]
    d = [m.data_ptr() for m in mats]
    assert seen["ptrs"] == [[d[0], d[1]], [d[2], d[3]], [1000, 2000], [d[4], 0], [0, d[5]]]
    assert seen["scal"] == [1.5, 0.0, 2.5, -0.5]
    assert seen["seg"] == [1, 1] and seen["nseg"] == 2


# ---- one real and one complex operand: the oracle ------------------------------------

def _mixed_value(i):
    return ((i % 11) - 5) * 0.0625  # tests/test_gemm_vbatched_mixed.cpp:20-25


def _mixed_loop(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
    """Loop port of the mixed test's oracle (tests/test_gemm_vbatched_mixed.cpp:26-42):
    'C' conjugates an element (a no-op on a real one), beta == 0 does not read C."""
    def at(X, ld, t, i, j):
        z = complex(X[i + j * ld] if t == "N" else X[j + i * ld])
        return z.conjugate() if t == "C" else z

    C = C.astype(np.complex128).copy()
    for j in range(n):
        for i in range(m):
            s = 0j
            if alpha != 0:
                for l in range(k):
                    s += at(A, lda, ta, i, l) * at(B, ldb, tb, l, j)
            z = alpha * s
            if beta != 0:
                z += beta * C[i + j * ldc]
            C[i + j * ldc] = z
    return C


@pytest.mark.parametrize("left", [False, True])
@pytest.mark.parametrize("ta,tb", [(a, b) for a in "NTC" for b in "NTC"])
def test_oracle_mixed_operands_match_reference_test_loop(left, ta, tb):
    m, n, k = [3, 7, 0, 5, 2], [4, 2, 3, 0, 3], [5, 0, 2, 4, 1]
    la = [max(1, m[q] if ta == "N" else k[q]) + 2 for q in range(5)]
    lb = [max(1, k[q] if tb == "N" else n[q]) + 1 for q in range(5)]
    lc = [max(1, m[q]) + 3 for q in range(5)]
    cv = lambda i: complex(_mixed_value(i), _mixed_value(3 * i + 1))
    rv = _mixed_value
    A = [np.array([(cv if left else rv)(p + q) for p in range(la[q] * max(1, k[q] if ta == "N" else m[q]))])
         for q in range(5)]
    B = [np.array([(rv if left else cv)(p + q + 4) for p in range(lb[q] * max(1, n[q] if tb == "N" else k[q]))])
         for q in range(5)]
    C = [np.array([cv(p + q + 2) for p in range(lc[q] * max(1, n[q]))]) for q in range(5)]
    alpha, beta = 0.7 - 0.2j, -0.3 + 0.1j
    got = restated.gemm_vbatched(ta, tb, m, n, k, alpha, A, la, B, lb, beta, C, lc)
    for q in range(5):
        want = _mixed_loop(ta, tb, m[q], n[q], k[q], alpha, A[q], la[q], B[q], lb[q], beta, C[q], lc[q])
        assert np.max(np.abs(got[q] - want)) <= 1e-13
