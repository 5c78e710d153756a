"""The mixed batched GEMM (one real and one complex operand, complex output;
ddla_{c,z}_gemm_vbatched_{rc,cr}) on the reference test's one-stage cases
(tests/test_gemm_vbatched_mixed.cpp:63-118, 200-222): the nine transpose pairs
for both operand orders and both precisions, the zero-alpha / zero-beta cases
(NaN in C when beta is 0), its tolerances (1e-5 / 1e-12 relative to 1 + |ref|),
a bad leading dimension and a null operand rejected before anything is written,
and the no-op calls that must not touch null entries."""
import numpy as np
import pytest

from oracle import restated

pytestmark = pytest.mark.gpu

RT = {"f": np.float32, "d": np.float64}
ZT = {"f": np.complex64, "d": np.complex128}
TOL = {"f": 1e-5, "d": 1e-12}


def _value(i):
    return ((i % 11) - 5) * 0.0625


def _sample(cplx, i):
    return complex(_value(i), _value(3 * i + 1)) if cplx else _value(i)


def _vec(size, cplx, dt, off):
    return np.array([_sample(cplx, p + off) for p in range(size)], dtype=dt)


def _dev(x):
    import torch
    return None if x is None else torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _case(r, left, ta, tb, zero_alpha, zero_beta):
    m, n, k = [3, 7, 0, 5, 2], [4, 2, 3, 0, 3], [5, 0, 2, 4, 1]
    adt = ZT[r] if left else RT[r]
    bdt = RT[r] if left else ZT[r]
    la = [max(1, m[q] if ta == "N" else k[q]) + 2 for q in range(5)]
    lb = [max(1, k[q] if tb == "N" else n[q]) + 1 for q in range(5)]
    lc = [max(1, m[q]) + 3 for q in range(5)]
    A = [_vec(la[q] * max(1, k[q] if ta == "N" else m[q]), left, adt, q) for q in range(5)]
    B = [_vec(lb[q] * max(1, n[q] if tb == "N" else k[q]), not left, bdt, q + 4) for q in range(5)]
    C = [_vec(lc[q] * max(1, n[q]), True, ZT[r], q + 2) for q in range(5)]
    alpha = ZT[r](0) if zero_alpha else ZT[r](0.7 - 0.2j)
    beta = ZT[r](0) if zero_beta else ZT[r](-0.3 + 0.1j)
    if zero_beta:
        for q in range(5):
            C[q].reshape(max(1, n[q]), lc[q]).T[:m[q], :n[q]] = complex(np.nan, 0)
    Ap = [None if (zero_alpha or k[q] == 0) else A[q] for q in range(5)]
    Bp = [None if (zero_alpha or k[q] == 0) else B[q] for q in range(5)]
    return m, n, k, la, lb, lc, A, B, C, Ap, Bp, alpha, beta


@pytest.mark.parametrize("r", ["f", "d"])
@pytest.mark.parametrize("left", [False, True])
@pytest.mark.parametrize("ta,tb,zero_alpha,zero_beta",
                         [(a, b, False, False) for a in "NTC" for b in "NTC"] +
                         [("C", "C", True, True), ("N", "N", False, True)])
def test_mixed_one_stage(handle, r, left, ta, tb, zero_alpha, zero_beta):
    from libddla_b200.ddla import _c_api as C_
    from libddla_b200.ddla import batched
    m, n, k, la, lb, lc, A, B, C, Ap, Bp, alpha, beta = _case(r, left, ta, tb, zero_alpha, zero_beta)
    hi = [None if x is None else x.astype(np.complex128) for x in Ap], [None if x is None else x.astype(np.complex128)
                                                                          for x in Bp]
    want = restated.gemm_vbatched(ta, tb, m, n, k, complex(alpha), hi[0], la, hi[1], lb, complex(beta),
                                  [c.astype(np.complex128) for c in C], lc)
    dA, dB, dC = [_dev(x) for x in Ap], [_dev(x) for x in Bp], [_dev(c) for c in C]
    # the operand types must be visible to the helper even where every entry is null
    if all(x is None for x in dA):
        dA[0] = _dev(A[0])  # alpha == 0 reads no operand; a present entry is ignored
    if all(x is None for x in dB):
        dB[0] = _dev(B[0])
    batched.gemm_vbatched(handle, ta, tb, m, n, k, alpha, dA, la, dB, lb, beta, dC, lc)
    got = [t.cpu().numpy() for t in dC]
    for q in range(5):
        assert np.all(np.isfinite(got[q])), (q, got[q])
        err = np.abs(got[q].astype(np.complex128) - want[q]) / (1 + np.abs(want[q]))
        assert float(err.max()) <= TOL[r], (r, left, ta, tb, q, float(err.max()))
    # a bad leading dimension in the last entry is rejected before any matrix is written
    bad = list(la)
    bad[-1] = 0
    with pytest.raises(C_.DdlaError, match="gemmVbatched: invalid dimensions at batch 4"):
        batched.gemm_vbatched(handle, ta, tb, m, n, k, alpha, dA, bad, dB, lb, beta, dC, lc)
    assert all(np.array_equal(t.cpu().numpy(), g, equal_nan=True) for t, g in zip(dC, got))
    if not zero_alpha:
        nullA = list(dA)
        nullA[-1] = None
        with pytest.raises(C_.DdlaError, match=r"gemmVbatched\(mixed\): null matrix at batch 4"):
            batched.gemm_vbatched(handle, ta, tb, m, n, k, alpha, nullA, la, dB, lb, beta, dC, lc)
        assert all(np.array_equal(t.cpu().numpy(), g, equal_nan=True) for t, g in zip(dC, got))


@pytest.mark.parametrize("r", ["f", "d"])
def test_mixed_noops_and_errors(handle, r):
    import torch

    from libddla_b200.ddla import _c_api as C_
    p = "c" if r == "f" else "z"
    f = getattr(C_, f"ddla_{p}_gemm_vbatched_rc")
    one = np.array([1.0], dtype=ZT[r])
    zero = np.array([0.0], dtype=ZT[r])
    a1, a0 = one.ctypes.data, zero.ctypes.data
    # an empty batch touches nothing, whatever the pointers are
    C_.check_status(f(handle.ptr, b"N", b"N", None, None, None, a1, None, None, None, None, a0, None, None, 0), "empty")
    # m = n = 2, k = 0, beta = 1: nothing to do, the null entries are not looked at
    dims = torch.tensor([2], dtype=torch.int32, device="cuda")
    zk = torch.tensor([0], dtype=torch.int32, device="cuda")
    nul = torch.zeros(1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    D, Z0, N0 = dims.data_ptr(), zk.data_ptr(), nul.data_ptr()
    C_.check_status(f(handle.ptr, b"N", b"C", D, D, Z0, a1, N0, D, N0, D, a1, N0, D, 1), "no-op")
    with pytest.raises(C_.DdlaError, match=r"gemm\(real,complex\): invalid transpose flag"):
        C_.check_status(f(handle.ptr, b"N", b"X", D, D, Z0, a1, N0, D, N0, D, a1, N0, D, 1), "trans")
    with pytest.raises(C_.DdlaError, match=r"gemmVbatched\(mixed\): negative batch count"):
        C_.check_status(f(handle.ptr, b"N", b"N", D, D, Z0, a1, N0, D, N0, D, a1, N0, D, -1), "negative")
    with pytest.raises(C_.DdlaError, match=r"gemmVbatched\(mixed\): null metadata array"):
        C_.check_status(f(handle.ptr, b"N", b"N", D, None, Z0, a1, N0, D, N0, D, a1, N0, D, 1), "metadata")
    # beta != 1 with a null C must write C: rejected
    with pytest.raises(C_.DdlaError, match=r"gemmVbatched\(mixed\): null matrix at batch 0"):
        C_.check_status(f(handle.ptr, b"N", b"N", D, D, Z0, a1, N0, D, N0, D, a0, N0, D, 1), "null C")


# ---- two stages (tests/test_gemm_vbatched_mixed.cpp:110-198) --------------------------

PATTERNS = {0: "rzzr", 1: "zrzr", 2: "rzzz", 3: "zrzz", 4: "zzzr", 5: "rrrz"}  # (A0, B0, C0, AB1)


def _loop(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
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


@pytest.mark.parametrize("r", ["f", "d"])
@pytest.mark.parametrize("pattern", sorted(PATTERNS))
@pytest.mark.parametrize("left", [False, True])
def test_mixed_two_stage(handle, r, pattern, left):
    import torch

    from libddla_b200.ddla import _c_api as C_
    from libddla_b200.ddla import batched
    code = PATTERNS[pattern]
    cz = {c: c == "z" for c in "rz"}
    dt = lambda c: ZT[r] if c == "z" else RT[r]
    m0, n0, k0, outer = [2, 4, 2, 4, 0], [3, 2, 3, 2, 0], [5, 3, 5, 3, 0], [4, 5, 4, 5, 0]
    la0 = [max(1, x) + 2 for x in k0]
    lb0 = [max(1, x) + 3 for x in n0]
    lc0 = [max(1, x) + 4 for x in m0]
    m1 = [n0[q] if left else outer[q] for q in range(5)]
    n1 = [outer[q] if left else m0[q] for q in range(5)]
    k1 = [m0[q] if left else n0[q] for q in range(5)]
    ext_ld = [max(1, k1[q] if left else m1[q]) + 2 for q in range(5)]
    la1 = [lc0[q] if left else ext_ld[q] for q in range(5)]
    lb1 = [ext_ld[q] if left else lc0[q] for q in range(5)]
    lc1 = [max(1, x) + 3 for x in m1]
    a = [_vec(la0[q] * max(1, m0[q]), cz[code[0]], dt(code[0]), q) for q in range(5)]
    b = [_vec(lb0[q] * max(1, k0[q]), cz[code[1]], dt(code[1]), 2 * q + 1) for q in range(5)]
    ext = [_vec(ext_ld[q] * max(1, n1[q] if left else k1[q]), cz[code[3]], dt(code[3]), 3 * q) for q in range(5)]
    out = [_vec(lc1[q] * max(1, n1[q]), True, ZT[r], 1) for q in range(5)]
    a0 = dt(code[2])(_sample(cz[code[2]], 17))
    a1, beta = ZT[r](0.6 + 0.2j), ZT[r](-0.2 + 0.1j)
    ops1 = ("C", "N") if left else ("N", "C")
    ref = []
    for q in range(5):
        tmp = _loop("C", "T", m0[q], n0[q], k0[q], complex(a0), a[q], la0[q], b[q], lb0[q], 0,
                    np.zeros(lc0[q] * max(1, n0[q])), lc0[q])
        x, y = (tmp, ext[q]) if left else (ext[q], tmp)
        ref.append(_loop(ops1[0], ops1[1], m1[q], n1[q], k1[q], complex(a1), x, la1[q], y, lb1[q], complex(beta),
                         out[q], lc1[q]))
    init_tmp = []
    for q in range(2):  # entries q, q+2, q+4 share temporary q
        t = _vec(lc0[q] * max(1, n0[q]), cz[code[2]], dt(code[2]), 61)
        t.reshape(max(1, n0[q]), lc0[q]).T[:m0[q], :n0[q]] = np.nan
        init_tmp.append(t)
    dtmp = [_dev(t) for t in init_tmp]
    dA, dB, dE, dC = [_dev(x) for x in a], [_dev(x) for x in b], [_dev(x) for x in ext], [_dev(x) for x in out]
    c0 = [dtmp[q % 2].data_ptr() for q in range(5)]
    tdt = {"f": torch.complex64, "d": torch.complex128}[r]

    def call(beta0=0, segs=(2, 3), m_1=m1, n_1=n1, k_1=k1, la_1=la1, lb_1=lb1):
        batched.gemm_vbatched2s(handle, "CT", m0, n0, k0, a0, dA, la0, dB, lb0, c0, lc0, "".join(ops1), m_1, n_1,
                                k_1, a1, dE, la_1, lb_1, beta, dC, lc1, left, list(segs), tdt, beta0=beta0,
                                pattern=code)

    def unchanged():
        assert all(t.cpu().numpy().tobytes() == o.tobytes() for t, o in zip(dC, out))
        assert all(t.cpu().numpy().tobytes() == o.tobytes() for t, o in zip(dtmp, init_tmp))

    dec = lambda v, i: [x - (1 if j == i else 0) for j, x in enumerate(v)]
    cases = [(dict(segs=(1, 2)), "gemmVbatched2s\\(mixed\\): segment total mismatch"),
             (dict(beta0=1), "gemmVbatched2s\\(mixed\\): stage-zero beta must be zero"),
             (dict(k_1=dec(k1, 3)) if left else dict(n_1=dec(n1, 3)), "incompatible intermediate dimensions"),
             (dict(m_1=dec(m1, 3)) if left else dict(k_1=dec(k1, 3)), "incompatible intermediate dimensions"),
             (dict(la_1=dec(la1, 3)) if left else dict(lb_1=dec(lb1, 3)), "incompatible intermediate dimensions")]
    for kw, msg in cases:
        with pytest.raises(C_.DdlaError, match=msg):
            call(**kw)
        unchanged()
    call()
    for q in range(5):
        got = dC[q].cpu().numpy().astype(np.complex128)
        err = np.abs(got - ref[q]) / (1 + np.abs(ref[q]))
        assert np.all(np.isfinite(got)) and float(err.max()) <= TOL[r], (r, code, left, q, float(err.max()))
