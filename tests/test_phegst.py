"""phegst through the C ABI (ddla_?_phegst): the type-1 reduction A <- L^-1 A L^-H
with a caller's factor, on the reference test's analytic pair
(tests/test_phegst.cpp:53-155: B = L L^H with L bidiagonal, A = L S L^H, so the
result is S; a second pass reduces 1.25 A + 0.37 B to 1.25 S + 0.37 I) with the
descriptors padded as there, the unread triangles and A's imaginary diagonal set
to NaN, the factor and everything past n checked bit for bit; against the
oracle's phegst on random pairs at orders crossing the 64-row blocks of the
solve; and the reference's argument errors."""
import numpy as np
import pytest

from oracle import restated
from test_phegst_oracle import DT, _pair

pytestmark = pytest.mark.gpu


def _ddla():
    from libddla_b200 import ddla
    return ddla


def _upload(handle, host, rows, cols, block):
    ddla = _ddla()
    M = ddla.DistributedMatrix(handle, rows, cols, mb=block, nb=block, dtype=host.dtype, lld=host.shape[0])
    M.from_host(host, full_lld=True)
    return M


def _inputs(p, uplo, n, src, factor_host, pad_a=3, pad_f=2):
    other = np.triu_indices(n, 1) if uplo == "L" else np.tril_indices(n, -1)
    Ah = np.full((n + 2 + pad_a, n + 3), 8157.0, dtype=DT[p], order="F")
    Ah[:n, :n] = src.astype(DT[p])
    Ah[other] = np.nan
    if p in "cz" and n:
        Ah.imag[np.diag_indices(n)] = np.nan
    Fh = np.full((n + 3 + pad_f, n + 2), 8157.0, dtype=DT[p], order="F")
    Fh[:n, :n] = factor_host.astype(DT[p])
    Fh[other] = np.nan
    return Ah, Fh


@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("n,block", [(1, 4), (17, 4), (17, 17), (17, 64), (64, 64), (200, 64)])
def test_phegst_analytic_pair(handle, p, uplo, n, block):
    ddla = _ddla()
    A, B, S = _pair(p, n)
    L = np.linalg.cholesky(B)
    factor = L if uplo == "L" else np.conj(L).T
    eps = np.finfo(DT[p]).eps
    for rep in range(2):
        want = S if rep == 0 else 1.25 * S + 0.37 * np.eye(n)
        src = A if rep == 0 else 1.25 * A + 0.37 * B
        Ah, Fh = _inputs(p, uplo, n, src, factor)
        dA = _upload(handle, Ah, n + 2, n + 3, block)
        dF = _upload(handle, Fh, n + 3, n + 2, block)
        ddla.phegst(dA, dF, uplo, n)
        got = dA.to_host(full_lld=True)
        g = got[:n, :n]
        err = np.abs(g - want) / np.maximum(np.abs(want), 1.0)
        assert float(err.max()) / (eps * n) <= 400, (p, uplo, n, block, rep, float(err.max()) / (eps * n))
        if p in "cz":
            assert np.all(np.imag(np.diag(g)) == 0)
        assert np.array_equal(g, np.conj(g).T)
        mask = np.ones(got.shape, dtype=bool)
        mask[:n, :n] = False
        assert got[mask].tobytes() == Ah[mask].tobytes()
        assert dF.to_host(full_lld=True).tobytes(order="F") == Fh.tobytes(order="F")


@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("n", [63, 64, 65, 130, 1100])
def test_phegst_matches_oracle(handle, p, uplo, n):
    ddla = _ddla()
    rng = np.random.default_rng(n + ord(p) + ord(uplo))
    G = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if p in "cz" else 0)
    B = G @ np.conj(G).T / n + np.eye(n)
    H = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if p in "cz" else 0)
    A = (H + np.conj(H).T) / 2
    L = np.linalg.cholesky(B)
    factor = L if uplo == "L" else np.conj(L).T
    Ah, Fh = _inputs(p, uplo, n, A, factor)
    want = restated.phegst(Ah, Fh, uplo, n)[:n, :n]
    dA = _upload(handle, Ah, n + 2, n + 3, 64)
    dF = _upload(handle, Fh, n + 3, n + 2, 64)
    ddla.phegst(dA, dF, uplo, n)
    got = dA.to_host(full_lld=True)[:n, :n]
    eps = np.finfo(DT[p]).eps
    rel = float(np.abs(got - want).max() / np.abs(want).max())
    assert rel <= 50 * eps * np.sqrt(n), (p, uplo, n, rel)


def test_phegst_argument_errors(handle):
    ddla = _ddla()
    C = ddla._c_api
    n = 20
    A, B, _ = _pair("d", n)
    L = np.linalg.cholesky(B)
    Ah, Fh = _inputs("d", "L", n, A, L)
    dA = _upload(handle, Ah, n + 2, n + 3, 8)
    dF = _upload(handle, Fh, n + 3, n + 2, 8)
    dF_other = _upload(handle, Fh, n + 3, n + 2, 4)
    before = dA.to_host(full_lld=True).tobytes(order="F")
    with pytest.raises(C.DdlaError, match="phegst: invalid order or triangle"):
        ddla.phegst(dA, dF, "X", n)
    with pytest.raises(C.DdlaError, match="phegst: invalid order or triangle"):
        C.check_status(C.lib.ddla_d_phegst(handle.ptr, b"L", -1, dA.data_ptr, dA.desc.ctypes.data, dF.data_ptr,
                                           dF.desc.ctypes.data), "negative order")
    with pytest.raises(C.DdlaError, match="phegst: matching square source-zero descriptors required"):
        ddla.phegst(dA, dF, "L", n + 3)
    with pytest.raises(C.DdlaError, match="phegst: matching square source-zero descriptors required"):
        ddla.phegst(dA, dF_other, "L", n)
    with pytest.raises(C.DdlaError, match="phegst: A and factor must be disjoint"):
        ddla.phegst(dA, dA, "L", n)
    assert dA.to_host(full_lld=True).tobytes(order="F") == before  # rejected calls change nothing
    ddla.phegst(dA, dF, "l", 0)  # n = 0 touches nothing
    assert dA.to_host(full_lld=True).tobytes(order="F") == before
