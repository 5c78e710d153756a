"""pdiag_logdet (the descriptor form of diag_logdet, src/PBLAS/pdiag_logdet.cpp on a
1x1 grid) through the C ABI: the same result as diag_logdet and as the oracle's
DiagLogTerm / DiagLogJoin / finish_diagonal_log restatement, with LLD_ padding and a
leading sub-block; its errors."""
import numpy as np
import pytest

from oracle import restated

pytestmark = pytest.mark.gpu

DT = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}


def _ddla():
    from libddla_b200 import ddla
    return ddla


def _matrix(p, nd, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((nd, nd)) + 2.0 * np.eye(nd)
    if p in "cz":
        A = A + 1j * rng.standard_normal((nd, nd))
    A[np.diag_indices(nd)] *= np.where(np.arange(nd) % 7 == 3, -1.0, 1.0)  # negative entries: phase pi
    return A.astype(DT[p])


@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("n,nd,pad", [(1, 1, 0), (100, 100, 3), (257, 300, 1), (1000, 1000, 0)])
def test_pdiag_logdet_matches_diag_logdet_and_oracle(handle, p, n, nd, pad):
    ddla = _ddla()
    A = _matrix(p, nd, 31 * nd + n)
    M = ddla.DistributedMatrix(handle, nd, nd, mb=64, nb=64, dtype=DT[p], lld=nd + pad)
    host = np.zeros((nd + pad, nd), dtype=DT[p], order="F")
    host[:nd] = A
    M.from_host(host, full_lld=True)
    got = ddla.pdiag_logdet(M, n)
    plain = ddla.diag_logdet(M, n)
    ref = restated.diag_logdet(host, n=n, lda=nd + pad)
    assert got == plain
    tol = 2e-5 if p in "sc" else 3e-12
    assert abs(got.real - ref.real) <= tol * max(1.0, abs(ref.real))
    assert abs(got.imag - ref.imag) <= tol * max(1.0, abs(ref.imag))


def test_pdiag_logdet_errors(handle):
    ddla = _ddla()
    C = ddla._c_api
    M = ddla.DistributedMatrix(handle, 8, 8, mb=4, nb=4, dtype=np.float64)
    host = np.eye(8)
    host[5, 5] = np.nan
    M.from_host(host)
    with pytest.raises(C.DdlaError, match="pdiag_logdet: nonfinite diagonal"):
        ddla.pdiag_logdet(M, 8)
    with pytest.raises(C.DdlaError, match="pdiag_logdet: order exceeds descriptor"):
        ddla.pdiag_logdet(M, 9)
    assert ddla.pdiag_logdet(M, 0) == 0j
    assert ddla.pdiag_logdet(M, 5) == 0j  # log prod(1) = 0 before the NaN
