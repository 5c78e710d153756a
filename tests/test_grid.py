"""The distributed Cholesky path on process grids of several ranks.

Every rank of a P x Q grid is a thread of this process with its own handle
(a local group), all on the one visible GPU: the ranks exchange panels by
device-to-device copies ordered with CUDA events, so no kernel of one rank
ever waits on another's.  Each rank holds only its ScaLAPACK block-cyclic
piece; the pieces are reassembled on the host and compared with the oracle
(the restatement of the reference's CPU arm) on the same matrix:

* ppotrf, both triangles, s/d/c/z, grids 2x1, 1x2, 2x2, 2x3, 3x2, block sizes
  that do and do not divide n, source offsets RSRC/CSRC != 0, and orders
  smaller than one block (the reference's own grid cases, tests/
  test_ppotrf_grids.cpp, at tolerances 3e-12 double / 2e-5 single relative);
* ppotrs / pposv side 'L' with B's columns spread over the process columns;
* a matrix that is not positive definite: every rank returns the same info
  (the order of the failing minor) and B is left unchanged;
* pdiag_logdet summed over the grid.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"s": 2e-5, "c": 2e-5, "d": 3e-12, "z": 3e-12}
DT = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}


def _spd(n, p, seed):
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((n, n))
    if p in "cz":
        G = G + 1j * rng.standard_normal((n, n))
    A = G @ G.conj().T / max(1, n) + np.eye(n)
    return A.astype(DT[p])


def _run_grid(P, Q, fn, major="R"):
    from libddla_b200 import ddla
    from libddla_b200.ddla import grid

    group = grid.LocalGroup(P * Q, timeout_s=60.0)

    def body(rank):
        h = ddla.Handle(ddla.Backend.GPU, local_group=group, rank=rank, nprows=P, npcols=Q, major=major)
        try:
            return fn(h, rank)
        finally:
            h.destroy()

    try:
        return grid.run_ranks(P * Q, body)
    finally:
        group.close()


def _factor_on_grid(A, p, uplo, P, Q, nb, rsrc=0, csrc=0, major="R"):
    from libddla_b200 import ddla
    from libddla_b200.ddla import grid

    n = A.shape[0]

    def fn(h, rank):
        row, col = grid.rank_to_rc(rank, P, Q, major)
        assert h.grid_coords == (row, col) and h.grid_dims == (P, Q)
        M = ddla.DistributedMatrix(h, n, n, mb=nb, nb=nb, dtype=DT[p], irsrc=rsrc, icsrc=csrc)
        M.from_host(grid.local_piece(A, nb, nb, P, Q, row, col, rsrc, csrc))
        _, info = ddla.ppotrf(M, uplo)
        return info, M.to_host()

    res = _run_grid(P, Q, fn, major)
    infos = {r[0] for r in res}
    assert len(infos) == 1, infos
    F = grid.assemble([r[1] for r in res], n, n, nb, nb, P, Q, rsrc, csrc, major)
    return infos.pop(), F


GRIDS = [(2, 1), (1, 2), (2, 2), (2, 3), (3, 2)]


@pytest.mark.parametrize("P,Q", GRIDS)
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("p", ["d", "z", "s", "c"])
def test_ppotrf_grid_matches_oracle(P, Q, uplo, p):
    from oracle import restated

    n, nb = 97, 16
    A = _spd(n, p, 10 + P * 7 + Q)
    info, F = _factor_on_grid(A, p, uplo, P, Q, nb)
    ref, rinfo = restated.potrf(A, uplo)
    assert info == rinfo == 0
    tri = np.tril if uplo == "L" else np.triu
    err = np.max(np.abs(tri(F) - tri(ref))) / np.max(np.abs(tri(ref)))
    assert err <= TOL[p], err
    # the other triangle is not touched
    other = np.triu if uplo == "L" else np.tril
    assert np.array_equal(other(F, 1 if uplo == "L" else -1), other(A, 1 if uplo == "L" else -1))


@pytest.mark.parametrize("n,nb,rsrc,csrc,major", [(130, 32, 1, 0, "R"), (64, 32, 0, 1, "C"), (5, 8, 1, 1, "R"),
                                                   (1, 4, 0, 0, "C"), (200, 24, 1, 2, "R")])
def test_ppotrf_grid_offsets_and_small_orders(n, nb, rsrc, csrc, major):
    from oracle import restated

    P, Q = 2, 3
    A = _spd(n, "d", n + nb)
    for uplo in "LU":
        info, F = _factor_on_grid(A, "d", uplo, P, Q, nb, rsrc, csrc, major)
        ref, _ = restated.potrf(A, uplo)
        tri = np.tril if uplo == "L" else np.triu
        assert info == 0
        assert np.max(np.abs(tri(F) - tri(ref))) <= 3e-12 * np.max(np.abs(ref))


def _solve_on_grid(A, Bm, p, uplo, P, Q, nb, nbb, do_factor=True, rsrc=0, csrc=0):
    from libddla_b200 import ddla
    from libddla_b200.ddla import grid

    n, nrhs = Bm.shape

    def fn(h, rank):
        row, col = grid.rank_to_rc(rank, P, Q)
        M = ddla.DistributedMatrix(h, n, n, mb=nb, nb=nb, dtype=DT[p], irsrc=rsrc, icsrc=csrc)
        M.from_host(grid.local_piece(A, nb, nb, P, Q, row, col, rsrc, csrc))
        Bd = ddla.DistributedMatrix(h, n, nrhs, mb=nb, nb=nbb, dtype=DT[p], irsrc=rsrc, icsrc=0)
        Bd.from_host(grid.local_piece(Bm, nb, nbb, P, Q, row, col, rsrc, 0))
        if do_factor:
            _, info = ddla.pposv(M, Bd, uplo)
        else:
            info = 0
            ddla.ppotrs(M, Bd, uplo)
        return info, Bd.to_host()

    res = _run_grid(P, Q, fn)
    infos = {r[0] for r in res}
    assert len(infos) == 1, infos
    X = grid.assemble([r[1] for r in res], n, nrhs, nb, nbb, P, Q, rsrc, 0)
    return infos.pop(), X


@pytest.mark.parametrize("P,Q", GRIDS)
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("p", ["d", "z", "s"])
def test_pposv_grid_matches_oracle(P, Q, uplo, p):
    from oracle import restated

    n, nb, nrhs = 90, 16, 7
    A = _spd(n, p, 3 + P + 5 * Q)
    rng = np.random.default_rng(9)
    Bm = rng.standard_normal((n, nrhs)).astype(DT[p])
    if p in "cz":
        Bm = (Bm + 1j * rng.standard_normal((n, nrhs))).astype(DT[p])
    info, X = _solve_on_grid(A, Bm, p, uplo, P, Q, nb, nbb=3)
    _, Xref, rinfo = restated.pposv(A, Bm, uplo)
    assert info == rinfo == 0
    err = np.max(np.abs(X - Xref)) / np.max(np.abs(Xref))
    assert err <= 50 * TOL[p], err


def test_ppotrs_grid_with_factor_from_grid():
    """ppotrs alone on a factor the grid produced; B with one column block per process column."""
    from libddla_b200 import ddla
    from libddla_b200.ddla import grid
    from oracle import restated

    P, Q, n, nb, nrhs = 2, 2, 150, 32, 20
    A = _spd(n, "d", 77)
    Bm = np.random.default_rng(4).standard_normal((n, nrhs))
    for uplo in "LU":
        def fn(h, rank):
            row, col = grid.rank_to_rc(rank, P, Q)
            M = ddla.DistributedMatrix(h, n, n, mb=nb, nb=nb, dtype=np.float64)
            M.from_host(grid.local_piece(A, nb, nb, P, Q, row, col))
            _, info = ddla.ppotrf(M, uplo)
            Bd = ddla.DistributedMatrix(h, n, nrhs, mb=nb, nb=8, dtype=np.float64)
            Bd.from_host(grid.local_piece(Bm, nb, 8, P, Q, row, col))
            ddla.ppotrs(M, Bd, uplo)
            return info, Bd.to_host()

        res = _run_grid(P, Q, fn)
        assert {r[0] for r in res} == {0}
        X = grid.assemble([r[1] for r in res], n, nrhs, nb, 8, P, Q)
        ref = restated.ppotrs(restated.potrf(A, uplo)[0], Bm, uplo)
        assert np.max(np.abs(X - ref)) <= 1e-11 * np.max(np.abs(ref))
        assert np.max(np.abs(A @ X - Bm)) <= 1e-10 * np.max(np.abs(Bm))


@pytest.mark.parametrize("P,Q", [(2, 2), (1, 3)])
def test_not_positive_definite_on_grid(P, Q):
    """Every rank reports the order of the first failing minor; pposv leaves B unchanged."""
    n, nb = 70, 16
    A = _spd(n, "d", 5)
    A[40, 40] = -1.0  # the leading minor of order 41 is the first that fails
    from oracle import restated

    _, rinfo = restated.potrf(A, "L")
    Bm = np.random.default_rng(2).standard_normal((n, 3))
    info, X = _solve_on_grid(A, Bm, "d", "L", P, Q, nb, nbb=2)
    assert info == rinfo == 41
    assert np.array_equal(X, Bm)


@pytest.mark.parametrize("p", ["d", "z"])
def test_pdiag_logdet_summed_over_grid(p):
    from libddla_b200 import ddla
    from libddla_b200.ddla import grid

    P, Q, n, nb = 2, 3, 101, 8
    A = _spd(n, p, 12)
    d = np.diag(A).copy()
    d[::7] *= -1  # negative real entries: the parity term
    np.fill_diagonal(A, d)

    def fn(h, rank):
        row, col = grid.rank_to_rc(rank, P, Q)
        M = ddla.DistributedMatrix(h, n, n, mb=nb, nb=nb, dtype=DT[p])
        M.from_host(grid.local_piece(A, nb, nb, P, Q, row, col))
        return ddla.pdiag_logdet(M)

    vals = _run_grid(P, Q, fn)
    ref = np.sum(np.log(np.abs(d)))
    phase = np.angle(np.prod(d / np.abs(d)))
    for v in vals:
        assert abs(v.real - ref) <= 1e-12 * abs(ref)
        assert abs(np.angle(np.exp(1j * (v.imag - phase)))) <= 1e-12
