"""pdiag_logdet on a process grid: each rank reduces the diagonal entries its
block-cyclic local matrix holds, the ranks sum five doubles (the reference's one
MPI_Allreduce, src/PBLAS/pdiag_logdet.cpp:41-47), and the finish gives log det.

CPU: the oracle's grid-local states on every rank of several grids sum to the
1x1 answer; two gloo ranks (a 2x1 grid) run pdiag_logdet_grid with the oracle's
local states, one all-reduce, and the library's native finish, and both get the
oracle's answer; a nonfinite entry on one rank raises on both.
GPU: the library's grid-local kernel (ddla_?_pdiag_logdet_local) on every rank's
local piece of 2x1, 1x2, 2x2 and 3x2 grids, summed and finished, against the
oracle and against the 1x1 pdiag_logdet of the whole matrix.
"""
import math
import os

import numpy as np
import pytest

from oracle import restated

GRIDS = [(1, 1), (2, 1), (1, 2), (2, 2), (3, 2), (2, 3)]


def _matrix(p, n, seed, neg=0):
    rng = np.random.default_rng(seed)
    d = rng.uniform(0.5, 2.0, n) * rng.choice([-1, 1], n) if neg else rng.uniform(0.5, 2.0, n)
    if p in "cz":
        d = d * np.exp(1j * rng.uniform(-1, 1, n))
    A = rng.standard_normal((n, n)) * 0.01
    if p in "cz":
        A = A + 1j * rng.standard_normal((n, n)) * 0.01
    A[np.arange(n), np.arange(n)] = d
    return A.astype({"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}[p])


def _finish_oracle(total):
    if total[4]:
        raise ValueError("nonfinite")
    if total[2]:
        return complex(-math.inf, 0)
    ph = math.remainder(total[1] + (int(total[3]) & 1) * math.pi, 2 * math.pi)
    return complex(total[0], math.pi if ph <= -math.pi else ph)


@pytest.mark.parametrize("p", ["d", "z"])
@pytest.mark.parametrize("grid", GRIDS)
def test_oracle_grid_states_sum_to_whole(p, grid):
    pr, pc = grid
    n, mb, nb = 37, 4, 3
    A = _matrix(p, n, 5, neg=1)
    total = np.zeros(5)
    for row in range(pr):
        for col in range(pc):
            loc = restated.block_cyclic_local(A, mb, nb, pr, pc, row, col, rsrc=pr - 1, csrc=0)
            total += restated.diag_log_local_state(loc, n, mb, nb, pr, pc, row, col, rsrc=pr - 1, csrc=0)
    got = _finish_oracle(total)
    want = restated.diag_logdet(A)
    assert abs(got.real - want.real) <= 1e-12 * max(1.0, abs(want.real))
    assert abs(math.remainder(got.imag - want.imag, 2 * math.pi)) <= 1e-12


def test_native_finish_matches_reference_rules():
    from libddla_b200 import ddla

    assert ddla.pdiag_logdet_finish([1.5, 0.25, 0, 0, 0]) == complex(1.5, 0.25)
    r = ddla.pdiag_logdet_finish([2.0, 0.0, 0, 3, 0])  # odd negative parity: phase pi
    assert r.real == 2.0 and abs(r.imag - math.pi) < 1e-15
    r = ddla.pdiag_logdet_finish([2.0, 3 * math.pi, 0, 0, 0])  # wrapped to (-pi, pi]
    assert abs(r.imag - math.pi) < 1e-12
    assert ddla.pdiag_logdet_finish([7.0, 1.0, 2, 1, 0]) == complex(-math.inf, 0)
    with pytest.raises(ddla.DdlaError, match="nonfinite"):
        ddla.pdiag_logdet_finish([0, 0, 0, 0, 1])
    r = ddla.pdiag_logdet_finish([1.25, 0.5, 0, 0, 0], single=True)
    assert r == complex(np.float32(1.25), np.float32(0.5))


def _gloo_worker(rank, world, port, p, poison, out):
    import torch.distributed as dist

    from libddla_b200 import ddla

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n, mb, nb, pr, pc = 29, 4, 4, 2, 1
        A = _matrix(p, n, 8, neg=1)
        if poison:
            A[0, 0] = np.nan  # held by rank 0 only
        loc = restated.block_cyclic_local(A, mb, nb, pr, pc, rank, 0)
        state = restated.diag_log_local_state(loc, n, mb, nb, pr, pc, rank, 0)
        try:
            r = ddla.pdiag_logdet_grid(None, p, n, 0, None, (pr, pc, rank, 0), local_state=state)
            out.put((rank, "ok", r))
        except ddla.DdlaError as exc:
            out.put((rank, "raised", str(exc)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("poison", [False, True])
def test_pdiag_logdet_grid_over_two_gloo_ranks(poison):
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, "z", poison, q)) for r in range(2)]
    for pr_ in procs:
        pr_.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for pr_ in procs:
        pr_.join(timeout=60)
        assert pr_.exitcode == 0
    if poison:
        assert [r[1] for r in results] == ["raised", "raised"]  # every rank raises together
        assert all("nonfinite" in r[2] for r in results)
        return
    want = restated.diag_logdet(_matrix("z", 29, 8, neg=1))
    for _, kind, r in results:
        assert kind == "ok"
        assert abs(r.real - want.real) <= 1e-12 * max(1.0, abs(want.real))
        assert abs(math.remainder(r.imag - want.imag, 2 * math.pi)) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("p", ["s", "d", "c", "z"])
@pytest.mark.parametrize("grid", [(2, 1), (1, 2), (2, 2), (3, 2)])
def test_grid_local_kernel_emulating_every_rank(handle, p, grid):
    from libddla_b200 import ddla

    pr, pc = grid
    n, mb, nb = 1000, 64, 32
    A = _matrix(p, n, 12, neg=1)
    tol = 2e-5 if p in "sc" else 1e-11
    total = np.zeros(5)
    for row in range(pr):
        for col in range(pc):
            loc = restated.block_cyclic_local(A, mb, nb, pr, pc, row, col, rsrc=0, csrc=pc - 1)
            lld = max(1, loc.shape[0]) + 3  # padded local leading dimension
            dL = ddla.DistributedMatrix(handle, lld, max(1, loc.shape[1]), mb=lld, nb=max(1, loc.shape[1]),
                                        dtype=A.dtype)
            buf = np.zeros((lld, max(1, loc.shape[1])), dtype=A.dtype, order="F")
            buf[:loc.shape[0], :loc.shape[1]] = loc
            dL.from_host(buf)
            desc = np.zeros(9, dtype=np.int32)
            desc[:] = [1, 0, n, n, mb, nb, 0, pc - 1, lld]
            st = ddla.pdiag_logdet_local(handle, p, n, dL.data_ptr, desc, (pr, pc, row, col))
            so = restated.diag_log_local_state(loc, n, mb, nb, pr, pc, row, col, rsrc=0, csrc=pc - 1)
            np.testing.assert_array_equal(st[2:], so[2:])
            assert abs(st[0] - so[0]) <= tol * max(1.0, abs(so[0]))
            total += st
    got = ddla.pdiag_logdet_finish(total, single=p in "sc")
    want = restated.diag_logdet(A)
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=mb, nb=nb)
    whole = ddla.pdiag_logdet(dA)
    for ref in (want, whole):
        assert abs(got.real - ref.real) <= tol * max(1.0, abs(ref.real))
        assert abs(math.remainder(got.imag - ref.imag, 2 * math.pi)) <= tol * 10
