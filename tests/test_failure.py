"""Failure paths of the Cholesky routines, made on the host or by a wait that runs out.

* Allocation failure (the reference's preparation_failure_{ppotrf,ppotrs,pposv}
  cases, tests/pblas_alloc_failure.cpp with tests/CMakeLists.txt:94-178): the
  n-th allocation of a call fails; the call must raise, leave A and B exactly as
  they were, release every workspace, and the handle must then solve normally.
* A device wait that runs out: with the wait budget cut to one cycle, the fused
  solve's CTAs give up on the flags of the block rows before them, the kernel
  records the timeout in its status word and returns; the host raises it as an
  error; with the default budget restored the same handle solves normally.
No GPU is faulted, trapped or hung: every wait ends by its budget.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ddla():
    from libddla_b200 import ddla

    return ddla


def _spd(rng, n):
    G = rng.standard_normal((n, n))
    return G @ G.T / n + np.eye(n)


@pytest.mark.parametrize("op", ["ppotrf", "ppotrs", "pposv", "ppotrf_bottom_right"])
def test_allocation_failure_leaves_matrices_and_handle_intact(handle, op):
    ddla = _ddla()
    C = ddla._c_api
    rng = np.random.default_rng(31)
    n, nrhs = 300, 5
    A = _spd(rng, n)
    B = rng.standard_normal((n, nrhs))
    F, info = np.linalg.cholesky(A), 0
    fired = 0
    for nth in (1, 2, 3):
        dA = ddla.DistributedMatrix.from_global_matrix(handle, F if op == "ppotrs" else A, mb=64, nb=64)
        dB = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=64, nb=64)
        before_a, before_b = dA.to_host(full_lld=True), dB.to_host(full_lld=True)
        C.ddla_c_fail_allocation(nth)
        try:
            if op == "ppotrf":
                ddla.ppotrf(dA, "L")
            elif op == "ppotrs":
                ddla.ppotrs(dA, dB, "L")
            elif op == "pposv":
                ddla.pposv(dA, dB, "L")
            else:
                ddla.ppotrf_bottom_right(dA, "L")
        except C.DdlaError as exc:
            fired += 1
            assert "out of memory" in str(exc) or "allocation" in str(exc), str(exc)
            np.testing.assert_array_equal(dA.to_host(full_lld=True), before_a)
            np.testing.assert_array_equal(dB.to_host(full_lld=True), before_b)
        finally:
            C.ddla_c_fail_allocation(0)
        assert C.ddla_c_live_workspaces() == 0
    assert fired >= 1  # every routine allocates its workspace before any device work
    # the same handle, unarmed: a normal solve
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=64, nb=64)
    dB = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=64, nb=64)
    X, info = ddla.pposv(dA, dB, "L")
    assert info == 0
    assert np.max(np.abs(A @ X.to_global_matrix() - B)) <= 1e-10 * np.max(np.abs(B))
    assert C.ddla_c_live_workspaces() == 0


def test_allocation_failure_of_handle_and_malloc():
    ddla = _ddla()
    C = ddla._c_api
    C.ddla_c_fail_allocation(1)  # the handle's pinned word in ddla_c_set
    try:
        with pytest.raises(C.DdlaError):
            ddla.Handle(ddla.Backend.GPU)
    finally:
        C.ddla_c_fail_allocation(0)
    with ddla.Handle(ddla.Backend.GPU) as h:
        C.ddla_c_fail_allocation(1)
        try:
            with pytest.raises(C.DdlaError):
                h.malloc(1 << 20)
        finally:
            C.ddla_c_fail_allocation(0)
        p = h.malloc(1 << 20)
        h.free(p)


def test_wait_timeout_is_reported_and_handle_recovers(handle):
    ddla = _ddla()
    C = ddla._c_api
    rng = np.random.default_rng(32)
    n, nrhs = 8192, 16
    R = rng.random((n, n))
    A = 2.0 * np.eye(n) + (R + R.T) / (4 * n)  # diagonally dominant: SPD
    del R
    B = rng.standard_normal((n, nrhs))
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=256, nb=256)
    _, info = ddla.ppotrf(dA, "L")
    assert info == 0
    dB = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=256, nb=256)
    assert C.ddla_c_set_wait_budget(handle.ptr, 1) == 0
    try:
        with pytest.raises(C.DdlaError, match="timed out"):
            ddla.ppotrs(dA, dB, "L")
    finally:
        assert C.ddla_c_set_wait_budget(handle.ptr, 0) == 0
    dB = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=256, nb=256)
    ddla.ppotrs(dA, dB, "L")
    X = dB.to_global_matrix()
    assert np.max(np.abs(A @ X - B)) <= 1e-9 * np.max(np.abs(B))
