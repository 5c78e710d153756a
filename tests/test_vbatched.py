"""Batched uneven Cholesky (ddla_{s,d}_posv_vbatched): parity of every matrix's
factor, solution and log-determinant with the oracle's per-matrix potrf /
ppotrs / diag_logdet, LAPACK info on failures, graph-plan replay, the 1024
kernel instance, argument errors and the autotuner's table."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import restated

pytestmark = pytest.mark.gpu


def _ddla():
    from libddla_b200 import ddla
    return ddla


def spd_batch(rng, orders, dt):
    """A_i = G_i G_i^T / n_i + 0.1 I with G_i iid N(0,1); b_i iid N(0,1)."""
    mats, rhs = [], []
    for n in orders:
        G = rng.standard_normal((n, n))
        mats.append((G @ G.T / n + 0.1 * np.eye(n)).astype(dt))
        rhs.append(rng.standard_normal(n).astype(dt))
    return mats, rhs


def run_batch(handle, mats, rhs, dt, max_n=None, plan=False):
    import torch
    from libddla_b200.ddla import batched
    pb = batched.pack(mats, rhs, dtype=dt, max_n=max_n)
    if plan:
        p = batched.VbatchedPlan(handle, pb)
        p.run()
        torch.cuda.synchronize()
        p.close()
    else:
        batched.posv_vbatched(handle, pb)
        torch.cuda.synchronize()
    F = [pb.matrix(i).cpu().numpy() for i in range(pb.batch)]
    X = [pb.vector(i).cpu().numpy() for i in range(pb.batch)] if rhs is not None else None
    return F, X, pb.logdet.cpu().numpy(), pb.info.cpu().numpy()


def check_against_oracle(A, F, x, ld, info, b, dt):
    Fo, info_o = restated.potrf(A, "L")
    assert info == info_o
    tol = 1e-4 if dt == np.float32 else 1e-12
    n = A.shape[0]
    # the upper triangle is untouched
    iu = np.triu_indices(n, 1)
    assert np.array_equal(F[iu], A[iu])
    rel_f = np.max(np.abs(np.tril(F) - np.tril(Fo))) / np.max(np.abs(Fo))
    assert rel_f < tol, rel_f
    ld_o = 2.0 * restated.diag_logdet(np.tril(Fo)).real
    assert abs(ld - ld_o) <= (1e-4 if dt == np.float32 else 1e-11) * max(1.0, abs(ld_o)), (ld, ld_o)
    if x is not None:
        xo = restated.ppotrs(Fo, b.reshape(n, 1).astype(dt), "L").ravel()
        rel_x = np.max(np.abs(x - xo)) / np.max(np.abs(xo))
        assert rel_x < tol * 10, rel_x


EDGE = [1, 2, 7, 8, 9, 15, 16, 17, 31, 32, 33, 47, 63, 64, 65, 100, 127, 128, 129, 255, 256, 257, 300, 480, 511, 512]


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_vbatched_parity(handle, dt):
    rng = np.random.default_rng(0xDD1A0004)
    orders = EDGE + list(rng.integers(16, 513, size=24))
    rng.shuffle(orders)
    mats, rhs = spd_batch(rng, orders, dt)
    F, X, ld, info = run_batch(handle, mats, rhs, dt)
    for i, A in enumerate(mats):
        check_against_oracle(A, F[i], X[i], ld[i], info[i], rhs[i], dt)


def test_vbatched_factor_only(handle):
    rng = np.random.default_rng(11)
    orders = [5, 40, 130, 512]
    mats, _ = spd_batch(rng, orders, np.float64)
    F, X, ld, info = run_batch(handle, mats, None, np.float64)
    assert X is None
    for i, A in enumerate(mats):
        check_against_oracle(A, F[i], None, ld[i], info[i], None, np.float64)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_vbatched_not_positive_definite(handle, dt):
    rng = np.random.default_rng(12)
    orders = [40, 64, 100, 200, 300, 17, 512, 33]
    mats, rhs = spd_batch(rng, orders, dt)
    # matrix 1: indefinite at leading minor 10; 3: at the last order; 5: NaN on the
    # diagonal; 6: negative first pivot
    mats[1][9, 9] = -50.0
    mats[3][199, 199] = -1e3
    mats[5][4, 4] = np.nan
    mats[6][0, 0] = -1.0
    F, X, ld, info = run_batch(handle, mats, rhs, dt)
    for i, A in enumerate(mats):
        Fo, info_o = restated.potrf(A, "L")
        assert info[i] == info_o, (i, info[i], info_o)
        if info_o:
            assert np.isnan(ld[i])
            assert np.array_equal(X[i], rhs[i])  # b untouched
            k = info_o - 1  # leading columns are the factor's
            if k:
                rel = np.max(np.abs(np.tril(F[i])[:, :k] - np.tril(Fo)[:, :k])) / np.max(np.abs(np.tril(Fo)[:, :k]))
                assert rel < (1e-4 if dt == np.float32 else 1e-12)
        else:
            check_against_oracle(A, F[i], X[i], ld[i], info[i], rhs[i], dt)
    assert info[1] == 10 and info[3] == 200 and info[5] == 5 and info[6] == 1


def test_vbatched_plan_replay_matches_direct(handle):
    """The graph-captured launch replayed several times gives the direct call's bits
    (and the work counters are reset after every launch)."""
    import torch
    from libddla_b200.ddla import batched
    rng = np.random.default_rng(13)
    orders = list(rng.integers(16, 513, size=300))
    mats, rhs = spd_batch(rng, orders, np.float64)
    F0, X0, ld0, info0 = run_batch(handle, mats, rhs, np.float64)
    pb = batched.pack(mats, rhs, dtype=np.float64)
    A0 = pb.mats.clone()
    B0 = pb.rhs.clone()
    plan = batched.VbatchedPlan(handle, pb)
    assert plan.info()["grid"] > 0
    for _ in range(3):
        pb.mats.copy_(A0)
        pb.rhs.copy_(B0)
        torch.cuda.synchronize()  # the plan runs on the handle's stream, not torch's
        plan.run()
        torch.cuda.synchronize()
        assert np.array_equal(pb.info.cpu().numpy(), info0)
        assert np.array_equal(pb.logdet.cpu().numpy(), ld0)
        for i in range(0, pb.batch, 37):
            assert np.array_equal(pb.matrix(i).cpu().numpy(), F0[i])
            assert np.array_equal(pb.vector(i).cpu().numpy(), X0[i])
    plan.close()


def test_vbatched_nmax_1024(handle):
    rng = np.random.default_rng(14)
    orders = [600, 1000, 1024, 513, 20]
    mats, rhs = spd_batch(rng, orders, np.float64)
    F, X, ld, info = run_batch(handle, mats, rhs, np.float64)
    for i, A in enumerate(mats):
        check_against_oracle(A, F[i], X[i], ld[i], info[i], rhs[i], np.float64)


def test_vbatched_empty_and_argument_errors(handle):
    import torch
    ddla = _ddla()
    from libddla_b200.ddla import batched
    C = ddla._c_api
    pb = batched.pack([np.eye(4)], [np.ones(4)], dtype=np.float64)
    # empty batch: no-op
    C.check_status(C.ddla_d_posv_vbatched(handle.ptr, b"L", None, None, None, None, None, None, 0, 0), "empty")
    args = (pb.d_n.data_ptr(), pb.d_A.data_ptr(), pb.d_lda.data_ptr(), pb.d_B.data_ptr(), pb.logdet.data_ptr(),
            pb.info.data_ptr(), 1)
    with pytest.raises(ddla.DdlaError):
        C.check_status(C.ddla_d_posv_vbatched(handle.ptr, b"U", *args, 4), "uplo U")
    with pytest.raises(ddla.DdlaError):
        C.check_status(C.ddla_d_posv_vbatched(handle.ptr, b"L", *args, 2048), "max_n")
    with pytest.raises(ddla.DdlaError):
        C.check_status(C.ddla_d_posv_vbatched(handle.ptr, b"L", *args, 3), "order > max_n")
    with pytest.raises(ddla.DdlaError):
        C.check_status(C.ddla_d_posv_vbatched(handle.ptr, b"L", None, *args[1:], 4), "null orders")
    # an order-0 matrix in a batch: info 0, logdet 0
    pb0 = batched.pack([np.zeros((0, 0)), 2 * np.eye(3)], [np.zeros(0), np.ones(3)], dtype=np.float64)
    batched.posv_vbatched(handle, pb0)
    torch.cuda.synchronize()
    assert list(pb0.info.cpu().numpy()) == [0, 0]
    ld = pb0.logdet.cpu().numpy()
    assert ld[0] == 0.0 and abs(ld[1] - 3 * np.log(2.0)) < 1e-14
    assert np.allclose(pb0.vector(1).cpu().numpy(), 0.5)


def test_vbatched_autotune_and_tune_file(handle, tmp_path):
    """The autotuner fills a table for the device; DDLA_VBATCHED_TUNE_FILE persists it
    and a fresh process loads it."""
    from libddla_b200.ddla import batched
    t0 = batched.tuning(handle, "d", 512)
    assert t0["grid"] > 0 and t0["widths"] == [8, 16]
    path = tmp_path / "vb.tune"
    code = (
        "import json, sys; sys.path.insert(0, '.');"
        "from libddla_b200 import ddla; from libddla_b200.ddla import batched;"
        "h = ddla.Handle(ddla.Backend.GPU);"
        "t = batched.tuning(h, 'd', 512);"
        "do = sys.argv[1] == 'tune';"
        "do and batched.autotune(h, 'd', 300);"
        "t2 = batched.tuning(h, 'd', 512);"
        "print(json.dumps({'before': t, 'after': t2}))"
    )
    env = dict(os.environ, DDLA_VBATCHED_TUNE_FILE=str(path))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", code, "tune"], cwd=root, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert not out["before"]["tuned"] and out["after"]["tuned"]
    assert all(v in (0, 1) for v in out["after"]["variant"]) and len(out["after"]["variant"]) == 32
    assert path.exists() and path.read_text().split()[1] == "d"
    r = subprocess.run([sys.executable, "-c", code, "load"], cwd=root, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    out2 = json.loads(r.stdout.strip().splitlines()[-1])
    assert out2["before"]["tuned"] and out2["before"] == out["after"]
