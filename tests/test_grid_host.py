"""Host side of the process-grid path, without a GPU.

* The block-cyclic pieces `grid.local_piece` cuts have the shapes the library's
  own num_loc gives (ddla_c_numloc, the reference's ddla_desc.h:25-38), and
  `grid.assemble` puts every rank's piece back, for several grids, block sizes,
  source offsets and both rank orders.
* The NCCL library loads and makes clique ids; two gloo ranks exchange one
  (`grid.exchange_nccl_id`, the first step of `grid.nccl_grid_handle`) and
  both hold the same 128 bytes.
* A local group is created and released through the C ABI; the handle API
  rejects grids that do not match the group.
"""
import os

import numpy as np
import pytest


@pytest.mark.parametrize("m,n,mb,nb,P,Q,rsrc,csrc,major", [
    (97, 97, 16, 16, 2, 3, 0, 0, "R"), (130, 40, 32, 8, 3, 2, 1, 1, "C"), (5, 9, 8, 2, 2, 2, 1, 0, "R"),
    (1, 1, 4, 4, 3, 1, 2, 0, "C"), (200, 13, 24, 3, 2, 3, 1, 2, "R")])
def test_local_pieces_round_trip(native_lib, m, n, mb, nb, P, Q, rsrc, csrc, major):
    from libddla_b200.ddla import grid

    A = np.arange(m * n, dtype=np.float64).reshape(m, n)
    pieces = []
    for rank in range(P * Q):
        row, col = grid.rank_to_rc(rank, P, Q, major)
        p = grid.local_piece(A, mb, nb, P, Q, row, col, rsrc, csrc)
        assert p.shape == (native_lib.ddla_c_numloc(m, mb, row, rsrc, P), native_lib.ddla_c_numloc(n, nb, col, csrc, Q))
        assert p.flags.f_contiguous
        pieces.append(p)
    assert np.array_equal(grid.assemble(pieces, m, n, mb, nb, P, Q, rsrc, csrc, major), A)


def test_nccl_clique_id(native_lib):
    from libddla_b200.ddla import grid

    assert grid.nccl_available()
    a, b = grid.nccl_unique_id(), grid.nccl_unique_id()
    assert len(a) == 128 and a != b


def test_local_group_lifecycle(native_lib):
    import ctypes

    from libddla_b200.ddla import grid

    g = grid.LocalGroup(6, timeout_s=1.0)
    assert g.nranks == 6 and g.ptr.value
    g.close()
    bad = ctypes.c_void_p()
    assert native_lib.ddla_c_local_group_create(ctypes.byref(bad), 0, 1.0) == native_lib.STATUS_INVALID_VALUE


def _exchange(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from libddla_b200.ddla import grid

        uid = grid.exchange_nccl_id()
        out.put((rank, uid))
    finally:
        dist.destroy_process_group()


def test_nccl_id_exchange_over_two_gloo_ranks(native_lib):
    import multiprocessing as mp
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_exchange, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0] == got[1] and len(got[0]) == 128
