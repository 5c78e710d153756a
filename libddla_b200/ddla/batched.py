"""Batched uneven Cholesky (factor + solve + log-determinant) from Python.

Thin ctypes layer over ddla_{s,d}_posv_vbatched / _plan (include/ddla_c.h;
semantics in include/ddla/ddla_batched.h).  PyTorch provides the device
memory: `pack` copies a list of square matrices (and right-hand sides) into one
device buffer with the device-resident order / leading-dimension / pointer
arrays the C ABI takes.  No reference counterpart: the reference has no
batched Cholesky; its per-matrix equivalent is ops.pposv + ops.diag_logdet.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _c_api as C

_ALIGN = 32  # elements: every matrix and vector starts on a 256-byte boundary


def _torch():
    import torch
    return torch


@dataclass
class PackedBatch:
    """Device-resident batch: one buffer of matrices, one of right-hand sides,
    and the arrays the C ABI reads (all torch tensors on one CUDA device)."""
    dtype: np.dtype
    orders: np.ndarray        # host copy of the orders
    a_offsets: np.ndarray     # element offset of matrix i in `mats`
    b_offsets: np.ndarray
    mats: "object"            # torch 1-D tensor
    rhs: "object"             # torch 1-D tensor or None
    d_n: "object"
    d_lda: "object"
    d_A: "object"             # int64 device pointers
    d_B: "object"
    logdet: "object"          # float64 [batch]
    info: "object"            # int32 [batch]
    max_n: int

    @property
    def batch(self) -> int:
        return len(self.orders)

    def matrix(self, i: int):
        """Device view of matrix i, column-major (n x n, lda = n)."""
        n = int(self.orders[i])
        o = int(self.a_offsets[i])
        return self.mats[o:o + n * n].view(n, n).t()

    def vector(self, i: int):
        n = int(self.orders[i])
        o = int(self.b_offsets[i])
        return self.rhs[o:o + n]


def pack(mats: Sequence[np.ndarray], rhs: Optional[Sequence[np.ndarray]] = None, device="cuda",
         dtype=np.float64, max_n: Optional[int] = None) -> PackedBatch:
    """Copy host matrices (square, any layout) and optional vectors to the device."""
    torch = _torch()
    dt = np.dtype(dtype)
    tdt = {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32}[dt]
    orders = np.array([m.shape[0] for m in mats], dtype=np.int32)
    for m in mats:
        if m.ndim != 2 or m.shape[0] != m.shape[1]:
            raise ValueError("pack: matrices must be square")
    sizes = (orders.astype(np.int64) ** 2 + _ALIGN - 1) // _ALIGN * _ALIGN
    a_off = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    host = np.zeros(int(sizes.sum()) if len(sizes) else 0, dtype=dt)
    for i, m in enumerate(mats):
        n = orders[i]
        host[a_off[i]:a_off[i] + n * n] = np.asarray(m, dtype=dt).ravel(order="F")
    d_mats = torch.from_numpy(host).to(device)
    d_rhs = None
    b_off = np.zeros(len(mats), dtype=np.int64)
    if rhs is not None:
        vs = (orders.astype(np.int64) + _ALIGN - 1) // _ALIGN * _ALIGN
        b_off = np.concatenate([[0], np.cumsum(vs)[:-1]]).astype(np.int64)
        hb = np.zeros(int(vs.sum()) if len(vs) else 0, dtype=dt)
        for i, v in enumerate(rhs):
            hb[b_off[i]:b_off[i] + orders[i]] = np.asarray(v, dtype=dt).ravel()
        d_rhs = torch.from_numpy(hb).to(device)
    es = dt.itemsize
    a_ptrs = d_mats.data_ptr() + a_off * es
    b_ptrs = (d_rhs.data_ptr() + b_off * es) if d_rhs is not None else None
    mx = int(orders.max()) if len(orders) else 0
    return PackedBatch(
        dtype=dt, orders=orders, a_offsets=a_off, b_offsets=b_off, mats=d_mats, rhs=d_rhs,
        d_n=torch.from_numpy(orders).to(device),
        d_lda=torch.from_numpy(np.maximum(orders, 1).astype(np.int32)).to(device),
        d_A=torch.from_numpy(a_ptrs.astype(np.int64)).to(device),
        d_B=torch.from_numpy(b_ptrs.astype(np.int64)).to(device) if b_ptrs is not None else None,
        logdet=torch.zeros(len(mats), dtype=torch.float64, device=device),
        info=torch.zeros(len(mats), dtype=torch.int32, device=device),
        max_n=int(max_n if max_n is not None else mx))


def _sfx(pb: PackedBatch) -> str:
    return "d" if pb.dtype == np.float64 else "s"


def _args(pb: PackedBatch):
    return (pb.d_n.data_ptr(), pb.d_A.data_ptr(), pb.d_lda.data_ptr(),
            pb.d_B.data_ptr() if pb.d_B is not None else None,
            pb.logdet.data_ptr(), pb.info.data_ptr(), pb.batch, pb.max_n)


def posv_vbatched(handle, pb: PackedBatch, uplo: str = "L") -> None:
    """One persistent launch over the batch (enqueued on the handle's stream)."""
    fn = getattr(C, f"ddla_{_sfx(pb)}_posv_vbatched")
    C.check_status(fn(handle.ptr, uplo.encode(), *_args(pb)), "posv_vbatched")


class VbatchedPlan:
    """The launch captured once in a CUDA graph; run() replays it on the handle's
    stream (its own CUDA stream: inputs written through torch must be complete,
    e.g. torch.cuda.synchronize(), before run())."""

    def __init__(self, handle, pb: PackedBatch, uplo: str = "L"):
        self._pb = pb
        self._ptr = ctypes.c_void_p()
        fn = getattr(C, f"ddla_{_sfx(pb)}_posv_vbatched_plan")
        C.check_status(fn(handle.ptr, uplo.encode(), *_args(pb), ctypes.byref(self._ptr)), "VbatchedPlan")

    def run(self) -> None:
        C.check_status(C.ddla_vbatched_plan_run(self._ptr), "VbatchedPlan.run")

    def info(self):
        g = ctypes.c_int()
        f = ctypes.c_double()
        C.check_status(C.ddla_vbatched_plan_info(self._ptr, ctypes.byref(g), ctypes.byref(f)), "VbatchedPlan.info")
        return {"grid": g.value, "flops": f.value}

    def close(self) -> None:
        if self._ptr:
            C.check_status(C.ddla_vbatched_plan_destroy(self._ptr), "VbatchedPlan.close")
            self._ptr = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(handle, dtype: str, max_n: int) -> None:
    C.check_status(C.ddla_vbatched_autotune(handle.ptr, dtype.encode(), int(max_n)), "vbatched autotune")


def tuning(handle, dtype: str, max_n: int) -> dict:
    g = ctypes.c_int()
    w = (ctypes.c_int * 2)()
    v = (ctypes.c_ubyte * 64)()
    t = ctypes.c_int()
    C.check_status(C.ddla_vbatched_tuning(handle.ptr, dtype.encode(), int(max_n), ctypes.byref(g), w, v, 64,
                                          ctypes.byref(t)), "vbatched tuning")
    nb = (512 if max_n <= 512 else 1024) // 16
    return {"grid": g.value, "widths": [w[0], w[1]], "variant": [v[i] for i in range(nb)], "tuned": bool(t.value)}


def shard_lpt(orders, world: int):
    """Partition a batch over `world` ranks by longest-processing-time on the
    factorization cost n^3 (each matrix to the least-loaded rank, largest first).
    Returns one sorted index list per rank; every index appears exactly once and
    the loads differ by at most the cost of one matrix."""
    import heapq

    if world < 1:
        raise ValueError("shard_lpt: world must be >= 1")
    orders = [int(n) for n in orders]
    order = sorted(range(len(orders)), key=lambda i: (-orders[i], i))
    heap = [(0.0, r) for r in range(world)]
    shards = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(orders[i]) ** 3, r))
    return [sorted(s) for s in shards]


def sharded_run(orders, compute, group=None, device=None):
    """One process per GPU over a batch: this rank's LPT shard (shard_lpt) is
    handed to compute(indices) -> (len(indices), k) tensor of per-matrix results
    (e.g. logdet and info from posv_vbatched on the shard), and one all-gather of
    (index, values) rows gives every rank the (len(orders), k) float64 result in
    the batch's order.  It is the only exchange step of the sharded batch.
    Without an initialised torch.distributed group it runs the whole batch
    locally.  device: where the exchange buffers live (the backend's device,
    e.g. cuda:r for NCCL); default: compute's result device."""
    import torch

    dist = torch.distributed
    world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    rank = dist.get_rank(group) if world > 1 else 0
    shards = shard_lpt(orders, world)
    mine = shards[rank]
    vals = torch.as_tensor(compute(list(mine)), dtype=torch.float64)
    if vals.dim() == 1:
        vals = vals.unsqueeze(1)
    if vals.shape[0] != len(mine):
        raise ValueError("sharded_run: compute must return one row per index")
    dev = torch.device(device) if device is not None else vals.device
    k = vals.shape[1]
    out = torch.full((len(orders), k), float("nan"), dtype=torch.float64, device=dev)
    if world == 1:
        out[torch.as_tensor(list(mine), dtype=torch.long, device=dev)] = vals.to(dev)
        return out
    m = max(len(sh) for sh in shards)
    buf = torch.full((m, 1 + k), -1.0, dtype=torch.float64, device=dev)
    if mine:
        buf[:len(mine), 0] = torch.as_tensor(list(mine), dtype=torch.float64, device=dev)
        buf[:len(mine), 1:] = vals.to(dev)
    gathered = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(gathered, buf, group=group)
    for g in gathered:
        rows = g[:, 0] >= 0
        out[g[rows, 0].long()] = g[rows, 1:]
    return out


# ---- variable-size batched GEMM --------------------------------------------
_GV_SFX = {"torch.float32": "s", "torch.float64": "d", "torch.complex64": "c", "torch.complex128": "z"}


def gemm_vbatched(handle, transA: str, transB: str, m, n, k, alpha, A_list, lda, B_list, ldb, beta, C_list, ldc,
                  d_m=None, d_n=None, d_k=None) -> None:
    """C_i = alpha op(A_i) op(B_i) + beta C_i for every i (ddla_?_gemm_vbatched, the
    reference's gemmVbatched).  A_list / B_list / C_list are CUDA tensors (or None
    for a null entry) holding column-major matrices at their data_ptr; m, n, k,
    lda, ldb, ldc are per-entry integer sequences.  d_m / d_n / d_k override the
    device size arrays (e.g. to pass a null one).  Completes before returning."""
    torch = _torch()
    tensors = [t for t in list(A_list) + list(B_list) + list(C_list) if t is not None]
    if not tensors:
        raise ValueError("gemm_vbatched: at least one matrix is needed to fix the type")
    first = lambda xs: next((str(t.dtype) for t in xs if t is not None), None)
    ta_, tb_, tc_ = first(A_list), first(B_list), first(C_list)
    kinds = {t for t in (ta_, tb_, tc_) if t is not None}
    mixed = ""
    if len(kinds) > 1:
        # one real and one complex operand, complex output: the mixed overloads
        if ta_ is not None and tb_ is not None and "complex" in ta_ and "complex" not in tb_:
            mixed = "_cr"
        elif ta_ is not None and tb_ is not None and "complex" not in ta_ and "complex" in tb_:
            mixed = "_rc"
        else:
            raise TypeError(f"gemm_vbatched: operand types {ta_}, {tb_}, {tc_} do not form a supported combination")
    sfx = _GV_SFX[tc_ or str(tensors[0].dtype)]
    dev = tensors[0].device
    batch = len(C_list)

    def iarr(v):
        return torch.tensor(np.asarray(v, dtype=np.int32), device=dev)

    def parr(ts):
        return torch.tensor(np.array([0 if t is None else t.data_ptr() for t in ts], dtype=np.int64), device=dev)

    dm = iarr(m) if d_m is None else d_m
    dn = iarr(n) if d_n is None else d_n
    dk = iarr(k) if d_k is None else d_k
    dlda, dldb, dldc = iarr(lda), iarr(ldb), iarr(ldc)
    pa, pb, pc = parr(A_list), parr(B_list), parr(C_list)
    sdt = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}[sfx]
    al = np.array([alpha], dtype=sdt)
    be = np.array([beta], dtype=sdt)
    torch.cuda.synchronize(dev)  # inputs written on torch's stream; the call runs on the handle's

    fn = getattr(C, f"ddla_{sfx}_gemm_vbatched{mixed}")
    C.check_status(fn(handle.ptr, transA.encode(), transB.encode(), _ptr(dm), _ptr(dn), _ptr(dk), al.ctypes.data,
                      _ptr(pa), _ptr(dlda), _ptr(pb), _ptr(dldb), be.ctypes.data, _ptr(pc), _ptr(dldc), batch),
                   "gemm_vbatched")
    C.check_status(C.ddla_c_synchronize(handle.ptr), "gemm_vbatched: synchronize")


def _ptr(t):
    return None if t is None or (hasattr(t, "numel") and t.numel() == 0) else t.data_ptr()


def _addr(x):
    """Device address of an entry: a CUDA tensor, an int address, or None (null)."""
    if x is None:
        return 0
    return int(x) if isinstance(x, int) else x.data_ptr()


def gemm_vbatched2s(handle, ops0: str, m0, n0, k0, alpha0, A0, lda0, B0, ldb0, C0, ldc0,
                    ops1: str, m1, n1, k1, alpha1, AB1, lda1, ldb1, beta1, C1, ldc1,
                    c0_left: bool, segments, dtype, beta0=0, pattern: str = "") -> None:
    """The two-stage batched GEMM (ddla_?_gemm_vbatched2s, the reference's
    gemmVbatched2s): per segment, C0_i = alpha0 op(A0_i) op(B0_i), then
    C1_i = alpha1 op(X_i) op(Y_i) + beta1 C1_i with (X, Y) = (C0_i, AB1_i) when
    c0_left, else (AB1_i, C0_i).  ops0 / ops1 are two-letter transpose pairs
    ("NN", "TC", ...); matrix entries are CUDA tensors, int device addresses (C0
    entries of different segments may share storage) or None; dtype is the
    torch dtype of C1.  pattern (e.g. "rzzr") selects a mixed overload by the
    element types of (A0, B0, C0, AB1), r real, z complex; alpha0 / beta0 then
    have C0's type.  Completes before returning."""
    torch = _torch()
    sfx = _GV_SFX[str(dtype)]
    batch = len(C1)
    tensors = [x for xs in (A0, B0, C0, AB1, C1) for x in xs if x is not None and not isinstance(x, int)]
    dev = tensors[0].device if tensors else torch.device("cuda")

    def iarr(v):
        return torch.tensor(np.asarray(v, dtype=np.int32), device=dev)

    def parr(xs):
        return torch.tensor(np.array([_addr(x) for x in xs], dtype=np.int64), device=dev)

    d = [iarr(v) for v in (m0, n0, k0, lda0, ldb0, ldc0, m1, n1, k1, lda1, ldb1, ldc1)]
    p = [parr(v) for v in (A0, B0, C0, AB1, C1)]
    sdt = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}[sfx]
    s0 = sdt
    if pattern:
        if sfx not in "cz" or len(pattern) != 4:
            raise ValueError("gemm_vbatched2s: a mixed pattern needs a complex C1 and four letters")
        s0 = sdt if pattern[2] == "z" else {"c": np.float32, "z": np.float64}[sfx]
    sc = [np.array([alpha0], dtype=s0), np.array([beta0], dtype=s0), np.array([alpha1], dtype=sdt),
          np.array([beta1], dtype=sdt)]
    seg = np.asarray(segments, dtype=np.int32)
    if dev.type == "cuda":
        torch.cuda.synchronize(dev)  # inputs written on torch's stream; the call runs on the handle's
    fn = getattr(C, f"ddla_{sfx}_gemm_vbatched2s" + (f"_{pattern}" if pattern else ""))
    C.check_status(fn(handle.ptr, ops0[0].encode(), ops0[1].encode(), _ptr(d[0]), _ptr(d[1]), _ptr(d[2]),
                      sc[0].ctypes.data, _ptr(p[0]), _ptr(d[3]), _ptr(p[1]), _ptr(d[4]), sc[1].ctypes.data,
                      _ptr(p[2]), _ptr(d[5]), ops1[0].encode(), ops1[1].encode(), _ptr(d[6]), _ptr(d[7]),
                      _ptr(d[8]), sc[2].ctypes.data, _ptr(p[3]), _ptr(d[9]), _ptr(d[10]), sc[3].ctypes.data,
                      _ptr(p[4]), _ptr(d[11]), int(bool(c0_left)), batch,
                      seg.ctypes.data if seg.size else None, int(seg.size)),
                   "gemm_vbatched2s")
    C.check_status(C.ddla_c_synchronize(handle.ptr), "gemm_vbatched2s: synchronize")
