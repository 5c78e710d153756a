"""The refinement solve's unit queue (k_bis_chain), checked on the host.

The kernel hands units out in increasing order and a unit waits only on counters
that units published.  This walks the queue exactly as the kernel decodes it
(ddlak_bis_queue_unit) and checks, against the waiting and publishing rules the
kernel follows:
  * every wait of a unit is already satisfied by the units before it in the queue,
    so the earliest unfinished unit can always run and the queue cannot deadlock;
  * every counter ends exactly at the value its readers wait for, so no reader
    starts before all of its inputs are in, and none waits forever;
  * every panel product (phase s, tile t, inner index k) and every entry of the
    triangular diagonal-block products is computed by exactly one unit;
  * all forward units come before all backward units.
No device work is involved.
"""
import ctypes

import pytest

BS, CT, TPB, KS = 1024, 64, 16, 256
QPB = BS // KS


def _lib():
    from libddla_b200.ddla import _c_api as C
    lib = C.lib
    lib.ddlak_bis_queue_size.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_longlong),
                                         ctypes.POINTER(ctypes.c_longlong)]
    lib.ddlak_bis_queue_size.restype = ctypes.c_int
    ip = ctypes.POINTER(ctypes.c_int)
    lib.ddlak_bis_queue_unit.argtypes = [ctypes.c_int, ctypes.c_longlong, ip, ip, ip, ip]
    lib.ddlak_bis_queue_unit.restype = ctypes.c_int
    return lib


def _queue(n):
    lib = _lib()
    nf, tot = ctypes.c_longlong(), ctypes.c_longlong()
    assert lib.ddlak_bis_queue_size(n, ctypes.byref(nf), ctypes.byref(tot)) == 0
    k, s, i, q = (ctypes.c_int() for _ in range(4))
    units = []
    for u in range(tot.value):
        assert lib.ddlak_bis_queue_unit(n, u, ctypes.byref(k), ctypes.byref(s), ctypes.byref(i), ctypes.byref(q)) == 0
        units.append((k.value, s.value, i.value, q.value))
    return nf.value, units


def _cover(acc, key, lo, hi):
    acc.setdefault(key, []).append((lo, hi))


def _exactly_once(intervals, lo, hi):
    iv = sorted(intervals)
    pos = lo
    for a, b in iv:
        if a != pos or b <= a:
            return False
        pos = b
    return pos == hi


@pytest.mark.parametrize("n", [1, 5, 64, 65, 1000, 1024, 1025, 2049, 3000, 4100, 8192, 9000, 20000])
def test_queue_order_counts_and_coverage(n):
    nf, units = _queue(n)
    S, Tt = -(-n // BS), -(-n // CT)
    bsz = lambda s: min(BS, n - s * BS)
    dp = lambda s: -(-bsz(s) // CT)
    nq = lambda s: -(-bsz(s) // KS)
    fds = lambda b, p: -(-min((p + 1) * CT, b) // KS)
    bds = lambda b, p: -(-b // KS) - (p * CT) // KS
    need_b = lambda s: 0 if s == S - 1 else QPB * (S - 2 - s) + nq(S - 1)

    cnt = {}
    panel_f, panel_b, diag_f, diag_b = {}, {}, {}, {}
    for u, (kind, s, idx, kq) in enumerate(units):
        assert (kind in (0, 1, 4)) == (u < nf), (n, u, kind)
        assert 0 <= s < S
        b = bsz(s)
        waits, inc = [], []
        if kind == 0:  # forward diagonal slice: rows of part idx, columns of slice kq
            r0 = idx * CT
            k0, k1 = kq * KS, min(kq * KS + KS, r0 + CT, b)
            assert k1 > k0
            waits = [(("cf", s * TPB + t), QPB * s) for t in range(k0 // CT, (k1 - 1) // CT + 1)]
            inc = [(("yd", s * TPB + idx), 1)]
            _cover(diag_f, (s, idx), k0, k1)
        elif kind in (1, 4):  # forward panel: row tile idx below block s
            assert idx // TPB > s and idx < Tt
            k0, k1 = (kq * KS, min(kq * KS + KS, b)) if kind == 1 else (0, b)
            waits = [(("yd", s * TPB + p), fds(b, p)) for p in range(k0 // CT, (k1 - 1) // CT + 1)]
            inc = [(("cf", idx), 1 if kind == 1 else nq(s))]
            _cover(panel_f, (s, idx), k0, k1)
        elif kind == 2:  # backward diagonal slice
            r0 = idx * CT
            k0, k1 = max(kq * KS, r0), min(kq * KS + KS, b)
            assert k1 > k0
            waits = [(("cb", s * TPB + t), need_b(s)) for t in range(k0 // CT, (k1 - 1) // CT + 1)]
            if s == S - 1:
                waits.append((("fd", 0), nf))
            inc = [(("xd", s * TPB + idx), 1)]
            _cover(diag_b, (s, idx), k0, k1)
        else:  # backward panel: column tile idx left of block s, rows of block s
            assert kind in (3, 5) and idx // TPB < s
            k0, k1 = (kq * KS, min(kq * KS + KS, b)) if kind == 3 else (0, b)
            waits = [(("xd", s * TPB + p), bds(b, p)) for p in range(k0 // CT, (k1 - 1) // CT + 1)]
            inc = [(("cb", idx), 1 if kind == 3 else nq(s))]
            _cover(panel_b, (s, idx), k0, k1)
        for key, want in waits:
            assert cnt.get(key, 0) >= want, ("a wait on a later unit", n, u, units[u], key, want, cnt.get(key, 0))
        for key, v in inc:
            cnt[key] = cnt.get(key, 0) + v
        if kind in (0, 1, 4):
            cnt[("fd", 0)] = cnt.get(("fd", 0), 0) + 1

    assert cnt.get(("fd", 0), 0) == nf
    for s in range(S):
        for t in range(dp(s)):
            assert cnt.get(("cf", s * TPB + t), 0) == QPB * s, ("cnt_f", n, s, t)
            assert cnt.get(("cb", s * TPB + t), 0) == need_b(s), ("cnt_b", n, s, t)
        for p in range(dp(s)):
            assert cnt[("yd", s * TPB + p)] == fds(bsz(s), p)
            assert cnt[("xd", s * TPB + p)] == bds(bsz(s), p)
            # forward part p needs columns 0 .. min((p+1)*64, bsz); backward part p columns p*64 .. bsz
            assert _exactly_once(diag_f[(s, p)], 0, min((p + 1) * CT, bsz(s))), ("diag_f", n, s, p)
            assert _exactly_once(diag_b[(s, p)], p * CT, bsz(s)), ("diag_b", n, s, p)
        for t in range((s + 1) * TPB, Tt):
            assert _exactly_once(panel_f[(s, t)], 0, bsz(s)), ("panel_f", n, s, t)
        for c in range(s * TPB):
            assert _exactly_once(panel_b[(s, c)], 0, bsz(s)), ("panel_b", n, s, c)
    assert len(panel_f) == sum(max(0, Tt - (s + 1) * TPB) for s in range(S))
    assert len(panel_b) == sum(s * TPB for s in range(S))


def test_queue_rejects_bad_arguments():
    lib = _lib()
    x = ctypes.c_longlong()
    k = ctypes.c_int()
    assert lib.ddlak_bis_queue_size(0, ctypes.byref(x), ctypes.byref(x)) != 0
    nf, tot = ctypes.c_longlong(), ctypes.c_longlong()
    assert lib.ddlak_bis_queue_size(100, ctypes.byref(nf), ctypes.byref(tot)) == 0
    assert lib.ddlak_bis_queue_unit(100, tot.value, *(ctypes.byref(k) for _ in range(4))) != 0
    assert lib.ddlak_bis_queue_unit(100, -1, *(ctypes.byref(k) for _ in range(4))) != 0
