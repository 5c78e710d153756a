"""The oracle's Python face (TEST INFRASTRUCTURE ONLY: imported by tests/, the
smoke check and bench.py's CPU baseline, never by the product).

potrf, potrf_bottom_right, ppotrs, pposv and diag_logdet are ctypes wrappers of
oracle/ddla_oracle.c, whose C code restates the reference's CPU arm (see
ddla_oracle.c for the reference file:line each routine follows).  The batched
GEMM (gemm_vbatched, gemm_vbatched2s) and the Hermitian-definite reduction
(herm_complete, phegst) are restated here in NumPy/SciPy, each citing the
reference lines it follows.  Every function takes NumPy arrays and works on
copies.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB = None

_TC = {np.dtype(np.float32): "s", np.dtype(np.float64): "d", np.dtype(np.complex64): "c",
       np.dtype(np.complex128): "z"}


def _lib():
    global _LIB
    if _LIB is None:
        from .build import build

        path = build()
        L = ctypes.CDLL(str(path))
        vp, i, c = ctypes.c_void_p, ctypes.c_int, ctypes.c_char
        for p in "sdcz":
            getattr(L, f"oracle_{p}_potrf").argtypes = [c, i, vp, i]
            getattr(L, f"oracle_{p}_potrf").restype = i
            getattr(L, f"oracle_{p}_trsm").argtypes = [c, c, c, i, i, vp, i, vp, i]
            getattr(L, f"oracle_{p}_trsm").restype = None
            getattr(L, f"oracle_{p}_ppotrs").argtypes = [c, c, i, i, vp, i, vp, i]
            getattr(L, f"oracle_{p}_ppotrs").restype = None
            getattr(L, f"oracle_{p}_pposv").argtypes = [c, c, i, i, vp, i, vp, i]
            getattr(L, f"oracle_{p}_pposv").restype = i
            getattr(L, f"oracle_{p}_potrf_bottom_right").argtypes = [c, i, vp, i]
            getattr(L, f"oracle_{p}_potrf_bottom_right").restype = i
            getattr(L, f"oracle_{p}_diag_logdet").argtypes = [i, vp, i, vp]
            getattr(L, f"oracle_{p}_diag_logdet").restype = i
        _LIB = L
    return _LIB


def _f(a: np.ndarray) -> np.ndarray:
    return np.array(a, order="F", copy=True)


def potrf(a: np.ndarray, uplo: str = "L", n: int | None = None):
    """Return (factor array, info).  Only the uplo triangle of the leading n x n is touched."""
    A = _f(a)
    n = A.shape[1] if n is None else n
    info = getattr(_lib(), f"oracle_{_TC[A.dtype]}_potrf")(uplo.encode(), n, A.ctypes.data, max(1, A.shape[0]))
    return A, int(info)


def potrf_bottom_right(a: np.ndarray, uplo: str = "U", n: int | None = None):
    """Return (factor array, info) of the bottom-right factorization: A = U U^H ('U') or L^H L ('L')."""
    A = _f(a)
    n = A.shape[1] if n is None else n
    info = getattr(_lib(), f"oracle_{_TC[A.dtype]}_potrf_bottom_right")(uplo.encode(), n, A.ctypes.data,
                                                                         max(1, A.shape[0]))
    return A, int(info)


def ppotrs(factor: np.ndarray, b: np.ndarray, uplo: str = "L", side: str = "L", n: int | None = None):
    A = np.asfortranarray(factor)
    B = _f(b.astype(A.dtype))
    n = A.shape[1] if n is None else n
    nrhs = B.shape[1] if side == "L" else B.shape[0]
    getattr(_lib(), f"oracle_{_TC[A.dtype]}_ppotrs")(side.encode(), uplo.encode(), n, nrhs, A.ctypes.data,
                                                     max(1, A.shape[0]), B.ctypes.data, max(1, B.shape[0]))
    return B


def pposv(a: np.ndarray, b: np.ndarray, uplo: str = "L", side: str = "L"):
    """Return (factor, X, info); X is b unchanged when info != 0 (pposv.cpp:36-38)."""
    A = _f(a)
    B = _f(b.astype(A.dtype))
    n = A.shape[1]
    nrhs = B.shape[1] if side == "L" else B.shape[0]
    info = getattr(_lib(), f"oracle_{_TC[A.dtype]}_pposv")(side.encode(), uplo.encode(), n, nrhs, A.ctypes.data,
                                                           max(1, A.shape[0]), B.ctypes.data, max(1, B.shape[0]))
    return A, B, int(info)


def diag_logdet(a: np.ndarray, n: int | None = None, lda: int | None = None):
    """Return complex(log magnitude, phase), or raise ValueError for a nonfinite diagonal."""
    A = np.asfortranarray(a)
    n = A.shape[1] if n is None else n
    lda = max(1, A.shape[0]) if lda is None else lda
    out = np.zeros(2, dtype=np.float64)
    st = getattr(_lib(), f"oracle_{_TC[A.dtype]}_diag_logdet")(n, A.ctypes.data, lda, out.ctypes.data)
    if st != 0:
        raise ValueError("diag_logdet: nonfinite diagonal")
    return complex(out[0], out[1])


def gemm_vbatched(ta: str, tb: str, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
    """The variable-size batched GEMM, entry by entry, on host arrays.

    Restates the reference's gemmVbatched (src/BLAS/gemm_vbatched.cpp:349-399) as
    its kernel applies it per entry (src/vbatched/gemm_template_kernel_vbatched.hpp:
    61-85 for the early exits and gemm_template_device.hpp:226-227 for the store),
    with the product of its test's reference_gemm (tests/test_gemm_vbatched.cpp:
    56-90): op(X)(r, c) is X[r + c ld] for 'N', X[c + r ld] for 'T', its conjugate
    for 'C'.  Rules: m or n <= 0 leaves C; k == 0 or alpha == 0 makes C = beta C
    (0 for beta == 0, untouched for beta == 1 or a null C) without reading A or B;
    a null (None) A, B or C leaves C; beta == 0 never reads C.  A, B, C are lists
    of 1-D column-major arrays (or None); returns new arrays for C.
    """
    def view(x, rows, cols, ld):
        return x[:ld * cols].reshape(cols, ld).T[:rows]

    def op(x, t, rows, cols, ld):
        if t in "Nn":
            return view(x, rows, cols, ld)
        s = view(x, cols, rows, ld).T
        return np.conj(s) if t in "Cc" else s

    out = []
    for b in range(len(C)):
        c = None if C[b] is None else C[b].copy()
        out.append(c)
        mb, nb, kb = int(m[b]), int(n[b]), int(k[b])
        if mb <= 0 or nb <= 0:
            continue
        cv = None if c is None else view(c, mb, nb, int(ldc[b]))
        if kb == 0 or alpha == 0:
            if beta == 1 or cv is None:
                continue
            cv[...] = 0 if beta == 0 else beta * cv
            continue
        if A[b] is None or B[b] is None or cv is None:
            continue
        prod = alpha * (op(A[b], ta, mb, kb, int(lda[b])) @ op(B[b], tb, kb, nb, int(ldb[b])))
        cv[...] = prod if beta == 0 else prod + beta * cv
    return out


def gemm_vbatched2s(ops0, m0, n0, k0, alpha0, A0, lda0, B0, ldb0, C0, ldc0,
                    ops1, m1, n1, k1, alpha1, AB1, lda1, ldb1, beta1, C1, ldc1, c0_left, segments):
    """Two dependent variable-size GEMM stages over segments of the batch.

    Restates the reference's gemmVbatched2s (src/BLAS/gemm_vbatched.cpp:420-465,
    src/vbatched/gemm_template_kernel_vbatched.hpp:440-497): segment by segment,
    stage 0 gives C0_b = alpha0 op(A0_b) op(B0_b) (stage-zero beta is zero), then
    stage 1 gives C1_b = alpha1 op(X_b) op(Y_b) + beta1 C1_b with (X, Y) = (C0_b,
    AB1_b) when c0_left, else (AB1_b, C0_b), the C0 operand read with lda1 / ldb1.
    C0 entries are (buffer, offset) pairs so that entries of different segments can
    share temporary storage, as the reference's test does; the buffers are updated
    in place.  Returns the new C1 list.
    """
    out = [None if c is None else c.copy() for c in C1]
    start = 0
    for seg in segments:
        for b in range(start, start + seg):
            buf, off = C0[b]
            t = gemm_vbatched(ops0[0], ops0[1], [m0[b]], [n0[b]], [k0[b]], alpha0, [A0[b]], [lda0[b]], [B0[b]],
                              [ldb0[b]], 0, [buf[off:].copy()], [ldc0[b]])[0]
            buf[off:off + t.size] = t
        for b in range(start, start + seg):
            buf, off = C0[b]
            tmp = buf[off:]
            x, y = (tmp, AB1[b]) if c0_left else (AB1[b], tmp)
            out[b] = gemm_vbatched(ops1[0], ops1[1], [m1[b]], [n1[b]], [k1[b]], alpha1, [x], [lda1[b]], [y],
                                   [ldb1[b]], beta1, [out[b]], [ldc1[b]])[0]
        start += seg
    return out


def herm_complete(a: np.ndarray, uplo: str, n: int) -> None:
    """In place: the leading n x n becomes Hermitian from its uplo triangle, with a
    real diagonal (the reference's herm_complete, used by phegst.cpp:140-176)."""
    if n == 0:
        return
    v = a[:n, :n]
    low = uplo.upper() == "L"
    sel = np.tril(v, -1) if low else np.triu(v, 1)
    d = np.real(np.diag(v)).astype(v.dtype)
    v[...] = sel + np.conj(sel.T) + np.diag(d)


def phegst(a: np.ndarray, factor: np.ndarray, uplo: str = "L", n: int | None = None) -> np.ndarray:
    """Type-1 reduction of a Hermitian-definite pair on host arrays (returns a copy).

    Restates the reference's phegst at a 1x1 grid (src/Eigensolver/phegst.cpp:
    140-176, include/ddla/ddla.h:2540-2562): with B = L L^H (uplo 'L') or U^H U
    ('U') held in factor's selected triangle, A is completed to a Hermitian
    matrix from its selected triangle (real diagonal), then A <- op(L)^-1 A and
    A <- A op(L)^-H (op(L) = L, or U^H), and the result is completed again from
    its selected triangle.  Only the selected triangles of A and factor are read;
    rows and columns past n are left as they were.
    """
    from scipy.linalg import solve_triangular

    a = np.array(a, copy=True, order="F")
    n = a.shape[1] if n is None else n
    if n == 0:
        return a
    low = uplo.upper() == "L"
    f = factor[:n, :n]
    L = np.tril(f) if low else np.conj(np.triu(f)).T  # the lower factor, other triangle never read
    hi = np.complex128 if np.iscomplexobj(a) else np.float64
    w = np.array(a[:n, :n], dtype=hi)
    herm_complete(w, uplo, n)
    w = solve_triangular(L.astype(hi), w, lower=True)
    w = np.conj(solve_triangular(L.astype(hi), np.conj(w).T, lower=True)).T
    herm_complete(w, uplo, n)
    a[:n, :n] = w.astype(a.dtype)
    return a


def block_cyclic_local(a: np.ndarray, mb: int, nb: int, pr: int, pc: int, row: int, col: int,
                       rsrc: int = 0, csrc: int = 0) -> np.ndarray:
    """The local matrix rank (row, col) of a pr x pc grid holds of the global matrix a, ScaLAPACK
    block-cyclic with mb x nb blocks from source process (rsrc, csrc): global (i, j) is local
    (i // (mb pr) * mb + i % mb, j // (nb pc) * nb + j % nb) on the rank owning row block i // mb
    and column block j // nb (the index maps of the reference's include/ddla/ddla_desc.h:10-38)."""
    m, n = a.shape
    rows = [i for i in range(m) if (rsrc + i // mb) % pr == row]
    cols = [j for j in range(n) if (csrc + j // nb) % pc == col]
    return np.asfortranarray(a[np.ix_(rows, cols)]) if rows and cols else np.zeros((len(rows), len(cols)), a.dtype)


def diag_log_local_state(local: np.ndarray, n: int, mb: int, nb: int, pr: int, pc: int, row: int, col: int,
                         rsrc: int = 0, csrc: int = 0) -> np.ndarray:
    """One rank's pdiag_logdet state {magnitude, phase, zero, negative parity, nonfinite}: the
    reference's DiagLogTerm over the items of its layout (src/diag_logdet_impl.h:50-94: items walk
    the local rows when pr >= pc, else the local columns; item -> global g -> local entry; entries
    of other ranks contribute nothing), joined in order by DiagLogJoin (:42-48)."""
    along_rows = pr >= pc
    lr, lc = local.shape
    count = 0 if lr == 0 or lc == 0 else (lr if along_rows else lc)
    block, peers = (mb, pr) if along_rows else (nb, pc)
    coord, src = (row, rsrc) if along_rows else (col, csrc)
    offset = (coord - src + peers) % peers
    mag = phase = 0.0
    flags = 0
    for item in range(count):
        g = (item // block * peers + offset) * block + item % block
        if g >= n or (rsrc + g // mb) % pr != row or (csrc + g // nb) % pc != col:
            continue
        v = complex(local[g // (mb * pr) * mb + g % mb, g // (nb * pc) * nb + g % nb])
        x, y = v.real, v.imag
        if not (np.isfinite(x) and np.isfinite(y)):
            t = (0.0, 0.0, 1)
        else:
            ax, ay = abs(x), abs(y)
            hi, lo = max(ax, ay), min(ax, ay)
            if hi == 0:
                t = (0.0, 0.0, 2)
            else:
                m_ = float(np.log(hi) + 0.5 * np.log1p((lo / hi) ** 2))
                t = (m_, 0.0, 4 if x < 0 else 0) if y == 0 else (m_, float(np.arctan2(y, x)), 0)
        mag += t[0]
        phase += t[1]
        flags = ((flags | t[2]) & 3) | ((flags ^ t[2]) & 4)
    return np.array([mag, phase, float(flags & 2 != 0), float(flags & 4 != 0), float(flags & 1 != 0)])
