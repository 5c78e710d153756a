/*
 * ddla_oracle.c -- TEST INFRASTRUCTURE ONLY: the CPU oracle that the GPU
 * Cholesky path is checked against.  Nothing in the product links or calls it;
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
 *
 * It restates, in plain C, what the reference computes on a CPU handle over a
 * 1x1 process grid:
 *   ppotrf  -> ?potrf_(uplo, n, A, LLD, info)      src/Cholesky/ppotrf.cpp:39-54,
 *                                                  src/Cholesky/potrf.cpp:41-59
 *   ppotrs  -> ?trsm_(side, uplo, first, 'N', ...) then ?trsm_(..., second, ...)
 *              with first/second from src/Cholesky/ppotrs.cpp:44-48, reached via
 *              src/PBLAS/ptrtrs.cpp:150-155 and src/BLAS/trsm.cpp:137-144
 *   pposv   -> ppotrf, then ppotrs when info == 0  src/Cholesky/pposv.cpp:22-40
 *   potrf_bottom_right -> the blocked loop of src/Cholesky/potrf_bottom_right.cpp:208-256
 *              (128-blocks from the bottom-right corner: reverse-pack the block
 *              onto the opposite triangle, potrf_bottom_right_transform.cpp:18-47,
 *              ?potrf of that triangle, map back, potrf_bottom_right.cpp:77-107;
 *              then ?trsm of the panel and ?syrk/?herk of the leading block,
 *              potrf_bottom_right.cpp:27-56, 233-252)
 *   diag_logdet -> DiagLogTerm / DiagLogJoin / finish_diagonal_log,
 *              src/diag_logdet_impl.h:42-113, summed in index order as the
 *              sequential CPU loop of src/diag_logdet.cpp:12-38 does.
 * ?potrf_ and ?trsm_ are third-party (LAPACK / BLAS, whatever the reference
 * links: OpenBLAS 0.3.20 in its CI); their published reference algorithms are
 * restated here: ?potf2 (unblocked, dot-product form, info = first j with
 * a_jj <= 0 or NaN, a_jj left holding the failed value) and the reference
 * BLAS ?trsm loops for alpha = 1.  Arithmetic is in the storage precision, as
 * LAPACK's is.
 */
#include <complex.h>
#include <float.h>
#include <math.h>
#include <stddef.h>
#include <stdlib.h>

#define IDX(i, j, ld) ((size_t)(i) + (size_t)(j) * (size_t)(ld))

#define RCONJ(x) (x)
#define CCONJF(x) conjf(x)
#define CCONJ(x) conj(x)
#define RREAL(x) (x)
#define CREALF(x) crealf(x)
#define CREAL(x) creal(x)

/* P: prefix, T: storage type, R: real type, CONJ/REAL: helpers, SQRT: real sqrt */
#define DEFINE_ORACLE(P, T, R, CONJ, REAL, SQRT)                                                            \
    int oracle_##P##_potrf(char uplo, int n, T* A, int lda)                                                 \
    {                                                                                                       \
        int i, j, k;                                                                                        \
        if (n <= 0) return 0;                                                                               \
        if (uplo == 'U' || uplo == 'u') {                                                                   \
            /* A = U^H U, column by column (dpotf2, UPLO = 'U') */                                          \
            for (j = 0; j < n; ++j) {                                                                       \
                T dot = 0;                                                                                  \
                R ajj;                                                                                      \
                for (k = 0; k < j; ++k) dot += CONJ(A[IDX(k, j, lda)]) * A[IDX(k, j, lda)];                 \
                ajj = REAL(A[IDX(j, j, lda)]) - REAL(dot);                                                  \
                if (!(ajj > 0)) { A[IDX(j, j, lda)] = ajj; return j + 1; }                                   \
                ajj = SQRT(ajj);                                                                            \
                A[IDX(j, j, lda)] = ajj;                                                                    \
                for (i = j + 1; i < n; ++i) {                                                               \
                    T s = A[IDX(j, i, lda)];                                                                \
                    for (k = 0; k < j; ++k) s -= CONJ(A[IDX(k, j, lda)]) * A[IDX(k, i, lda)];               \
                    A[IDX(j, i, lda)] = s / ajj;                                                            \
                }                                                                                           \
            }                                                                                               \
        } else {                                                                                            \
            /* A = L L^H, row-oriented dot products (dpotf2, UPLO = 'L') */                                 \
            for (j = 0; j < n; ++j) {                                                                       \
                T dot = 0;                                                                                  \
                R ajj;                                                                                      \
                for (k = 0; k < j; ++k) dot += A[IDX(j, k, lda)] * CONJ(A[IDX(j, k, lda)]);                 \
                ajj = REAL(A[IDX(j, j, lda)]) - REAL(dot);                                                  \
                if (!(ajj > 0)) { A[IDX(j, j, lda)] = ajj; return j + 1; }                                   \
                ajj = SQRT(ajj);                                                                            \
                A[IDX(j, j, lda)] = ajj;                                                                    \
                for (i = j + 1; i < n; ++i) {                                                               \
                    T s = A[IDX(i, j, lda)];                                                                \
                    for (k = 0; k < j; ++k) s -= A[IDX(i, k, lda)] * CONJ(A[IDX(j, k, lda)]);               \
                    A[IDX(i, j, lda)] = s / ajj;                                                            \
                }                                                                                           \
            }                                                                                               \
        }                                                                                                   \
        return 0;                                                                                           \
    }                                                                                                       \
                                                                                                            \
    /* op(A) X = B (side 'L') or X op(A) = B (side 'R'), A triangular, alpha = 1, diag 'N';                \
       trans 'N' or 'C' ('T' equals 'C' for real types).  Reference BLAS ?trsm loop order. */              \
    void oracle_##P##_trsm(char side, char uplo, char trans, int m, int n, const T* A, int lda, T* B,      \
                           int ldb)                                                                         \
    {                                                                                                       \
        int i, j, k;                                                                                        \
        const int lower = (uplo == 'L');                                                                    \
        const int notr = (trans == 'N');                                                                    \
        if (m <= 0 || n <= 0) return;                                                                       \
        if (side == 'L') {                                                                                  \
            if (notr) {                                                                                     \
                if (!lower) { /* U X = B: back substitution */                                              \
                    for (j = 0; j < n; ++j)                                                                 \
                        for (k = m - 1; k >= 0; --k)                                                        \
                            if (B[IDX(k, j, ldb)] != 0) {                                                   \
                                B[IDX(k, j, ldb)] /= A[IDX(k, k, lda)];                                     \
                                for (i = 0; i < k; ++i) B[IDX(i, j, ldb)] -= B[IDX(k, j, ldb)] * A[IDX(i, k, lda)]; \
                            }                                                                               \
                } else { /* L X = B */                                                                      \
                    for (j = 0; j < n; ++j)                                                                 \
                        for (k = 0; k < m; ++k)                                                             \
                            if (B[IDX(k, j, ldb)] != 0) {                                                   \
                                B[IDX(k, j, ldb)] /= A[IDX(k, k, lda)];                                     \
                                for (i = k + 1; i < m; ++i) B[IDX(i, j, ldb)] -= B[IDX(k, j, ldb)] * A[IDX(i, k, lda)]; \
                            }                                                                               \
                }                                                                                           \
            } else {                                                                                        \
                if (!lower) { /* U^H X = B */                                                               \
                    for (j = 0; j < n; ++j)                                                                 \
                        for (i = 0; i < m; ++i) {                                                           \
                            T t = B[IDX(i, j, ldb)];                                                        \
                            for (k = 0; k < i; ++k) t -= CONJ(A[IDX(k, i, lda)]) * B[IDX(k, j, ldb)];       \
                            B[IDX(i, j, ldb)] = t / CONJ(A[IDX(i, i, lda)]);                                \
                        }                                                                                   \
                } else { /* L^H X = B */                                                                    \
                    for (j = 0; j < n; ++j)                                                                 \
                        for (i = m - 1; i >= 0; --i) {                                                      \
                            T t = B[IDX(i, j, ldb)];                                                        \
                            for (k = i + 1; k < m; ++k) t -= CONJ(A[IDX(k, i, lda)]) * B[IDX(k, j, ldb)];   \
                            B[IDX(i, j, ldb)] = t / CONJ(A[IDX(i, i, lda)]);                                \
                        }                                                                                   \
                }                                                                                           \
            }                                                                                               \
        } else {                                                                                            \
            if (notr) {                                                                                     \
                if (!lower) { /* X U = B */                                                                 \
                    for (j = 0; j < n; ++j) {                                                               \
                        for (k = 0; k < j; ++k)                                                             \
                            if (A[IDX(k, j, lda)] != 0)                                                     \
                                for (i = 0; i < m; ++i) B[IDX(i, j, ldb)] -= A[IDX(k, j, lda)] * B[IDX(i, k, ldb)]; \
                        for (i = 0; i < m; ++i) B[IDX(i, j, ldb)] /= A[IDX(j, j, lda)];                     \
                    }                                                                                       \
                } else { /* X L = B */                                                                      \
                    for (j = n - 1; j >= 0; --j) {                                                          \
                        for (k = j + 1; k < n; ++k)                                                         \
                            if (A[IDX(k, j, lda)] != 0)                                                     \
                                for (i = 0; i < m; ++i) B[IDX(i, j, ldb)] -= A[IDX(k, j, lda)] * B[IDX(i, k, ldb)]; \
                        for (i = 0; i < m; ++i) B[IDX(i, j, ldb)] /= A[IDX(j, j, lda)];                     \
                    }                                                                                       \
                }                                                                                           \
            } else {                                                                                        \
                if (!lower) { /* X U^H = B */                                                               \
                    for (k = n - 1; k >= 0; --k) {                                                          \
                        const T d = CONJ(A[IDX(k, k, lda)]);                                                \
                        for (i = 0; i < m; ++i) B[IDX(i, k, ldb)] /= d;                                     \
                        for (j = 0; j < k; ++j) {                                                           \
                            const T t = CONJ(A[IDX(j, k, lda)]);                                            \
                            if (t != 0)                                                                     \
                                for (i = 0; i < m; ++i) B[IDX(i, j, ldb)] -= t * B[IDX(i, k, ldb)];         \
                        }                                                                                   \
                    }                                                                                       \
                } else { /* X L^H = B */                                                                    \
                    for (k = 0; k < n; ++k) {                                                               \
                        const T d = CONJ(A[IDX(k, k, lda)]);                                                \
                        for (i = 0; i < m; ++i) B[IDX(i, k, ldb)] /= d;                                     \
                        for (j = k + 1; j < n; ++j) {                                                       \
                            const T t = CONJ(A[IDX(j, k, lda)]);                                            \
                            if (t != 0)                                                                     \
                                for (i = 0; i < m; ++i) B[IDX(i, j, ldb)] -= t * B[IDX(i, k, ldb)];         \
                        }                                                                                   \
                    }                                                                                       \
                }                                                                                           \
            }                                                                                               \
        }                                                                                                   \
    }                                                                                                       \
                                                                                                            \
    /* ppotrs_run on a 1x1 grid: src/Cholesky/ppotrs.cpp:40-61 */                                           \
    void oracle_##P##_ppotrs(char side, char uplo, int n, int nrhs, const T* A, int lda, T* B, int ldb)    \
    {                                                                                                       \
        const int left = (side == 'L');                                                                     \
        const char first = (left == (uplo == 'L')) ? 'N' : 'C';                                             \
        const char second = (left == (uplo == 'L')) ? 'C' : 'N';                                            \
        const int rows = left ? n : nrhs, cols = left ? nrhs : n;                                           \
        if (n == 0 || nrhs == 0) return;                                                                    \
        oracle_##P##_trsm(side, uplo, first, rows, cols, A, lda, B, ldb);                                   \
        oracle_##P##_trsm(side, uplo, second, rows, cols, A, lda, B, ldb);                                  \
    }                                                                                                       \
                                                                                                            \
    /* pposv_run on a 1x1 grid: src/Cholesky/pposv.cpp:22-40 */                                             \
    int oracle_##P##_pposv(char side, char uplo, int n, int nrhs, T* A, int lda, T* B, int ldb)            \
    {                                                                                                       \
        int info = oracle_##P##_potrf(uplo, n, A, lda);                                                     \
        if (info == 0) oracle_##P##_ppotrs(side, uplo, n, nrhs, A, lda, B, ldb);                            \
        return info;                                                                                        \
    }                                                                                                       \
                                                                                                            \
    /* A = U U^H ('U') or L^H L ('L') from the bottom-right corner.  Returns info: 0, or           \
       block_start + block_n - solver_info + 1 for the first block whose ?potrf fails (that block is \
       left as it was, the loop stops), potrf_bottom_right.cpp:89-99, 224-226. */                     \
    int oracle_##P##_potrf_bottom_right(char uplo, int n, T* A, int lda)                                    \
    {                                                                                                       \
        const int NB = 128;                                                                                 \
        const int upper = (uplo == 'U');                                                                    \
        int b0, r, c, i, j, k, info = 0;                                                                    \
        T* work;                                                                                            \
        if (n <= 0) return 0;                                                                               \
        work = (T*)malloc(sizeof(T) * (size_t)NB * NB);                                                     \
        if (!work) return -1;                                                                               \
        for (b0 = ((n - 1) / NB) * NB; b0 >= 0; b0 -= NB) {                                                 \
            const int bn = (n - b0) < NB ? (n - b0) : NB;                                                   \
            T* D = A + IDX(b0, b0, lda);                                                                    \
            int si;                                                                                         \
            for (c = 0; c < bn; ++c) /* the selected triangle, reversed, onto the opposite one of work */ \
                for (r = 0; r < bn; ++r)                                                                    \
                    if (upper ? r >= c : r <= c) work[IDX(r, c, bn)] = D[IDX(bn - 1 - r, bn - 1 - c, lda)]; \
            si = oracle_##P##_potrf(upper ? 'L' : 'U', bn, work, bn);                                       \
            if (si != 0) { info = b0 + bn - si + 1; break; }                                                \
            for (c = 0; c < bn; ++c)                                                                        \
                for (r = 0; r < bn; ++r)                                                                    \
                    if (upper ? r <= c : r >= c) D[IDX(r, c, lda)] = work[IDX(bn - 1 - r, bn - 1 - c, bn)]; \
            if (b0 == 0) continue;                                                                          \
            if (upper) {                                                                                    \
                T* Pn = A + IDX(0, b0, lda); /* b0 x bn: Pn := Pn inv(D^H), then A00 -= Pn Pn^H (upper) */  \
                oracle_##P##_trsm('R', 'U', 'C', b0, bn, D, lda, Pn, lda);                                  \
                for (j = 0; j < b0; ++j)                                                                    \
                    for (i = 0; i <= j; ++i) {                                                              \
                        T s = 0;                                                                            \
                        for (k = 0; k < bn; ++k) s += Pn[IDX(i, k, lda)] * CONJ(Pn[IDX(j, k, lda)]);        \
                        A[IDX(i, j, lda)] -= s;                                                             \
                        if (i == j) A[IDX(i, j, lda)] = REAL(A[IDX(i, j, lda)]);                            \
                    }                                                                                       \
            } else {                                                                                        \
                T* Pn = A + IDX(b0, 0, lda); /* bn x b0: Pn := inv(D^H) Pn, then A00 -= Pn^H Pn (lower) */  \
                oracle_##P##_trsm('L', 'L', 'C', bn, b0, D, lda, Pn, lda);                                  \
                for (j = 0; j < b0; ++j)                                                                    \
                    for (i = j; i < b0; ++i) {                                                              \
                        T s = 0;                                                                            \
                        for (k = 0; k < bn; ++k) s += CONJ(Pn[IDX(k, i, lda)]) * Pn[IDX(k, j, lda)];        \
                        A[IDX(i, j, lda)] -= s;                                                             \
                        if (i == j) A[IDX(i, j, lda)] = REAL(A[IDX(i, j, lda)]);                            \
                    }                                                                                       \
            }                                                                                               \
        }                                                                                                   \
        free(work);                                                                                         \
        return info;                                                                                        \
    }                                                                                                       \
                                                                                                            \
    /* DiagLogTerm + DiagLogJoin over i < n, then finish_diagonal_log.  Returns 1 (nonfinite: the         \
       reference throws domain_error and leaves the result untouched) or 0 with out[0] = log magnitude,    \
       out[1] = phase in (-pi, pi]. */                                                                      \
    int oracle_##P##_diag_logdet(int n, const T* A, int lda, double* out)                                   \
    {                                                                                                       \
        double magnitude = 0, phase = 0;                                                                    \
        int flags = 0, negative = 0, i;                                                                     \
        for (i = 0; i < n; ++i) {                                                                           \
            const R* d = (const R*)(A + IDX(i, i, lda));                                                    \
            const double x = (double)d[0];                                                                  \
            const double y = sizeof(T) == 2 * sizeof(R) ? (double)d[1] : 0.0;                               \
            const double lim = DBL_MAX;                                                                     \
            double ax, ay, hi, lo, ratio;                                                                   \
            if (!(x <= lim && x >= -lim && y <= lim && y >= -lim)) { flags |= 1; continue; }                \
            ax = fabs(x); ay = fabs(y);                                                                     \
            hi = ax > ay ? ax : ay; lo = ax > ay ? ay : ax;                                                 \
            if (hi == 0) { flags |= 2; continue; }                                                          \
            ratio = lo / hi;                                                                                \
            magnitude += log(hi) + 0.5 * log1p(ratio * ratio);                                              \
            if (y == 0) { if (x < 0) negative ^= 4; continue; }                                             \
            phase += atan2(y, x);                                                                           \
        }                                                                                                   \
        flags |= negative;                                                                                  \
        if (flags & 1) return 1;                                                                            \
        if (flags & 2) { out[0] = -INFINITY; out[1] = 0; return 0; }                                        \
        {                                                                                                   \
            const double pi = acos(-1.0);                                                                   \
            phase = remainder(phase + ((flags >> 2) & 1) * pi, 2 * pi);                                     \
            if (phase <= -pi) phase = pi;                                                                   \
            out[0] = (double)(R)magnitude;                                                                  \
            out[1] = (double)(R)phase;                                                                      \
        }                                                                                                   \
        return 0;                                                                                           \
    }

DEFINE_ORACLE(s, float, float, RCONJ, RREAL, sqrtf)
DEFINE_ORACLE(d, double, double, RCONJ, RREAL, sqrt)
DEFINE_ORACLE(c, float _Complex, float, CCONJF, CREALF, sqrtf)
DEFINE_ORACLE(z, double _Complex, double, CCONJ, CREAL, sqrt)
