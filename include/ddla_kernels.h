/*
 * ddla_kernels.h -- the thin C-ABI kernel layer under the ddla C++ API.
 *
 * The C++ host code (ddla::ppotrf, ppotrs, pposv, potrf, diag_logdet and the
 * mixed-precision / batched / adjoint additions) validates arguments, carves
 * workspace and reports info; every device computation it needs goes through
 * one of these entry points.  They take plain pointers, sizes and a CUDA
 * stream as void*, enqueue hand-written sm_100a kernels on that stream and
 * return a cudaError_t value (0 = success).  Nothing here synchronises.
 *
 * Type codes: 's' float, 'd' double, 'c' complex<float>, 'z' complex<double>
 * (interleaved re/im, the layout of std::complex).  Matrices are column-major.
 * uplo 'L' addresses A = L*L^H in the lower triangle, 'U' A = U^H*U in the
 * upper triangle; the opposite triangle is never read or written.
 */
#ifndef DDLA_KERNELS_H
#define DDLA_KERNELS_H

#ifdef __cplusplus
extern "C" {
#endif

/* Blocked Cholesky of the leading n x n of A (lda >= n) on the stream.
 * Replaces cusolverDn?potrf at src/Cholesky/potrf.cpp:106-113 (reached from
 * ppotrf_run, src/Cholesky/ppotrf.cpp:39-54).  *dinfo (device int) is set to 0
 * and then to the order of the first non-positive-definite leading minor. */
int ddlak_potrf(char type, char uplo, int n, void* A, long long lda, int* dinfo, void* stream);

/* Bytes of device scratch ddlak_potrs needs for (n, nrhs). */
unsigned long long ddlak_potrs_workspace(int n, int nrhs);

/* Solve A*X = B (side 'L', B n x nrhs) or X*A = B (side 'R', B nrhs x n) with
 * the Cholesky factor held in A (uplo as above), in place in B.  Replaces the
 * two cublas?trsm calls of ppotrs_run (src/Cholesky/ppotrs.cpp:44-61 ->
 * src/PBLAS/ptrtrs.cpp:150-155 -> src/BLAS/trsm.cpp:154-159).  The first int
 * of the scratch is a status word: nonzero after the launch means a device
 * wait gave up (1 = timeout) and B is incomplete. */
int ddlak_potrs(char type, char uplo, char side, int n, int nrhs, const void* A, long long lda, void* B,
                long long ldb, void* work, unsigned long long work_bytes, void* stream);

/* Bytes of device scratch ddlak_diag_logsum needs. */
unsigned long long ddlak_logdet_workspace(void);

/* Sum of log|a_ii| and arg(a_ii) over i < n with zero / nonfinite / negative
 * parity flags, the reduction of src/diag_logdet_kernels.cpp:13-25.  Leaves
 * {double magnitude; double phase; int flags} at the start of work. */
int ddlak_diag_logsum(char type, int n, const void* A, long long lda, void* work, void* stream);

/* Number of kernel launches the layer has made in this process. */
long long ddlak_launch_count(void);

/* Per-kernel CUDA-event timing.  While enabled, every launcher brackets its
 * kernels with events on its stream and records the launch's algorithmic
 * flops and bytes.  ddlak_profile_read waits for the events of one kind
 * (-1 = all kinds; kinds: 0 potrf_diag, 1 trsm_panel, 2 syrk_update,
 * 3 potrs_fused, 4 logdet, 5 mixed_update, 6 mixed_other, 7 symm_residual,
 * 8 batched, 9 adjoint) and returns their total device milliseconds, count,
 * flops and bytes; reset != 0 drops the records it read. */
void ddlak_profile_enable(int on);
int ddlak_profile_read(int kind, double* ms, long long* launches, double* flops, double* bytes, int reset);

#ifdef __cplusplus
}
#endif

#endif
