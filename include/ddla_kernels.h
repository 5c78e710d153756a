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

/* The factorization runs in super-steps of `group` block columns (128 wide; 64
 * for complex double): the diagonal blocks and panels of a super-step are
 * factored on a high-priority look-ahead stream, and the rest of the trailing
 * matrix is updated once per super-step with K = group * block width.
 * ddlak_potrf uses DDLAK_POTRF_GROUP; ddlak_potrf_grouped takes 1 ..
 * DDLAK_POTRF_MAX_GROUP (same results up to rounding). */
#define DDLAK_POTRF_GROUP 8
#define DDLAK_POTRF_MAX_GROUP 8
int ddlak_potrf_grouped(char type, char uplo, int group, int n, void* A, long long lda, int* dinfo, void* stream);

/* A batch of equal-order FP64 matrices (lower), matrix m at A + m*astride, its
 * info at dinfo[m] (zeroed here): the blocked factorization of ddlak_potrf
 * (block columns of 128, no look-ahead), one launch per kernel and block column
 * over the whole batch.  Needs even lda and astride, a 16-byte aligned A and
 * batch <= 65535 (cudaErrorInvalidValue otherwise). */
int ddlak_potrf_batched_f64(int batch, int n, void* A, long long lda, long long astride, int* dinfo, void* stream);

/* L L^T x = b in place for a batch of FP64 factors from ddlak_potrf_batched_f64
 * (order <= 1024, one right-hand side at B + m*bstride); logdet[m] = 2 sum log
 * l_ii when logdet is not null.  A matrix with dinfo[m] != 0 keeps b and gets
 * logdet NaN. */
int ddlak_potrs_batched_f64(int batch, int n, const void* L, long long lda, long long astride, void* B,
                            long long bstride, const int* dinfo, double* logdet, void* stream);

/* In place A <- J A J on the leading n x n (element (i, j) trades places with
 * (n-1-i, n-1-j); J the order-reversing permutation).  With it the bottom-right
 * factorization of src/Cholesky/potrf_bottom_right.cpp:208-256 (A = U U^H or
 * L^H L from the last column; its per-block reverse packing,
 * potrf_bottom_right_transform.cpp:18-47) is ddlak_potrf of the opposite
 * triangle between two swaps.  The opposite triangle and rows n..lda-1 are
 * permuted and restored, never altered. */
int ddlak_reverse_swap(char type, int n, void* A, long long lda, void* stream);

/* Validation pass of the variable-size batched GEMM (the reference's
 * validate_and_max_dimensions, src/BLAS/gemm_vbatched.cpp:72-106): zeroes the
 * four ints at d_summary, then writes summary[0..2] = largest m, n, k and
 * summary[3] = 1 + the index of an entry with a negative size or a leading
 * dimension below max(1, rows of its matrix) (0: all valid).  transA/transB
 * 'N', 'T', 'C' in either case. */
int ddlak_gemm_vbatched_check(char transA, char transB, const int* d_m, const int* d_n, const int* d_k,
                              const int* d_lda, const int* d_ldb, const int* d_ldc, int batch, int* d_summary,
                              void* stream);

/* C_b = alpha op(A_b) op(B_b) + beta C_b for b < batch (the reference's
 * gemm_vbatched core, src/BLAS/gemm_vbatched.cpp:162-219 and
 * src/vbatched/gemm_template_kernel_vbatched.hpp): type 's' 'd' 'c' 'z';
 * alpha/beta point to one host scalar of that type; max_m/max_n bound every
 * entry's m and n (from ddlak_gemm_vbatched_check).  Entries with m or n of
 * 0 are untouched; k == 0 or alpha == 0 gives C = beta C (C = 0 for beta == 0,
 * C unchanged for beta == 1) without reading A or B; a null A, B or C skips
 * the entry; beta == 0 never reads C. */
int ddlak_gemm_vbatched(char type, char transA, char transB, int max_m, int max_n, const int* d_m, const int* d_n,
                        const int* d_k, const void* alpha, const void* d_A, const int* d_lda, const void* d_B,
                        const int* d_ldb, const void* beta, void* d_C, const int* d_ldc, int batch, void* stream);

/* The mixed form of ddlak_gemm_vbatched: type 'c' or 'z' is the output's
 * type; complex_left = 1: A complex and B real, 0: A real and B complex ('C' on
 * the real operand is 'T').  alpha and beta are complex host scalars. */
int ddlak_gemm_vbatched_mixed(char type, int complex_left, char transA, char transB, int max_m, int max_n,
                              const int* d_m, const int* d_n, const int* d_k, const void* alpha, const void* d_A,
                              const int* d_lda, const void* d_B, const int* d_ldb, const void* beta, void* d_C,
                              const int* d_ldc, int batch, void* stream);

/* Zeroes *d_bad, then sets it to 1 + the index of an entry with m, n > 0 whose
 * product (alpha != 0 and k != 0) needs a null A or B, or whose C is null while
 * it must be written (a product, or beta != 1); the reference's
 * mixed_vbatched_pointer_check (src/BLAS/gemm_mixed.cpp:224-234). */
int ddlak_gemm_vbatched_pointers(const int* d_m, const int* d_n, const int* d_k, const void* const* d_A,
                                 const void* const* d_B, void* const* d_C, int alpha_zero, int beta_one, int batch,
                                 int* d_bad, void* stream);

/* Zeroes *d_bad, then sets it to 1 + the index of an entry (m1, n1, k1 > 0)
 * whose C0 operand in stage 1 of a two-stage GEMM -- rows x cols of op(X) read
 * with leading dimension ld1, X on the left when left != 0, transposed when
 * trans != 0 -- is not the m0 x n0 matrix with leading dimension ldc0 that
 * stage 0 writes (the reference's mixed_vbatched_stage_check,
 * src/BLAS/gemm_mixed.cpp:236-245). */
int ddlak_gemm_vbatched_footprint(const int* d_m0, const int* d_n0, const int* d_ldc0, const int* d_m1,
                                  const int* d_n1, const int* d_k1, const int* d_ld1, int left, int trans, int batch,
                                  int* d_bad, void* stream);

/* Hermitian completion of the leading n x n (the reference's herm_complete):
 * the triangle opposite uplo becomes the conjugate transpose of the uplo one and
 * the diagonal's imaginary part is zeroed.  type 's' 'd' 'c' 'z'. */
int ddlak_herm_complete(char type, char uplo, int n, void* A, long long lda, void* stream);

/* The forward half of ddlak_potrs: B <- L^-1 B (side 'L', B n x nrhs) or
 * B <- B L^-H (side 'R', B nrhs x n), the factor read through its L view
 * (uplo 'L': A's lower triangle; 'U': L = U^H).  Scratch and status word as for
 * ddlak_potrs (ddlak_potrs_workspace(n, nrhs) bytes).  Replaces the two
 * blas_impl::trsm_run calls of phegst (src/Eigensolver/phegst.cpp:145-152). */
int ddlak_forward_solve(char type, char uplo, char side, int n, int nrhs, const void* A, long long lda, void* B,
                        long long ldb, void* work, unsigned long long work_bytes, void* stream);

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

/* ddlak_potrs with its scratch in a fixed device array owned by the library
 * instead of caller memory: no allocation of any kind.  Limits (n <= 65536,
 * nrhs <= 256) are reported by ddlak_potrs_fixed_scratch_limits; larger
 * problems return cudaErrorInvalidValue before touching the device.  The first
 * call on a device looks the array's device address up (with that device
 * current), so it should come before any stream capture.  Every call shares the
 * array: calls that overlap on the GPU race.  *status_word receives the device
 * address of the status word (nonzero after the launch: a wait gave up). */
int ddlak_potrs_fixed_scratch_limits(int* max_n, int* max_nrhs);
int ddlak_potrs_fixed_scratch(char type, char uplo, char side, int n, int nrhs, const void* A, long long lda,
                              void* B, long long ldb, int** status_word, void* stream);

/* Bytes of device scratch ddlak_diag_logsum needs. */
unsigned long long ddlak_logdet_workspace(void);

/* Sum of log|a_ii| and arg(a_ii) over i < n with zero / nonfinite / negative
 * parity flags, the reduction of src/diag_logdet_kernels.cpp:13-25.  Leaves
 * {double magnitude; double phase; int flags} at the start of work. */
int ddlak_diag_logsum(char type, int n, const void* A, long long lda, void* work, void* stream);

/* The same partial state over the diagonal entries that rank (row, col) of a
 * pr x pc block-cyclic grid holds in its local matrix A (leading dimension lld,
 * local_rows x local_cols; blocks mb x nb, source process (rsrc, csrc)), with
 * the reference's item -> global-index mapping (src/diag_logdet_impl.h:55-74,
 * src/PBLAS/pdiag_logdet.cpp:26-37).  Summing the ranks' states and finishing
 * gives pdiag_logdet of the distributed matrix. */
int ddlak_diag_logsum_grid(char type, int n, const void* A, long long lld, int local_rows, int local_cols, int mb,
                           int nb, int pr, int pc, int row, int col, int rsrc, int csrc, void* work, void* stream);

/* ---- mixed precision (ddla::pposv_mixed; no reference counterpart) ------ */

/* Super-steps of the mixed factorization: block columns of 128 factored on the
 * look-ahead chain before one K = 128 * group trailing update of the rest
 * (ddlak_potrf_mixed uses DDLAK_MIXED_GROUP; ddlak_potrf_mixed_grouped takes
 * 1 .. DDLAK_MIXED_MAX_GROUP). */
#define DDLAK_MIXED_GROUP 4
#define DDLAK_MIXED_MAX_GROUP 8

/* Bytes of one of the two panel-operand slots of an order-n factorization
 * (enough for any group up to DDLAK_MIXED_MAX_GROUP). */
unsigned long long ddlak_mixed_panel_bytes(int n);

/* Host-side view of the factorization's update of a whole trailing region of t
 * tile rows (tiles of 128) (no device work): *kind = 2 when it runs by 256 x 256
 * blocks on CTA pairs, 1 by pairs of tiles of one tile row, 0 by single tiles,
 * and *ctas the size of its grid.  For kinds 1 and 2, CTA c decoded to the C tiles
 * it writes: tile row *row, tile columns *col0 .. *col0 + *ntiles - 1.  For tests
 * of the launch's coverage of the lower triangle. */
int ddlak_mixed_update_grid(int t, int* kind, long long* ctas);
int ddlak_mixed_update_cta_tiles(int t, long long c, long long* row, long long* col0, int* ntiles);

/* W = fl32(A) on the lower triangle (diagonal times diag_scale, a relative
 * shift), colsum[j] = sum_i |A(i,j)| of the full symmetric A, *anrm = max_j
 * colsum[j] (= ||A||_inf), all on the stream.  ldw must be a multiple of 4. */
int ddlak_convert_lower(int n, const void* A, long long lda, void* W, long long ldw, double diag_scale, void* colsum,
                        void* anrm, void* stream);

/* Cholesky of the FP32 matrix W (lower) with tensor-core trailing updates:
 * precision 'B' (BF16 operands) or 'T' (TF32 operands), FP32 accumulation,
 * FP64 diagonal blocks.  P0/P1: two buffers of ddlak_mixed_panel_bytes(n).
 * *dinfo as ddlak_potrf; *status nonzero if a tensor-core pipeline wait gave up.
 * The strictly upper triangle of W's leading n x n is used as scratch (the
 * update writes whole 128 x 128 tiles); ldw must be a multiple of 4. */
int ddlak_potrf_mixed(char precision, int n, void* W, long long ldw, void* P0, void* P1, int* dinfo, int* status,
                      void* stream);
/* The same with an explicit super-step group (1 .. DDLAK_MIXED_MAX_GROUP): the
 * trailing matrix is read and written once per `group` block columns. */
int ddlak_potrf_mixed_grouped(char precision, int group, int n, void* W, long long ldw, void* P0, void* P1,
                              int* dinfo, int* status, void* stream);

/* Inverses (FP64) of the 64 x 64 diagonal blocks of an FP32 factor (lower):
 * ddlak_inv_diag_bytes(n) bytes, one column-major block per block row. */
/* Left-looking mixed factorization fed from host memory: the lower part of A
 * (A_host, leading dimension lda_host) goes to A (device, lda) in column panels
 * of 128 * group columns on copy_stream, and on stream each panel is converted
 * to W (FP32), updated from every earlier column at once, factored and appended
 * to Lk, the K-contiguous low-precision copy of L (ldk elements per row, from
 * ddlak_mixed_lk_bytes; TF32 in FP32 words, or BF16).  colsum (n doubles) and
 * anrm receive ||A||_inf as ddlak_convert_lower's do; dinfo / status as
 * ddlak_potrf_mixed's.  Pinned host memory gives the overlap. */
unsigned long long ddlak_mixed_lk_bytes(char precision, int n, long long* ldk);
int ddlak_potrf_mixed_stream(char precision, int group, int n, const void* A_host, long long lda_host, void* A,
                             long long lda, void* W, long long ldw, void* Lk, long long ldk, void* colsum, void* anrm,
                             int* dinfo, int* status, void* copy_stream, void* stream);

unsigned long long ddlak_inv_diag_bytes(int n);
int ddlak_inv_diag_blocks(int n, const void* L32, long long ldl, void* Dinv, void* stream);

/* In-place solve L L^T X = B with an FP32 factor (lower, ldl) and FP64 B;
 * scratch as ddlak_potrs_workspace(n, nrhs).  Dinv (may be NULL) holds the
 * inverted diagonal blocks; with it the diagonal steps are products. */
int ddlak_potrs_mixed(int n, int nrhs, const void* L32, long long ldl, const void* Dinv, void* B, long long ldb,
                      void* work, unsigned long long work_bytes, void* stream);

/* Refinement solves by inverted diagonal super-blocks of order ddlak_bis_block()
 * (1024): ddlak_bis_inverse writes the FP64 inverses of the diagonal blocks of
 * an FP32 factor (ddlak_bis_inverse_bytes(n) bytes, one BS x BS block per
 * super-block, the strictly lower part mirrored into the upper half; tmp is
 * scratch of the same size); ddlak_bis_inverse_narrow rounds them to FP32
 * (half the bytes).  ddlak_bis_solve solves L L^T X = B in place (FP64 B,
 * nrhs <= 16, ldl a multiple of 4, L and Dinv 16-byte aligned) with FP64
 * arithmetic and the FP64 inverses; ddlak_bis_solve_f32 with FP32 arithmetic
 * and the FP32 inverses (the single-precision solve of ?sposv).  Each is one
 * persistent launch per 8 right-hand sides over the n/BS diagonal-block
 * products and streaming panel updates of both directions; if one of its
 * bounded waits gives up, X is NaN.  Scratch: ddlak_bis_solve_workspace(n,
 * nrhs) for either. */
int ddlak_bis_block(void);
unsigned long long ddlak_bis_inverse_bytes(int n);
int ddlak_bis_inverse(int n, const void* L32, long long ldl, void* Dinv, void* tmp, void* stream);
int ddlak_bis_inverse_narrow(int n, const void* Dinv, void* Dinv32, void* stream);
/* The same inverse blocks from an FP64 factor (lower, even ldl), read in place. */
int ddlak_bis_inverse_f64(int n, const void* L, long long ldl, void* Dinv, void* stream);
unsigned long long ddlak_bis_solve_workspace(int n, int nrhs);
int ddlak_bis_solve(int n, int nrhs, const void* L32, long long ldl, const void* Dinv, void* B, long long ldb,
                    void* work, unsigned long long work_bytes, void* stream);
/* L L^T X = B with an FP64 factor (lower, even ldl, 16-byte aligned), FP64 vectors and the
 * FP64 inverse blocks of ddlak_bis_inverse_f64: the FP64 form of the same persistent solve
 * (the plain ppotrs for nrhs <= 16 at large orders). */
int ddlak_bis_solve_f64(int n, int nrhs, const void* L, long long ldl, const void* Dinv, void* B, long long ldb,
                        void* work, unsigned long long work_bytes, void* stream);
int ddlak_bis_solve_f32(int n, int nrhs, const void* L32, long long ldl, const void* Dinv32, void* B, long long ldb,
                        void* work, unsigned long long work_bytes, void* stream);
/* Host-side view of that solve's unit queue (no device work): the number of
 * forward units and of all units for order n, and unit u decoded to its kind
 * (0 forward diagonal slice, 1 forward panel slice, 2 backward diagonal slice,
 * 3 backward panel slice, 4 forward bulk panel, 5 backward bulk panel), phase
 * (diagonal block), index (64-row part, row tile or column tile) and 256-wide
 * slice of the inner dimension.  For tests of the queue's ordering rules. */
int ddlak_bis_queue_size(int n, long long* forward_units, long long* total_units);
int ddlak_bis_queue_unit(int n, long long u, int* kind, int* phase, int* index, int* slice);

/* R = B - A X, A symmetric FP64 stored in its lower triangle, each lower tile read once
 * (atomics fold the partial products into R: its last bits depend on their order). */
int ddlak_symm_residual(int n, int nrhs, const void* A, long long lda, const void* X, long long ldx, const void* B,
                        long long ldb, void* R, long long ldr, void* stream);

/* out[j] = max_i |M(i,j)|;  Y += alpha X  (FP64, column-major). */
int ddlak_colmax(int n, int ncol, const void* M, long long ld, void* out, void* stream);
int ddlak_axpy(int n, int ncol, double alpha, const void* X, long long ldx, void* Y, long long ldy, void* stream);

/* GMRES helpers on n x ncol column blocks (ld = n), vectors vstride apart:
 * out[i*ncol+c] = <V_i(:,c), w(:,c)>;  w(:,c) -= sum_i coef[i*ncol+c] V_i(:,c);
 * y(:,c) = alpha x(:,c) / sqrt(nrm2[c]) (nrm2 NULL: alpha x). */
int ddlak_multidot(const void* V, long long vstride, int nv, const void* w, int n, int ncol, void* out, void* stream);
int ddlak_multi_axpy(const void* V, long long vstride, int nv, const void* coef, void* w, int n, int ncol,
                     void* stream);
int ddlak_scale_cols(const void* x, void* y, int n, int ncol, double alpha, const void* nrm2, void* stream);

/* ---- batched uneven Cholesky (ddla::posvVbatched; no reference counterpart) ---- */

/* Block-column widths of the kernel's two per-matrix variants (widths[2]) for
 * type 's'/'d' and kernel instance nmax (512 or 1024). */
int ddlak_vbatched_variants(char type, int nmax, int* widths);

/* SMs x resident CTAs of the persistent kernel on the current device (0 on error). */
int ddlak_vbatched_max_grid(char type, int nmax);

/* One persistent launch over batch matrices: d_A[i] (order d_n[i] <= nmax,
 * ld d_lda[i]) factored in place (lower), d_B[i] solved in place when d_B is
 * not NULL, d_logdet[i] = log det, d_info[i] = potrf info.  d_order (may be
 * NULL) is the processing order, d_wsel[i] (may be NULL) the variant of matrix
 * i, d_counters two ints that are zero before the launch and are left zero. */
int ddlak_posv_vbatched(char type, int nmax, int batch, const int* d_n, void* const* d_A, const int* d_lda,
                        void* const* d_B, double* d_logdet, int* d_info, const int* d_order,
                        const unsigned char* d_wsel, int* d_counters, int grid, void* stream);

/* Fills d_A[i] with a diagonally dominant SPD matrix of order d_n[i] and d_B[i]
 * (when not NULL) with ones: the autotuner's synthetic input. */
int ddlak_fill_spd_vbatched(char type, int batch, const int* d_n, void* const* d_A, const int* d_lda,
                            void* const* d_B, void* stream);

/* ---- likelihood adjoint (ddla::cholNll* / gpNll*; no reference counterpart) ----
 * Batches of equal-order problems at fixed element strides; see
 * include/ddla/ddla_batched.h for the formulas. */

/* A = sigma_f^2 exp(-|x_i-x_j|^2/(2 l^2)) + sigma^2 delta_ij (lower triangle);
 * X row-major n x d per problem, theta {l, sigma_f^2, sigma^2} at theta + m*tstride. */
int ddlak_gp_build(char type, int batch, int n, int d, const void* X, long long xstride, const double* theta,
                   int tstride, void* A, long long lda, long long astride, void* stream);

/* W = L^-1 (lower triangle written) for n <= 1024.  FP64 with W apart from L and
 * n > 64: recursive inversion on the FP64 tensor cores, which overwrites W's
 * strictly upper triangle as scratch; otherwise one CTA per matrix (W may be L). */
int ddlak_trtri_batched(char type, int batch, int n, const void* L, long long ldl, long long lstride, void* W,
                        long long ldw, long long wstride, void* stream);

/* W = L^-1 (lower triangle written; above it W is unspecified) for any n: the
 * fused forward substitution of ddlak_potrs on the identity, generated in the
 * kernel, skipping its zero blocks.  Scratch: ddlak_potrs_workspace(n, n);
 * the first int of it is the status word as for ddlak_potrs. */
int ddlak_trtri_blocked(char type, int n, const void* L, long long ldl, void* W, long long ldw, void* work,
                        unsigned long long work_bytes, void* stream);

/* out[m] = sum x_m .* y_m, and out[m] = 2 sum log L_m(i,i), in FP64. */
int ddlak_batched_dot(char type, int batch, int n, const void* x, long long xstride, const void* y,
                      long long ystride, double* out, void* stream);
int ddlak_batched_logdiag(char type, int batch, int n, const void* L, long long ldl, long long lstride, double* out,
                          void* stream);

/* Adjoint contraction on 128 x 128 lower tiles of A^-1 = W^T W (mode bit 2 set: W
 * already holds A^-1).  mode & 1 == 0: grad[m][0..2] = dloss/d{l, sigma_f^2,
 * sigma^2} through per-tile partials (partial: ddlak_adjoint_partial_bytes);
 * mode & 1 == 1: G = 1/2 (A^-1 - alpha alpha^T), dense symmetric. */
unsigned long long ddlak_adjoint_partial_bytes(int batch, int n);
int ddlak_adjoint_contract(char type, int mode, int batch, int n, const void* W, long long ldw, long long wstride,
                           const void* alpha, long long astride, const void* X, int d, long long xstride,
                           const double* theta, int tstride, double* partial, double* grad, void* G, long long ldg,
                           long long gstride, void* stream);

/* Number of kernel launches the layer has made in this process. */
long long ddlak_launch_count(void);

/* Clock budget, in SM cycles, after which a kernel's wait on another CTA's flag
 * gives up: the kernel records DDLAK_WAIT_TIMEOUT (1) in its status word and
 * returns, and the host routine reports the timeout (std::runtime_error in the
 * C++ API, status 6 in the C ABI).  cycles <= 0 restores the default, 4e9
 * (about 2 s at 1.9 GHz).  Applies to the current device for every kernel of
 * the library; synchronous with respect to the device. */
int ddlak_set_wait_budget(long long cycles);
long long ddlak_get_wait_budget(void);

/* Per-kernel CUDA-event timing.  While enabled, every launcher brackets its
 * kernels with events on its stream and records the launch's algorithmic
 * flops and bytes.  ddlak_profile_read waits for the events of one kind
 * (-1 = all kinds; kinds: 0 potrf_diag, 1 trsm_panel, 2 syrk_update,
 * 3 potrs_fused, 4 logdet, 5 mixed_update, 6 mixed_other, 7 symm_residual,
 * 8 batched, 9 adjoint) and returns their total device milliseconds, count,
 * flops and bytes; reset != 0 drops the records it read. */
void ddlak_profile_enable(int on);
int ddlak_profile_read(int kind, double* ms, long long* launches, double* flops, double* bytes, int reset);


/* ---- distributed (P x Q grid) Cholesky and solve: local steps -------------
 * Index map of a block-cyclically distributed dimension: local index l goes to
 * ((L / nb) * nprocs + (coord - src) mod nprocs) * nb + L mod nb - base with
 * L = first + l (ScaLAPACK's local-to-global map, offset); nprocs == 0 is the
 * identity l -> l.  A NULL map is the identity. */
typedef struct {
    int first, coord, src, nprocs, nb;
    long long base;
} ddlak_gmap;

/* C(i,j) = beta C(i,j) + alpha sum_p opA(i,p) opB(p,j) on an m x n C, contraction k,
 * opA(i,p) = A[ma(i) + p lda] ('N') or conj(A[ma(p) + i lda]) ('C'),
 * opB(p,j) = B[mb(p) + j ldb] ('N') or conj(B[mb(j) + p ldb]) ('C'),
 * mask 0: all of C; 1: only where mi(i) >= mj(j); 2: only where mi(i) <= mj(j).
 * alpha, beta: {re, im}; beta NULL writes C without reading it.  The trailing
 * update (herk / gemm / gemmBatched on stored tiles) of src/Cholesky/ppotrf.cpp:196-317
 * and the block updates of src/PBLAS/ptrtrs.cpp:209-224 on a grid. */
int ddlak_grid_gemm(char type, char opA, char opB, int mask, int m, int n, int k, const double* alpha, const void* A,
                    long long lda, const ddlak_gmap* ma, const void* B, long long ldb, const ddlak_gmap* mb,
                    const double* beta, void* C, long long ldc, const ddlak_gmap* mi, const ddlak_gmap* mj,
                    void* stream);
/* dst(i,j) = src(i,j), or conj(src(j,i)) when conj_trans, for i < rows, j < cols. */
int ddlak_grid_pack(char type, int conj_trans, int rows, int cols, const void* src, long long lds, void* dst,
                    long long ldd, void* stream);
/* dst(map(l), c) = src(l, c) for l < rows, c < cols. */
int ddlak_grid_unscatter(char type, int rows, int cols, const void* src, long long lds, void* dst, long long ldd,
                         const ddlak_gmap* map, void* stream);
/* W = I (n x n). */
int ddlak_grid_identity(char type, int n, void* W, long long ldw, void* stream);
/* dst[e] += src[e], e < count reals ('s' float, 'd' double). */
int ddlak_grid_accumulate(char real_type, unsigned long long count, const void* src, void* dst, void* stream);

#ifdef __cplusplus
}
#endif

#endif
