// ddla C++ API for the Cholesky path on B200.
//
// The five reference templates keep their exact signatures, argument meaning,
// info and exception behaviour (reference include/ddla/ddla.h):
//   ppotrf       1064-1070     ppotrs      1148-1155     pposv   1183-1190
//   potrf        2159-2160     diag_logdet 2900-2902
// Instantiated for float, double, std::complex<float>, std::complex<double>.
// A handle's matrices are device memory; the process grid is 1x1, so the
// descriptor supplies the leading dimension (LLD_) and is validated exactly as
// the reference validates it (src/ddla_desc.cpp:9-59).
//
// Additions beside the reference path (no reference counterpart):
//   pposv_mixed     FP64-accurate solve from a low-precision tensor-core factor
//                   plus iterative refinement / GMRES-IR (LAPACK ?sposv shape);
//   posvVbatched / VbatchedPlan / vbatchedAutotune (batched uneven SPD) and
//   cholNll* / gpNll* (likelihood and its adjoint): see ddla_batched.h.
#ifndef DDLA_H
#define DDLA_H

#include <complex>

#include <ddla/ddla_desc.h>
#include <ddla/ddla_handle_t.h>

namespace ddla {

template <typename T> struct real_type { using type = T; };
template <typename U> struct real_type<std::complex<U>> { using type = U; };
template <typename T> using real_type_t = typename real_type<T>::type;

// A = L*L^H (uplo 'L') or U^H*U ('U') of the leading n x n, in place.  info is
// 0 or the order of the first leading minor that is not positive definite.
// Returns with the handle's stream synchronised.
template <typename T>
void ppotrf(const DdlaHandle_t& handle, char uplo, int n, T* A, int ia, int ja, const int* descA, int& info);

// A*X = B (side 'L', B n x nrhs) or X*A = B (side 'R', B nrhs x n) with the
// factor from ppotrf; trans 'N' and 'C' are equivalent, 'T' is rejected.
template <typename T>
void ppotrs(const DdlaHandle_t& handle, char side, char uplo, char trans, int n, int nrhs, const T* A,
            const int* descA, T* B, const int* descB);

// ppotrf then, if info == 0, ppotrs.  B is untouched when info != 0.
template <typename T>
void pposv(const DdlaHandle_t& handle, char side, char uplo, char trans, int n, int nrhs, T* A, int ia, int ja,
           const int* descA, T* B, int ib, int jb, const int* descB, int& info);

// LAPACK-style factorization with a DEVICE info pointer; asynchronous.
template <typename T>
void potrf(const DdlaHandle_t& handle, char uplo, int n, T* A, int lda, int* info);

// Cholesky from the bottom-right corner (reference ddla.h:1090-1093, 1117-1121):
// uplo 'U' computes A = U*U^H in the upper triangle, 'L' A = L^H*L in the
// lower one; the other triangle and the padding rows are left as they were.
// info is 0 or the (1-based) index of the first pivot, counted from the bottom,
// that is not positive; A's selected triangle is then unspecified.  Both
// return with the handle's stream synchronised.  potrf_bottom_right throws
// std::runtime_error on a bad argument (potrf_bottom_right.cpp:171-187);
// ppotrf_bottom_right validates the descriptor like ppotrf and throws
// std::invalid_argument (ppotrf_bottom_right.cpp:62-70).
template <typename T>
void potrf_bottom_right(char uplo, int n, T* A, int lda, int& info, const DdlaHandle_t& handle);
template <typename T>
void ppotrf_bottom_right(const DdlaHandle_t& handle, char uplo, int n, T* A, const int* descA, int& info);

// Principal log of prod(A(i,i)), i < n, as (log magnitude, phase in (-pi, pi]).
// Zero diagonal -> (-inf, 0); nonfinite diagonal throws std::domain_error and
// leaves result unchanged.  Completes before returning.
template <typename T>
void diag_logdet(const DdlaHandle_t& handle, int n, const T* A, int lda, std::complex<real_type_t<T>>& result);

// The same through an int[9] descriptor (reference ddla.h:2914-2915,
// src/PBLAS/pdiag_logdet.cpp:11-48): n <= M_, N_, leading dimension LLD_;
// std::invalid_argument for a bad order or a null local matrix.
template <typename T>
void pdiag_logdet(const DdlaHandle_t& handle, int n, const T* A, const int* descA,
                  std::complex<real_type_t<T>>& result);

// pdiag_logdet on a pr x pc grid, split at the reference's one exchange step
// (src/PBLAS/pdiag_logdet.cpp:41-47, an MPI_Allreduce of four doubles): rank
// (row, col) computes state = {magnitude, phase, zero, negative parity,
// nonfinite} over the diagonal entries its local matrix A holds (descA checked
// against the pr x pc grid); the caller sums the five doubles over the ranks
// (any all-reduce) and pdiag_logdet_finish turns the sums into log det, throwing
// std::domain_error on every rank when any rank saw a nonfinite entry.  No
// reference counterpart as separate entry points.
template <typename T>
void pdiag_logdet_local(const DdlaHandle_t& handle, int n, const T* A, const int* descA, int pr, int pc, int row,
                        int col, double state[5]);
void pdiag_logdet_finish(const double total[5], double& re, double& im);

// A batch of GEMMs of differing sizes (reference ddla.h:1836-1849,
// src/BLAS/gemm_vbatched.cpp:349-399): for b < batch_count,
//   C_b = alpha op(A_b) op(B_b) + beta C_b,  op(A_b) d_m[b] x d_k[b],
// with every array device resident.  T is float, double, std::complex<float>
// or std::complex<double>; trans* are 'N', 'T' or 'C' in either case.  A GPU
// handle is required.  std::invalid_argument for: a null or non-GPU handle, a
// negative batch count, a null pointer array, a bad transpose mode, a null
// dimension array, and "gemmVbatched: invalid dimensions at batch <b>" for the
// first entry found with a negative size or a leading dimension below the
// rows of its matrix (the sizes are validated on the device and read back
// once).  An empty batch does nothing.  Per entry: m or n of 0 does nothing;
// k == 0 or alpha == 0 scales C by beta without reading A or B; a null A, B
// or C pointer skips the entry; beta == 0 never reads C.  Enqueued on the
// handle's stream.
template <typename T>
void gemmVbatched(const DdlaHandle_t& handle, char transA, char transB, int* d_m, int* d_n, int* d_k, T alpha,
                  const T* const* d_A_array, int* d_lda, const T* const* d_B_array, int* d_ldb, T beta,
                  T** d_C_array, int* d_ldc, int batch_count);

// One real and one complex operand, complex alpha, beta and output (reference
// ddla.h:1878-1939, src/BLAS/gemm_mixed.cpp:787-870): the rules of gemmVbatched,
// with 'C' on the real operand meaning 'T', and an entry whose product or
// scaling needs a null matrix rejected ("gemmVbatched(mixed): null matrix at
// batch <b>") before anything is written.
template <typename R>
void gemmVbatched(const DdlaHandle_t& handle, char transA, char transB, int* d_m, int* d_n, int* d_k,
                  std::complex<R> alpha, const R* const* d_A_array, int* d_lda,
                  const std::complex<R>* const* d_B_array, int* d_ldb, std::complex<R> beta,
                  std::complex<R>** d_C_array, int* d_ldc, int batch_count);
template <typename R>
void gemmVbatched(const DdlaHandle_t& handle, char transA, char transB, int* d_m, int* d_n, int* d_k,
                  std::complex<R> alpha, const std::complex<R>* const* d_A_array, int* d_lda,
                  const R* const* d_B_array, int* d_ldb, std::complex<R> beta, std::complex<R>** d_C_array,
                  int* d_ldc, int batch_count);

// Two stages with one real and one complex operand somewhere (reference
// ddla.h:1893-2030, src/BLAS/gemm_mixed.cpp:878-994): (A0, B0, C0, AB1) element
// types (R, Z, Z, R), (Z, R, Z, R), (R, Z, Z, Z), (Z, R, Z, Z), (Z, Z, Z, R),
// (R, R, R, Z) with Z = std::complex<R>; C1 is complex.  The rules of
// gemmVbatched2s, the mixed one-stage checks for both stages, and, when
// alpha_1 != 0, "gemmVbatched2s(mixed): incompatible intermediate dimensions"
// unless stage 1 reads C0 as the m0 x n0 matrix with leading dimension ldc0.
#define DDLA_GEMM_VBATCHED2S_MIXED(TA, TB, T0, TX)                                                               \
    template <typename R>                                                                                        \
    void gemmVbatched2s(const DdlaHandle_t& handle, char transA_0, char transB_0, int* d_m_0, int* d_n_0,       \
                        int* d_k_0, T0 alpha_0, const TA* const* d_A_array_0, int* d_lda_0,                      \
                        const TB* const* d_B_array_0, int* d_ldb_0, T0 beta_0, T0** d_C_array_0, int* d_ldc_0,  \
                        char transA_1, char transB_1, int* d_m_1, int* d_n_1, int* d_k_1,                        \
                        std::complex<R> alpha_1, const TX* const* d_AB_array_1, int* d_lda_1, int* d_ldb_1,      \
                        std::complex<R> beta_1, std::complex<R>** d_C_array_1, int* d_ldc_1, bool C0_left,       \
                        int batch_count, const int* segment_sizes, int segment_count);
DDLA_GEMM_VBATCHED2S_MIXED(R, std::complex<R>, std::complex<R>, R)
DDLA_GEMM_VBATCHED2S_MIXED(std::complex<R>, R, std::complex<R>, R)
DDLA_GEMM_VBATCHED2S_MIXED(R, std::complex<R>, std::complex<R>, std::complex<R>)
DDLA_GEMM_VBATCHED2S_MIXED(std::complex<R>, R, std::complex<R>, std::complex<R>)
DDLA_GEMM_VBATCHED2S_MIXED(std::complex<R>, std::complex<R>, std::complex<R>, R)
DDLA_GEMM_VBATCHED2S_MIXED(R, R, R, std::complex<R>)
#undef DDLA_GEMM_VBATCHED2S_MIXED

// Type-1 reduction of a Hermitian-definite pair with a caller's factor
// (reference ddla.h:2540-2562): with factorB holding B = L L^H ('L') or U^H U
// ('U'), A becomes L^-1 A L^-H (U^-H A U^-1), the whole leading n x n written
// Hermitian with a real diagonal.  Only the uplo triangles of A and factorB are
// read; factorB and everything outside the leading n x n are left as they were.
// descA / descB: matching square source-zero blocks covering n x n; the spans
// must not overlap.  std::invalid_argument for bad arguments (the reference's
// messages), std::runtime_error for a null handle.  Returns with the handle's
// stream synchronised.
template <typename T>
void phegst(const DdlaHandle_t& handle, char uplo, int n, T* A, const int* descA, const T* factorB,
            const int* descB);

// Two dependent batched GEMM stages sharing reusable temporaries (reference
// ddla.h:1851-1876, src/BLAS/gemm_vbatched.cpp:420-509): for each host-resident
// segment of segment_sizes in turn, stage 0 gives C0_b = alpha_0 op(A0_b)
// op(B0_b) for the segment's entries, then stage 1 gives C1_b = alpha_1 op(X_b)
// op(Y_b) + beta_1 C1_b with (X, Y) = (C0_b, AB1_b) if C0_left, else
// (AB1_b, C0_b); the C0 operand is read with d_lda_1 or d_ldb_1.  C0 entries of
// different segments may alias.  beta_0 must be zero, every segment positive and
// the segments must add up to batch_count (std::invalid_argument otherwise, as
// for the single-stage checks, which both stages also pass).
template <typename T>
void gemmVbatched2s(const DdlaHandle_t& handle, char transA_0, char transB_0, int* d_m_0, int* d_n_0, int* d_k_0,
                    T alpha_0, const T* const* d_A_array_0, int* d_lda_0, const T* const* d_B_array_0, int* d_ldb_0,
                    T beta_0, T** d_C_array_0, int* d_ldc_0, char transA_1, char transB_1, int* d_m_1, int* d_n_1,
                    int* d_k_1, T alpha_1, const T* const* d_AB_array_1, int* d_lda_1, int* d_ldb_1, T beta_1,
                    T** d_C_array_1, int* d_ldc_1, bool C0_left, int batch_count, const int* segment_sizes,
                    int segment_count);

// ppotrs<double> that allocates nothing (no reference counterpart): for callers
// that cannot allocate device memory while running.  The solve's flags live in
// a fixed device array inside the library (n <= 65536, nrhs <= 256; larger
// sizes throw std::invalid_argument).  The first call on a device should come
// before any stream capture; overlapping calls race on the shared array.
void ppotrs_noalloc(const DdlaHandle_t& handle, char side, char uplo, char trans, int n, int nrhs, const double* A,
                    const int* descA, double* B, const int* descB);

// Workspace split of the reference's check / size / run components
// (src/Cholesky/cholesky_workspace.h:133-154, 207-222, 239-249; plan_util.h).
// The *_workspace_size functions report device bytes; *_run performs the
// routine on caller scratch (no validation, no allocation).
namespace cholesky_impl {
template <typename T>
void ppotrf_workspace_size(const DdlaHandle_t& handle, char uplo, int n, const T* A, const int* descA,
                           std::size_t* backend_bytes, std::size_t* host_bytes);
template <typename T>
void ppotrf_run(const DdlaHandle_t& handle, char uplo, int n, T* A, int ia, int ja, const int* descA, int& info,
                void* backend_work, std::size_t backend_bytes, void* host_work, std::size_t host_bytes);
template <typename T>
void ppotrs_workspace_size(const DdlaHandle_t& handle, char side, int n, int nrhs, const int* descA,
                           const int* descB, std::size_t* backend_bytes, std::size_t* host_bytes);
// (src/Cholesky/cholesky_workspace.h:163-200)
template <typename T>
void ppotrf_bottom_right_workspace_size(const DdlaHandle_t& handle, char uplo, int n, T* A, const int* descA,
                                        std::size_t* backend_bytes, std::size_t* host_bytes);
template <typename T>
void ppotrf_bottom_right_run(const DdlaHandle_t& handle, char uplo, int n, T* A, const int* descA, int& info,
                             void* backend_work, std::size_t backend_bytes, void* host_work, std::size_t host_bytes);
template <typename T>
void ppotrs_run(const DdlaHandle_t& handle, char side, char uplo, char trans, int n, int nrhs, const T* A,
                const int* descA, T* B, const int* descB, void* backend_work, std::size_t backend_bytes,
                void* host_work, std::size_t host_bytes);
}  // namespace cholesky_impl

// ---------------------------------------------------------------------------
// Mixed precision (new): solve A*X = B for a Hermitian positive-definite FP64
// A to FP64 accuracy.  A low-precision Cholesky factor of A is computed with
// the trailing updates on the tensor cores (precision 'B': BF16 operands,
// 'T': TF32 operands; FP32 accumulation and FP32 storage, FP64 diagonal
// blocks), then X is refined in FP64 (residuals against the untouched FP64 A)
// with classical iterative refinement, switching to GMRES-IR preconditioned by
// the low-precision factor when refinement stagnates.  precision 'D' factors
// in FP64 directly.  uplo 'L' only.
//   On success A is unchanged, X holds the solution and iter >= 0 is the number
//   of refinement sweeps (GMRES iterations count one each; 0 when the first
//   solve already passes the stopping test).  If neither scheme
//   reaches the LAPACK ?sposv stopping test (||r|| <= ||x|| ||A|| eps sqrt(n))
//   within the iteration budget, the routine falls back to ppotrf/ppotrs in
//   FP64 (A then holds the FP64 factor) and sets iter = -(sweeps + 1).
//   info is ppotrf's info of whichever factorization produced X.
// ---------------------------------------------------------------------------
struct MixedReport {
    int iter = 0;            // refinement sweeps (>= 0), or -(sweeps+1) after the FP64 fallback
    int gmres = 0;           // 1 if GMRES-IR was used
    double shift = 0;        // diagonal shift applied to the low-precision factor (relative)
    double backward_error = 0;  // final max_j ||b_j - A x_j||_inf / (||A||_inf ||x_j||_inf)
};
void pposv_mixed(const DdlaHandle_t& handle, char uplo, char precision, int n, int nrhs, double* A,
                 const int* descA, const double* B, const int* descB, double* X, const int* descX, int& info,
                 MixedReport* report = nullptr);

// pposv_mixed with A, B and X in HOST memory (column-major, leading dimensions
// lda, ldb, ldx; only A's lower triangle is read).  The lower part of A goes to
// the device in column panels while the panels that have arrived are already
// factored (left-looking), so the host-to-device copy overlaps the tensor-core
// factorization; X comes back to host memory and the handle's stream is
// synchronised on return.  Pass pinned host memory (ddlaMallocHost /
// cudaHostAlloc) for the overlap: pageable memory is copied synchronously.
// Device scratch for A (n x n FP64), W and the factor's low-precision copy is
// taken per call from the handle's stream-ordered pool.  Same results and
// report as pposv_mixed on the device copies.
void pposv_mixed_host(const DdlaHandle_t& handle, char uplo, char precision, int n, int nrhs, const double* A,
                      int lda, const double* B, int ldb, double* X, int ldx, int& info,
                      MixedReport* report = nullptr);

}  // namespace ddla

#endif
