// ddla_batched.h -- batched uneven Cholesky (factor + solve + log-determinant)
// on a GPU handle.  No reference counterpart: the per-matrix equivalent is
// ppotrf + ppotrs + diag_logdet (src/Cholesky/ppotrf.cpp:326-349,
// ppotrs.cpp:65-85, diag_logdet.cpp:42-55).  The calling conventions are those
// of the reference's variable-size batched GEMM, ddla::gemmVbatched
// (include/ddla/ddla.h:1828-1849): dimension and matrix-pointer arrays are
// device resident, a GPU handle is required (any other handle throws
// std::invalid_argument), and the work is enqueued on the handle's stream.
#ifndef DDLA_BATCHED_H
#define DDLA_BATCHED_H

#include <vector>

#include <ddla/ddla_handle_t.h>

namespace ddla {

// For every i < batch_count, with n = d_n[i] (0 <= n <= max_n <= 1024),
// A = d_A_array[i] (column-major, d_lda[i] >= max(1, n)):
//   A = L L^T in place in the lower triangle (the upper one is not touched),
//   if d_B_array is not null: A x = b solved in place of b = d_B_array[i] (n values),
//   d_logdet[i] = log det A (FP64 accumulation), d_info[i] = LAPACK ?potrf info.
// A matrix with d_info[i] > 0 keeps its b and gets d_logdet[i] = NaN; its A
// holds the factor's first d_info[i]-1 columns.  uplo must be 'L'.
// All matrices run in ONE persistent kernel launch.  The call reads d_n back
// once (one synchronisation of the handle's stream) to build the work list and
// returns with the launch enqueued.
template <typename T>
void posvVbatched(const DdlaHandle_t& handle, char uplo, const int* d_n, T* const* d_A_array, const int* d_lda,
                  T* const* d_B_array, double* d_logdet, int* d_info, int batch_count, int max_n);

// The launch of posvVbatched built once (work list, per-matrix variant, launch
// grid) and captured in a CUDA graph: run() replays it on the handle's stream
// without any host synchronisation.  The arrays given at creation are used by
// every run; their matrix contents may change between runs, the orders may not.
class VbatchedPlan {
public:
    template <typename T>
    static VbatchedPlan* create(const DdlaHandle_t& handle, char uplo, const int* d_n, T* const* d_A_array,
                                const int* d_lda, T* const* d_B_array, double* d_logdet, int* d_info, int batch_count,
                                int max_n);
    ~VbatchedPlan();
    VbatchedPlan(const VbatchedPlan&) = delete;
    VbatchedPlan& operator=(const VbatchedPlan&) = delete;

    void run();
    double flops() const { return flops_; }  // sum over the batch of n^3/3 + n^2/2 + n/6 (+ 2 n^2 with b)
    int grid() const { return grid_; }

    struct Impl;

private:
    VbatchedPlan() = default;
    Impl* impl_ = nullptr;
    double flops_ = 0;
    int grid_ = 0;
};

// Project autotuner.  For each order bucket of 16 (orders 16b+1 .. 16b+16) it
// times both block-column widths of the kernel on synthetic matrices of that
// order, and it times the launch grid (one or the most resident CTAs per SM);
// the fastest choices are kept per (device, type, max_n bucket) and used by
// every later posvVbatched / VbatchedPlan.  When the environment variable
// DDLA_VBATCHED_TUNE_FILE names a file, tables are loaded from it on first use
// and written back after tuning.  type is 's' or 'd'.
void vbatchedAutotune(const DdlaHandle_t& handle, char type, int max_n);

struct VbatchedTuning {
    int nmax = 0;                       // 512 or 1024: the kernel instance for this max_n
    int grid = 0;                       // CTAs of the persistent launch
    int widths[2] = {0, 0};             // block-column width of variant 0 / 1
    std::vector<unsigned char> variant;  // per order bucket of 16
    bool tuned = false;                 // false: built-in defaults
};
VbatchedTuning vbatchedTuning(const DdlaHandle_t& handle, char type, int max_n);

// ---- negative log marginal likelihood and its adjoint ----------------------
// loss_b = 1/2 (y_b^T A_b^-1 y_b + log det A_b) for `batch` problems of order n,
// packed on the device: A, L, W [batch][n*n] column-major (leading dimension n),
// y, alpha [batch][n], X [batch][n][d] row-major, theta {l, sigma_f^2, sigma^2}
// per problem (theta_stride 3) or shared by all (theta_stride 0), logdet / quad
// / info [batch].  With alpha = A^-1 y the gradients are
//   dloss/dA = 1/2 (A^-1 - alpha alpha^T),  dloss/dy = alpha,
// and A^-1 = W^T W with W = L^-1 (lower).  Orders up to 1024 run one CTA per
// problem (the batched factorization of posvVbatched and a batched W = L^-1);
// larger orders take batch == 1 and the blocked single-matrix kernels.
// All calls are enqueued on the handle's stream; the forward ones read the
// orders back once (one synchronisation), the backward ones never synchronise.

// Forward on a given matrix: A (lower triangle) is replaced by L.
template <typename T>
void cholNllBatched(const DdlaHandle_t& handle, int batch, int n, T* A, const T* y, T* alpha, double* logdet,
                    double* quad, int* info);

// Forward of the Gaussian-process likelihood: A = K(theta) + sigma^2 I with
// K_ij = sigma_f^2 exp(-|x_i - x_j|^2 / (2 l^2)) is built on the device (lower
// triangle), then factored as in cholNllBatched.
template <typename T>
void gpNllBatched(const DdlaHandle_t& handle, int batch, int n, int d, const T* X, const double* theta,
                  int theta_stride, const T* y, T* A, T* alpha, double* logdet, double* quad, int* info);

// Dense adjoint from the forward's L and alpha: G = 1/2 (A^-1 - alpha alpha^T),
// full symmetric.  W is [batch][n*n] scratch.
template <typename T>
void cholNllGradBatched(const DdlaHandle_t& handle, int batch, int n, const T* L, const T* alpha, T* W, T* G);

// Hyperparameter gradient: grad[b][0..2] = dloss_b/d{l, sigma_f^2, sigma^2}, the
// adjoint contracted with dA/dtheta tile by tile (dA/dtheta is never stored).
template <typename T>
void gpNllGradBatched(const DdlaHandle_t& handle, int batch, int n, int d, const T* X, const double* theta,
                      int theta_stride, const T* L, const T* alpha, T* W, double* grad);

}  // namespace ddla

#endif
