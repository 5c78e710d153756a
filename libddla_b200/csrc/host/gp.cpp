// ddla::cholNllBatched / gpNllBatched / cholNllGradBatched / gpNllGradBatched
// (include/ddla/ddla_batched.h): the negative log marginal likelihood
// loss = 1/2 (y^T A^-1 y + log det A) and its adjoint (no reference counterpart).
//
// Orders up to 1024: the forward is one persistent batched factor + solve +
// log-determinant launch (posvVbatched) or, for FP64 batches of one even order
// from 512, the blocked factorization batched over the matrices and a batched
// substitution; the backward a batched W = L^-1 and
// the tiled (W^T W) contraction with the adjoint epilogue.  Larger orders
// (batch 1): the blocked factorization (ddlak_potrf), the fused solve, and for
// the backward W = L^-1 from the fused forward substitution on the identity.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <limits>
#include <type_traits>
#include <stdexcept>
#include <string>
#include <vector>

#include <ddla/ddla_batched.h>
#include <ddla_kernels.h>

#include "ddla_stream.h"

namespace ddla {

namespace {

constexpr int kBatchedMaxOrder = 1024;

template <class T> constexpr char tcode();
template <> constexpr char tcode<float>() { return 's'; }
template <> constexpr char tcode<double>() { return 'd'; }

void ck(int e, const char* what) { detail::kernel_check(e, what); }

void check_shape(const DdlaHandle_t& h, const char* routine, int batch, int n)
{
    detail::require_gpu(h, routine);
    if (batch < 0 || n < 0) throw std::invalid_argument(std::string(routine) + ": negative batch or order");
    if (n > kBatchedMaxOrder && batch > 1)
        throw std::invalid_argument(std::string(routine) + ": orders above 1024 take one problem per call");
}

void check_theta(const char* routine, int d, const double* theta, int tstride, const void* X)
{
    if (d < 1 || d > 16) throw std::invalid_argument(std::string(routine) + ": point dimension outside [1, 16]");
    if (tstride != 0 && tstride != 3) throw std::invalid_argument(std::string(routine) + ": theta stride must be 0 or 3");
    if (!theta || !X) throw std::invalid_argument(std::string(routine) + ": null points or theta");
}

// FP64 batches of one even order in [512, 1024] with a 16-byte aligned base take
// the batched blocked factorization; the rest the persistent posvVbatched launch.
template <class T>
bool uniform_blocked(int batch, int n, const T* A)
{
    return std::is_same<T, double>::value && n >= 512 && n <= kBatchedMaxOrder && n % 2 == 0 && batch <= 65535 &&
           (reinterpret_cast<uintptr_t>(A) & 15) == 0;
}

template <class T>
void factor_solve(const DdlaHandle_t& h, int batch, int n, T* A, const T* y, T* alpha, double* logdet, double* quad,
                  int* info)
{
    cudaStream_t st = h->stream;
    const long long nn = (long long)n * n;
    detail::cuda_check(cudaMemcpyAsync(alpha, y, sizeof(T) * (size_t)batch * n, cudaMemcpyDeviceToDevice, st),
                       "copy y");
    if (uniform_blocked<T>(batch, n, A)) {
        // equal orders from 512: the blocked factorization batched over the matrices (diagonal
        // blocks, panels and DMMA trailing updates, one launch each per block column), then one
        // substitution launch that also forms log det
        ck(ddlak_potrf_batched_f64(batch, n, A, n, nn, info, st), "factorization");
        ck(ddlak_potrs_batched_f64(batch, n, A, n, nn, alpha, n, info, logdet, st), "solve");
    } else if (n <= kBatchedMaxOrder) {
        // device arrays for the batched launch: orders, leading dimensions, pointers
        const size_t bytes = detail::padded_bytes<int>(batch) * 2 + detail::padded_bytes<T*>(batch) * 2;
        detail::DeviceScratch ws(h, bytes);
        char* w = ws.data();
        int* d_n = detail::take<int>(w, batch);
        int* d_lda = detail::take<int>(w, batch);
        T** d_A = detail::take<T*>(w, batch);
        T** d_B = detail::take<T*>(w, batch);
        std::vector<int> hn(batch, n), hl(batch, n > 0 ? n : 1);
        std::vector<T*> ha(batch), hb(batch);
        for (int m = 0; m < batch; ++m) {
            ha[m] = A + m * nn;
            hb[m] = alpha + (long long)m * n;
        }
        detail::cuda_check(cudaMemcpyAsync(d_n, hn.data(), sizeof(int) * batch, cudaMemcpyHostToDevice, st), "upload");
        detail::cuda_check(cudaMemcpyAsync(d_lda, hl.data(), sizeof(int) * batch, cudaMemcpyHostToDevice, st), "upload");
        detail::cuda_check(cudaMemcpyAsync(d_A, ha.data(), sizeof(T*) * batch, cudaMemcpyHostToDevice, st), "upload");
        detail::cuda_check(cudaMemcpyAsync(d_B, hb.data(), sizeof(T*) * batch, cudaMemcpyHostToDevice, st), "upload");
        posvVbatched<T>(h, 'L', d_n, d_A, d_lda, d_B, logdet, info, batch, n);
    } else {
        ck(ddlak_potrf(tcode<T>(), 'L', n, A, n, info, st), "factorization");
        int hinfo = 0;
        detail::cuda_check(cudaMemcpyAsync(h->host_word, info, sizeof(int), cudaMemcpyDeviceToHost, st), "info");
        detail::cuda_check(cudaStreamSynchronize(st), "stream synchronisation");
        hinfo = *h->host_word;
        if (hinfo == 0) {
            const size_t sb = ddlak_potrs_workspace(n, 1);
            detail::DeviceScratch ws(h, sb);
            ck(ddlak_potrs(tcode<T>(), 'L', 'L', n, 1, A, n, alpha, n, ws.data(), sb, st), "solve");
            ck(ddlak_batched_logdiag(tcode<T>(), 1, n, A, n, nn, logdet, st), "log-determinant");
        } else {
            detail::cuda_check(cudaMemcpyAsync(alpha, y, sizeof(T) * n, cudaMemcpyDeviceToDevice, st), "copy y");
            const double nan = std::numeric_limits<double>::quiet_NaN();
            detail::cuda_check(cudaMemcpyAsync(logdet, &nan, sizeof(double), cudaMemcpyHostToDevice, st), "logdet");
            detail::cuda_check(cudaStreamSynchronize(st), "stream synchronisation");
        }
    }
    ck(ddlak_batched_dot(tcode<T>(), batch, n, y, n, alpha, n, quad, st), "y^T alpha");
}

// W = L^-1 for the (W^T W) contraction: one CTA per matrix up to order 1024,
// the fused forward substitution on the identity above.
template <class T>
void inverse_factor(const DdlaHandle_t& h, int batch, int n, const T* L, T* W)
{
    cudaStream_t st = h->stream;
    const long long nn = (long long)n * n;
    if (n <= kBatchedMaxOrder) {
        ck(ddlak_trtri_batched(tcode<T>(), batch, n, L, n, nn, W, n, nn, st), "L^-1");
        return;
    }
    const size_t sb = ddlak_potrs_workspace(n, n);
    detail::DeviceScratch ws(h, sb);
    ck(ddlak_trtri_blocked(tcode<T>(), n, L, n, W, n, ws.data(), sb, st), "L^-1");
}

}  // namespace

template <typename T>
void cholNllBatched(const DdlaHandle_t& h, int batch, int n, T* A, const T* y, T* alpha, double* logdet, double* quad,
                    int* info)
{
    check_shape(h, "cholNllBatched", batch, n);
    if (batch == 0 || n == 0) return;
    if (!A || !y || !alpha || !logdet || !quad || !info) throw std::invalid_argument("cholNllBatched: null array");
    factor_solve<T>(h, batch, n, A, y, alpha, logdet, quad, info);
}

template <typename T>
void gpNllBatched(const DdlaHandle_t& h, int batch, int n, int d, const T* X, const double* theta, int tstride,
                  const T* y, T* A, T* alpha, double* logdet, double* quad, int* info)
{
    check_shape(h, "gpNllBatched", batch, n);
    if (batch == 0 || n == 0) return;
    check_theta("gpNllBatched", d, theta, tstride, X);
    if (!A || !y || !alpha || !logdet || !quad || !info) throw std::invalid_argument("gpNllBatched: null array");
    ck(ddlak_gp_build(tcode<T>(), batch, n, d, X, (long long)n * d, theta, tstride, A, n, (long long)n * n,
                      h->stream),
       "kernel matrix");
    factor_solve<T>(h, batch, n, A, y, alpha, logdet, quad, info);
}

template <typename T>
void cholNllGradBatched(const DdlaHandle_t& h, int batch, int n, const T* L, const T* alpha, T* W, T* G)
{
    check_shape(h, "cholNllGradBatched", batch, n);
    if (batch == 0 || n == 0) return;
    if (!L || !alpha || !W || !G) throw std::invalid_argument("cholNllGradBatched: null array");
    inverse_factor<T>(h, batch, n, L, W);
    const long long nn = (long long)n * n;
    ck(ddlak_adjoint_contract(tcode<T>(), 1, batch, n, W, n, nn, alpha, n, nullptr, 0, 0, nullptr, 0, nullptr,
                              nullptr, G, n, nn, h->stream),
       "adjoint");
}

template <typename T>
void gpNllGradBatched(const DdlaHandle_t& h, int batch, int n, int d, const T* X, const double* theta, int tstride,
                      const T* L, const T* alpha, T* W, double* grad)
{
    check_shape(h, "gpNllGradBatched", batch, n);
    if (batch == 0 || n == 0) return;
    check_theta("gpNllGradBatched", d, theta, tstride, X);
    if (!L || !alpha || !W || !grad) throw std::invalid_argument("gpNllGradBatched: null array");
    inverse_factor<T>(h, batch, n, L, W);
    detail::DeviceScratch part(h, ddlak_adjoint_partial_bytes(batch, n));
    const long long nn = (long long)n * n;
    ck(ddlak_adjoint_contract(tcode<T>(), 0, batch, n, W, n, nn, alpha, n, X, d, (long long)n * d, theta, tstride,
                              reinterpret_cast<double*>(part.data()), grad, nullptr, 0, 0, h->stream),
       "adjoint");
}

#define DDLA_GP_INST(T)                                                                                             \
    template void cholNllBatched<T>(const DdlaHandle_t&, int, int, T*, const T*, T*, double*, double*, int*);      \
    template void gpNllBatched<T>(const DdlaHandle_t&, int, int, int, const T*, const double*, int, const T*, T*,  \
                                  T*, double*, double*, int*);                                                    \
    template void cholNllGradBatched<T>(const DdlaHandle_t&, int, int, const T*, const T*, T*, T*);                \
    template void gpNllGradBatched<T>(const DdlaHandle_t&, int, int, int, const T*, const double*, int, const T*,  \
                                      const T*, T*, double*);
DDLA_GP_INST(float)
DDLA_GP_INST(double)
#undef DDLA_GP_INST

}  // namespace ddla
