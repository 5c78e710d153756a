// ddla::gemmVbatched and gemmVbatched2s: the reference's variable-size batched
// GEMM and its two-stage form (include/ddla/ddla.h:1836-1876,
// src/BLAS/gemm_vbatched.cpp:349-399, 420-509, src/public_dispatch.cpp:1125-1155)
// on the kernels of gemm_vbatched.cu.
// The checks run in the reference's order with its messages: handle, batch
// count (an empty batch returns before any other check), pointer arrays,
// transpose modes, dimension arrays, then one device validation pass whose
// summary (largest m, n, k and the first bad entry) is read back with one
// synchronisation of the handle's stream before the GEMM is enqueued.
#include <cuda_runtime.h>

#include <cctype>
#include <complex>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>

#include <ddla/ddla.h>
#include <ddla_kernels.h>

#include "ddla_stream.h"

namespace ddla {

namespace {

template <class T> constexpr char gv_code();
template <> constexpr char gv_code<float>() { return 's'; }
template <> constexpr char gv_code<double>() { return 'd'; }
template <> constexpr char gv_code<std::complex<float>>() { return 'c'; }
template <> constexpr char gv_code<std::complex<double>>() { return 'z'; }

bool valid_op(char t)
{
    return t == 'N' || t == 'n' || t == 'T' || t == 't' || t == 'C' || t == 'c';
}

void require_gpu_handle(const DdlaHandle_t& handle, const char* who)
{
    if (handle == nullptr || !handle->initialized)
        throw std::invalid_argument(std::string(who) + ": invalid DDLA handle");
    if (handle->backend != DdlaBackend::GPU)
        throw std::invalid_argument(std::string(who) + ": only the GPU backend is implemented");
}

// The device validation pass of one stage (the reference's
// vbatched_dimensions_check, src/BLAS/gemm_vbatched.cpp:135-160, 335-345): the
// dimension arrays must exist, every entry must be valid; returns the largest
// m, n, k through max3.  One synchronisation of the handle's stream.
void stage_dimensions(const DdlaHandle_t& handle, char ta, char tb, const int* d_m, const int* d_n, const int* d_k,
                      const int* d_lda, const int* d_ldb, const int* d_ldc, int batch, int max3[3])
{
    if (d_m == nullptr || d_n == nullptr || d_k == nullptr || d_lda == nullptr || d_ldb == nullptr ||
        d_ldc == nullptr)
        throw std::invalid_argument("gemmVbatched: null dimension array");
    cudaStream_t st = handle->stream;
    int summary[4];
    {
        detail::DeviceScratch work(handle, 4 * sizeof(int));
        int* d_summary = reinterpret_cast<int*>(work.data());
        detail::kernel_check(
            ddlak_gemm_vbatched_check(ta, tb, d_m, d_n, d_k, d_lda, d_ldb, d_ldc, batch, d_summary, st),
            "gemmVbatched: dimension check");
        detail::cuda_check(cudaMemcpyAsync(handle->host_word, d_summary, sizeof(summary), cudaMemcpyDeviceToHost, st),
                           "gemmVbatched: dimension summary");
        detail::cuda_check(cudaStreamSynchronize(st), "gemmVbatched: dimension summary");
        std::memcpy(summary, handle->host_word, sizeof(summary));
    }
    if (summary[3] != 0)
        throw std::invalid_argument("gemmVbatched: invalid dimensions at batch " + std::to_string(summary[3] - 1));
    max3[0] = summary[0];
    max3[1] = summary[1];
    max3[2] = summary[2];
}

}  // namespace

template <typename T>
void gemmVbatched(const DdlaHandle_t& handle, char transA, char transB, int* d_m, int* d_n, int* d_k, T alpha,
                  const T* const* d_A_array, int* d_lda, const T* const* d_B_array, int* d_ldb, T beta,
                  T** d_C_array, int* d_ldc, int batch_count)
{
    require_gpu_handle(handle, "gemmVbatched");
    if (batch_count < 0) throw std::invalid_argument("gemmVbatched: negative batch count");
    if (batch_count == 0) return;
    if (d_A_array == nullptr || d_B_array == nullptr || d_C_array == nullptr)
        throw std::invalid_argument("gemmVbatched: null matrix pointer array");
    if (!valid_op(transA) || !valid_op(transB))
        throw std::invalid_argument("gemmVbatched: invalid transpose operation");
    if (d_m == nullptr || d_n == nullptr || d_k == nullptr || d_lda == nullptr || d_ldb == nullptr ||
        d_ldc == nullptr)
        throw std::invalid_argument("gemmVbatched: null dimension array");
    detail::cuda_check(cudaSetDevice(handle->device), "cudaSetDevice");
    int mx[3];
    stage_dimensions(handle, transA, transB, d_m, d_n, d_k, d_lda, d_ldb, d_ldc, batch_count, mx);
    detail::kernel_check(ddlak_gemm_vbatched(gv_code<T>(), transA, transB, mx[0], mx[1], d_m, d_n, d_k, &alpha,
                                             d_A_array, d_lda, d_B_array, d_ldb, &beta, d_C_array, d_ldc, batch_count,
                                             handle->stream),
                         "gemmVbatched");
}

template <typename T>
void gemmVbatched2s(const DdlaHandle_t& handle, char transA_0, char transB_0, int* d_m_0, int* d_n_0, int* d_k_0,
                    T alpha_0, const T* const* d_A_array_0, int* d_lda_0, const T* const* d_B_array_0, int* d_ldb_0,
                    T beta_0, T** d_C_array_0, int* d_ldc_0, char transA_1, char transB_1, int* d_m_1, int* d_n_1,
                    int* d_k_1, T alpha_1, const T* const* d_AB_array_1, int* d_lda_1, int* d_ldb_1, T beta_1,
                    T** d_C_array_1, int* d_ldc_1, bool C0_left, int batch_count, const int* segment_sizes,
                    int segment_count)
{
    require_gpu_handle(handle, "gemmVbatched2s");
    if (batch_count < 0) throw std::invalid_argument("gemmVbatched2s: negative batch count");
    if (batch_count == 0) return;
    if (beta_0 != T{}) throw std::invalid_argument("gemmVbatched2s: stage-zero beta must be zero");
    if (segment_sizes == nullptr || segment_count <= 0)
        throw std::invalid_argument("gemmVbatched2s: missing segment sizes");
    long long total = 0;
    for (int s = 0; s < segment_count; ++s) {
        if (segment_sizes[s] <= 0) throw std::invalid_argument("gemmVbatched2s: segment sizes must be positive");
        total += segment_sizes[s];
    }
    if (total != batch_count)
        throw std::invalid_argument("gemmVbatched2s: segment total does not match batch count");
    if (d_A_array_0 == nullptr || d_B_array_0 == nullptr || d_C_array_0 == nullptr || d_AB_array_1 == nullptr ||
        d_C_array_1 == nullptr)
        throw std::invalid_argument("gemmVbatched2s: null matrix pointer array");
    // the transpose check keeps the single-stage message (the reference shares it)
    if (!valid_op(transA_0) || !valid_op(transB_0) || !valid_op(transA_1) || !valid_op(transB_1))
        throw std::invalid_argument("gemmVbatched: invalid transpose operation");
    detail::cuda_check(cudaSetDevice(handle->device), "cudaSetDevice");
    int mx0[3], mx1[3];
    stage_dimensions(handle, transA_0, transB_0, d_m_0, d_n_0, d_k_0, d_lda_0, d_ldb_0, d_ldc_0, batch_count, mx0);
    stage_dimensions(handle, transA_1, transB_1, d_m_1, d_n_1, d_k_1, d_lda_1, d_ldb_1, d_ldc_1, batch_count, mx1);
    const bool run0 = mx0[0] > 0 && mx0[1] > 0, run1 = mx1[0] > 0 && mx1[1] > 0;
    if (!run0 && !run1) return;
    cudaStream_t st = handle->stream;
    const char tc = gv_code<T>();
    // Segment by segment: stage 0 of the segment, then its stage 1, which reads
    // the segment's temporaries (segments may share temporary storage).  The
    // kernel walks a segment's entries in grid chunks of 65535.
    long long c = 0;
    for (int s = 0; s < segment_count; ++s) {
        const int nb = segment_sizes[s];
        if (run0)
            detail::kernel_check(ddlak_gemm_vbatched(tc, transA_0, transB_0, mx0[0], mx0[1], d_m_0 + c, d_n_0 + c,
                                                     d_k_0 + c, &alpha_0, d_A_array_0 + c, d_lda_0 + c,
                                                     d_B_array_0 + c, d_ldb_0 + c, &beta_0, d_C_array_0 + c,
                                                     d_ldc_0 + c, nb, st),
                                 "gemmVbatched2s: stage 0");
        if (run1) {
            const void* left = C0_left ? static_cast<const void*>(d_C_array_0 + c)
                                       : static_cast<const void*>(d_AB_array_1 + c);
            const void* right = C0_left ? static_cast<const void*>(d_AB_array_1 + c)
                                        : static_cast<const void*>(d_C_array_0 + c);
            detail::kernel_check(ddlak_gemm_vbatched(tc, transA_1, transB_1, mx1[0], mx1[1], d_m_1 + c, d_n_1 + c,
                                                     d_k_1 + c, &alpha_1, left, d_lda_1 + c, right, d_ldb_1 + c,
                                                     &beta_1, d_C_array_1 + c, d_ldc_1 + c, nb, st),
                                 "gemmVbatched2s: stage 1");
        }
        c += nb;
    }
}

// ---- one real and one complex operand (the reference's mixed overloads,
// include/ddla/ddla.h:1878-1939, src/BLAS/gemm_mixed.cpp:26-32, 224-234, 787-870) ----
namespace {

char mixed_op(char t)
{
    t = static_cast<char>(std::toupper(static_cast<unsigned char>(t)));
    if (t != 'N' && t != 'T' && t != 'C') throw std::invalid_argument("gemm(real,complex): invalid transpose flag");
    return t;
}

enum class Kind { real, cplx };

// One stage's checks (the reference's mixed_vbatched_check, GPU arm,
// src/BLAS/gemm_mixed.cpp:787-830): the metadata arrays, the device dimension
// pass (largest m, n, k into mx), then the device pointer pass.
void mixed_stage_check(const DdlaHandle_t& h, char ta, char tb, int* m, int* n, int* k, bool alpha_zero,
                       bool beta_one, const void* const* A, int* lda, const void* const* B, int* ldb,
                       void* const* C, int* ldc, int count, int mx[3])
{
    if (!m || !n || !k || !lda || !ldb || !ldc || !A || !B || !C)
        throw std::invalid_argument("gemmVbatched(mixed): null metadata array");
    stage_dimensions(h, ta, tb, m, n, k, lda, ldb, ldc, count, mx);
    cudaStream_t st = h->stream;
    {
        detail::DeviceScratch work(h, sizeof(int));
        int* d_bad = reinterpret_cast<int*>(work.data());
        detail::kernel_check(ddlak_gemm_vbatched_pointers(m, n, k, A, B, C, alpha_zero ? 1 : 0, beta_one ? 1 : 0,
                                                          count, d_bad, st),
                             "gemmVbatched(mixed): pointer check");
        detail::cuda_check(cudaMemcpyAsync(h->host_word, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st),
                           "gemmVbatched(mixed): pointer check");
        detail::cuda_check(cudaStreamSynchronize(st), "gemmVbatched(mixed): pointer check");
    }
    if (h->host_word[0] != 0)
        throw std::invalid_argument("gemmVbatched(mixed): null matrix at batch " + std::to_string(h->host_word[0] - 1));
}

// One stage on the kernels: a real output (two real operands), a complex one
// from two complex operands (the typed kernel) or from one real operand (mixed).
template <typename R>
void mixed_stage_run(const DdlaHandle_t& h, Kind ka, Kind kb, Kind kc, char ta, char tb, const int mx[3], int* m,
                     int* n, int* k, const void* alpha, const void* const* A, int* lda, const void* const* B,
                     int* ldb, const void* beta, void* const* C, int* ldc, int count)
{
    if (count == 0 || mx[0] == 0 || mx[1] == 0) return;
    const char rt = sizeof(R) == 4 ? 's' : 'd', zt = sizeof(R) == 4 ? 'c' : 'z';
    cudaStream_t st = h->stream;
    void* Cv = const_cast<void**>(C);  // the device array of C pointers
    int e;
    if (kc == Kind::real)
        e = ddlak_gemm_vbatched(rt, ta, tb, mx[0], mx[1], m, n, k, alpha, A, lda, B, ldb, beta, Cv, ldc, count, st);
    else if (ka == Kind::cplx && kb == Kind::cplx)
        e = ddlak_gemm_vbatched(zt, ta, tb, mx[0], mx[1], m, n, k, alpha, A, lda, B, ldb, beta, Cv, ldc, count, st);
    else
        e = ddlak_gemm_vbatched_mixed(zt, ka == Kind::cplx ? 1 : 0, ta, tb, mx[0], mx[1], m, n, k, alpha, A, lda, B,
                                      ldb, beta, Cv, ldc, count, st);
    detail::kernel_check(e, "gemmVbatched(mixed)");
}

template <typename R>
void mixed_vbatched(const DdlaHandle_t& handle, bool complex_left, char ta, char tb, int* m, int* n, int* k,
                    std::complex<R> alpha, const void* const* A, int* lda, const void* const* B, int* ldb,
                    std::complex<R> beta, std::complex<R>** C, int* ldc, int count)
{
    if (handle == nullptr) throw std::runtime_error("gemmVbatched(mixed): null handle");
    require_gpu_handle(handle, "gemmVbatched(mixed)");
    if (count < 0) throw std::invalid_argument("gemmVbatched(mixed): negative batch count");
    if (count == 0) return;
    ta = mixed_op(ta);
    tb = mixed_op(tb);
    detail::cuda_check(cudaSetDevice(handle->device), "cudaSetDevice");
    int mx[3];
    mixed_stage_check(handle, ta, tb, m, n, k, alpha == std::complex<R>(0), beta == std::complex<R>(1), A, lda, B,
                      ldb, reinterpret_cast<void* const*>(C), ldc, count, mx);
    const Kind ka = complex_left ? Kind::cplx : Kind::real, kb = complex_left ? Kind::real : Kind::cplx;
    mixed_stage_run<R>(handle, ka, kb, Kind::cplx, ta, tb, mx, m, n, k, &alpha, A, lda, B, ldb, &beta,
                       reinterpret_cast<void* const*>(C), ldc, count);
}

// Two stages, C0 of type T0 (the reference's mixed_vbatched_2s, src/BLAS/gemm_mixed.cpp:878-947).
template <typename R, typename T0>
void mixed_vbatched_2s(const DdlaHandle_t& h, Kind ka, Kind kb, Kind kx, char ta0, char tb0, int* m0, int* n0,
                       int* k0, T0 alpha0, const void* const* a0, int* lda0, const void* const* b0, int* ldb0,
                       T0 beta0, T0** c0, int* ldc0, char ta1, char tb1, int* m1, int* n1, int* k1,
                       std::complex<R> alpha1, const void* const* ab1, int* lda1, int* ldb1, std::complex<R> beta1,
                       std::complex<R>** c1, int* ldc1, bool left, int count, const int* segments, int segment_count)
{
    using Z = std::complex<R>;
    if (h == nullptr) throw std::runtime_error("gemmVbatched2s(mixed): null handle");
    require_gpu_handle(h, "gemmVbatched2s(mixed)");
    if (count < 0) throw std::invalid_argument("gemmVbatched2s(mixed): negative batch count");
    if (count == 0) return;
    if (beta0 != T0(0)) throw std::invalid_argument("gemmVbatched2s(mixed): stage-zero beta must be zero");
    if (!segments || segment_count <= 0) throw std::invalid_argument("gemmVbatched2s(mixed): missing segments");
    long long total = 0;
    for (int s = 0; s < segment_count; ++s) {
        if (segments[s] <= 0) throw std::invalid_argument("gemmVbatched2s(mixed): nonpositive segment");
        total += segments[s];
    }
    if (total != count) throw std::invalid_argument("gemmVbatched2s(mixed): segment total mismatch");
    ta0 = mixed_op(ta0);
    tb0 = mixed_op(tb0);
    ta1 = mixed_op(ta1);
    tb1 = mixed_op(tb1);
    detail::cuda_check(cudaSetDevice(h->device), "cudaSetDevice");
    const Kind k0k = std::is_same_v<T0, Z> ? Kind::cplx : Kind::real;
    const void* const* c0v = reinterpret_cast<const void* const*>(c0);
    int mx0[3], mx1[3];
    mixed_stage_check(h, ta0, tb0, m0, n0, k0, alpha0 == T0(0), beta0 == T0(1), a0, lda0, b0, ldb0,
                      reinterpret_cast<void* const*>(c0), ldc0, count, mx0);
    mixed_stage_check(h, ta1, tb1, m1, n1, k1, alpha1 == Z(0), beta1 == Z(1), left ? c0v : ab1, lda1,
                      left ? ab1 : c0v, ldb1, reinterpret_cast<void* const*>(c1), ldc1, count, mx1);
    // the intermediate's footprint, before either stage writes
    if (alpha1 != Z(0)) {
        const bool trans = (left ? ta1 : tb1) != 'N';
        detail::DeviceScratch work(h, sizeof(int));
        int* d_bad = reinterpret_cast<int*>(work.data());
        detail::kernel_check(ddlak_gemm_vbatched_footprint(m0, n0, ldc0, m1, n1, k1, left ? lda1 : ldb1, left ? 1 : 0,
                                                           trans ? 1 : 0, count, d_bad, h->stream),
                             "gemmVbatched2s(mixed): intermediate check");
        detail::cuda_check(cudaMemcpyAsync(h->host_word, d_bad, sizeof(int), cudaMemcpyDeviceToHost, h->stream),
                           "gemmVbatched2s(mixed): intermediate check");
        detail::cuda_check(cudaStreamSynchronize(h->stream), "gemmVbatched2s(mixed): intermediate check");
        if (h->host_word[0] != 0)
            throw std::invalid_argument("gemmVbatched2s(mixed): incompatible intermediate dimensions");
    }
    long long c = 0;
    for (int s = 0; s < segment_count; ++s) {
        const int nb = segments[s];
        mixed_stage_run<R>(h, ka, kb, k0k, ta0, tb0, mx0, m0 + c, n0 + c, k0 + c, &alpha0, a0 + c, lda0 + c, b0 + c,
                           ldb0 + c, &beta0, reinterpret_cast<void* const*>(c0) + c, ldc0 + c, nb);
        mixed_stage_run<R>(h, left ? k0k : kx, left ? kx : k0k, Kind::cplx, ta1, tb1, mx1, m1 + c, n1 + c, k1 + c,
                           &alpha1, (left ? c0v : ab1) + c, lda1 + c, (left ? ab1 : c0v) + c, ldb1 + c, &beta1,
                           reinterpret_cast<void* const*>(c1) + c, ldc1 + c, nb);
        c += nb;
    }
}

}  // namespace

template <typename R>
void gemmVbatched(const DdlaHandle_t& handle, char transA, char transB, int* d_m, int* d_n, int* d_k,
                  std::complex<R> alpha, const R* const* d_A_array, int* d_lda,
                  const std::complex<R>* const* d_B_array, int* d_ldb, std::complex<R> beta,
                  std::complex<R>** d_C_array, int* d_ldc, int batch_count)
{
    mixed_vbatched<R>(handle, false, transA, transB, d_m, d_n, d_k, alpha,
                      reinterpret_cast<const void* const*>(d_A_array), d_lda,
                      reinterpret_cast<const void* const*>(d_B_array), d_ldb, beta, d_C_array, d_ldc, batch_count);
}

template <typename R>
void gemmVbatched(const DdlaHandle_t& handle, char transA, char transB, int* d_m, int* d_n, int* d_k,
                  std::complex<R> alpha, const std::complex<R>* const* d_A_array, int* d_lda,
                  const R* const* d_B_array, int* d_ldb, std::complex<R> beta, std::complex<R>** d_C_array,
                  int* d_ldc, int batch_count)
{
    mixed_vbatched<R>(handle, true, transA, transB, d_m, d_n, d_k, alpha,
                      reinterpret_cast<const void* const*>(d_A_array), d_lda,
                      reinterpret_cast<const void* const*>(d_B_array), d_ldb, beta, d_C_array, d_ldc, batch_count);
}

#define DDLA_GV2M(TA, TB, T0, TX, KA, KB, KX)                                                                   \
    template <typename R>                                                                                        \
    void gemmVbatched2s(const DdlaHandle_t& handle, char transA_0, char transB_0, int* d_m_0, int* d_n_0,       \
                        int* d_k_0, T0 alpha_0, const TA* const* d_A_array_0, int* d_lda_0,                      \
                        const TB* const* d_B_array_0, int* d_ldb_0, T0 beta_0, T0** d_C_array_0, int* d_ldc_0,  \
                        char transA_1, char transB_1, int* d_m_1, int* d_n_1, int* d_k_1,                        \
                        std::complex<R> alpha_1, const TX* const* d_AB_array_1, int* d_lda_1, int* d_ldb_1,      \
                        std::complex<R> beta_1, std::complex<R>** d_C_array_1, int* d_ldc_1, bool C0_left,       \
                        int batch_count, const int* segment_sizes, int segment_count)                            \
    {                                                                                                            \
        mixed_vbatched_2s<R, T0>(handle, Kind::KA, Kind::KB, Kind::KX, transA_0, transB_0, d_m_0, d_n_0, d_k_0, \
                                 alpha_0, reinterpret_cast<const void* const*>(d_A_array_0), d_lda_0,            \
                                 reinterpret_cast<const void* const*>(d_B_array_0), d_ldb_0, beta_0,            \
                                 d_C_array_0, d_ldc_0, transA_1, transB_1, d_m_1, d_n_1, d_k_1, alpha_1,         \
                                 reinterpret_cast<const void* const*>(d_AB_array_1), d_lda_1, d_ldb_1, beta_1,   \
                                 d_C_array_1, d_ldc_1, C0_left, batch_count, segment_sizes, segment_count);      \
    }
// (A0, B0, C0, AB1) element types of the reference's six overloads (include/ddla/ddla.h:1893-2030)
DDLA_GV2M(R, std::complex<R>, std::complex<R>, R, real, cplx, real)
DDLA_GV2M(std::complex<R>, R, std::complex<R>, R, cplx, real, real)
DDLA_GV2M(R, std::complex<R>, std::complex<R>, std::complex<R>, real, cplx, cplx)
DDLA_GV2M(std::complex<R>, R, std::complex<R>, std::complex<R>, cplx, real, cplx)
DDLA_GV2M(std::complex<R>, std::complex<R>, std::complex<R>, R, cplx, cplx, real)
DDLA_GV2M(R, R, R, std::complex<R>, real, real, cplx)
#undef DDLA_GV2M

#define DDLA_GV2M_INST(R, TA, TB, T0, TX)                                                                        \
    template void gemmVbatched2s<R>(const DdlaHandle_t&, char, char, int*, int*, int*, T0, const TA* const*,    \
                                    int*, const TB* const*, int*, T0, T0**, int*, char, char, int*, int*, int*, \
                                    std::complex<R>, const TX* const*, int*, int*, std::complex<R>,             \
                                    std::complex<R>**, int*, bool, int, const int*, int);
#define DDLA_GV2M_TYPES(R)                                                                                       \
    DDLA_GV2M_INST(R, R, std::complex<R>, std::complex<R>, R)                                                    \
    DDLA_GV2M_INST(R, std::complex<R>, R, std::complex<R>, R)                                                    \
    DDLA_GV2M_INST(R, R, std::complex<R>, std::complex<R>, std::complex<R>)                                      \
    DDLA_GV2M_INST(R, std::complex<R>, R, std::complex<R>, std::complex<R>)                                      \
    DDLA_GV2M_INST(R, std::complex<R>, std::complex<R>, std::complex<R>, R)                                      \
    DDLA_GV2M_INST(R, R, R, R, std::complex<R>)
DDLA_GV2M_TYPES(float)
DDLA_GV2M_TYPES(double)
#undef DDLA_GV2M_TYPES
#undef DDLA_GV2M_INST

#define DDLA_GVM_INST(R)                                                                                        \
    template void gemmVbatched<R>(const DdlaHandle_t&, char, char, int*, int*, int*, std::complex<R>,          \
                                  const R* const*, int*, const std::complex<R>* const*, int*, std::complex<R>, \
                                  std::complex<R>**, int*, int);                                               \
    template void gemmVbatched<R>(const DdlaHandle_t&, char, char, int*, int*, int*, std::complex<R>,          \
                                  const std::complex<R>* const*, int*, const R* const*, int*, std::complex<R>, \
                                  std::complex<R>**, int*, int);
DDLA_GVM_INST(float)
DDLA_GVM_INST(double)
#undef DDLA_GVM_INST

#define DDLA_GV_INST(T)                                                                                          \
    template void gemmVbatched<T>(const DdlaHandle_t&, char, char, int*, int*, int*, T, const T* const*, int*, \
                                  const T* const*, int*, T, T**, int*, int);                                   \
    template void gemmVbatched2s<T>(const DdlaHandle_t&, char, char, int*, int*, int*, T, const T* const*, int*, \
                                    const T* const*, int*, T, T**, int*, char, char, int*, int*, int*, T,        \
                                    const T* const*, int*, int*, T, T**, int*, bool, int, const int*, int);
DDLA_GV_INST(float)
DDLA_GV_INST(double)
DDLA_GV_INST(std::complex<float>)
DDLA_GV_INST(std::complex<double>)
#undef DDLA_GV_INST

}  // namespace ddla
