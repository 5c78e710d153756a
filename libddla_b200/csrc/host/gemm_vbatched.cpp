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

#include <complex>
#include <cstring>
#include <stdexcept>
#include <string>

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
