// ddla::gemmVbatched: the reference's variable-size batched GEMM
// (include/ddla/ddla.h:1836-1849, src/BLAS/gemm_vbatched.cpp:349-399,
// src/public_dispatch.cpp:1125-1136) on the kernels of gemm_vbatched.cu.
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

}  // namespace

template <typename T>
void gemmVbatched(const DdlaHandle_t& handle, char transA, char transB, int* d_m, int* d_n, int* d_k, T alpha,
                  const T* const* d_A_array, int* d_lda, const T* const* d_B_array, int* d_ldb, T beta,
                  T** d_C_array, int* d_ldc, int batch_count)
{
    if (handle == nullptr || !handle->initialized)
        throw std::invalid_argument("gemmVbatched: invalid DDLA handle");
    if (handle->backend != DdlaBackend::GPU)
        throw std::invalid_argument("gemmVbatched: only the GPU backend is implemented");
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
    cudaStream_t st = handle->stream;

    int summary[4];
    {
        detail::DeviceScratch work(handle, 4 * sizeof(int));
        int* d_summary = reinterpret_cast<int*>(work.data());
        detail::kernel_check(
            ddlak_gemm_vbatched_check(transA, transB, d_m, d_n, d_k, d_lda, d_ldb, d_ldc, batch_count, d_summary, st),
            "gemmVbatched: dimension check");
        detail::cuda_check(cudaMemcpyAsync(handle->host_word, d_summary, sizeof(summary), cudaMemcpyDeviceToHost, st),
                           "gemmVbatched: dimension summary");
        detail::cuda_check(cudaStreamSynchronize(st), "gemmVbatched: dimension summary");
        std::memcpy(summary, handle->host_word, sizeof(summary));
    }
    if (summary[3] != 0)
        throw std::invalid_argument("gemmVbatched: invalid dimensions at batch " + std::to_string(summary[3] - 1));
    detail::kernel_check(ddlak_gemm_vbatched(gv_code<T>(), transA, transB, summary[0], summary[1], d_m, d_n, d_k,
                                             &alpha, d_A_array, d_lda, d_B_array, d_ldb, &beta, d_C_array, d_ldc,
                                             batch_count, st),
                         "gemmVbatched");
}

#define DDLA_GV_INST(T)                                                                                          \
    template void gemmVbatched<T>(const DdlaHandle_t&, char, char, int*, int*, int*, T, const T* const*, int*, \
                                  const T* const*, int*, T, T**, int*, int);
DDLA_GV_INST(float)
DDLA_GV_INST(double)
DDLA_GV_INST(std::complex<float>)
DDLA_GV_INST(std::complex<double>)
#undef DDLA_GV_INST

}  // namespace ddla
