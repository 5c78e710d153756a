// ddla::phegst on a 1x1 grid: the type-1 reduction of a Hermitian-definite pair
// with a caller's Cholesky factor (reference include/ddla/ddla.h:2540-2562,
// src/Eigensolver/phegst.cpp:26-75 checks, 140-176 run, 195-209 entry).
// With B = L L^H ('L') or U^H U ('U'), A <- L^-1 A L^-H (L = U^H for 'U'):
// the Hermitian completion of A from its uplo triangle, the forward solve
// A <- L^-1 A, the forward solve A <- A L^-H (the side-'R' form), and the
// completion again, which leaves the whole leading n x n Hermitian with a real
// diagonal.  Only the uplo triangles of A and of the factor are read; the
// factor and everything outside the leading n x n are left as they were.
#include <cuda_runtime.h>

#include <cctype>
#include <climits>
#include <complex>
#include <cstdint>
#include <stdexcept>
#include <string>

#include <ddla/ddla.h>
#include <ddla_kernels.h>

#include "ddla_stream.h"

namespace ddla {

namespace {

template <class T> constexpr char hg_code();
template <> constexpr char hg_code<float>() { return 's'; }
template <> constexpr char hg_code<double>() { return 'd'; }
template <> constexpr char hg_code<std::complex<float>>() { return 'c'; }
template <> constexpr char hg_code<std::complex<double>>() { return 'z'; }

// The element spans [p, p + (cols-1) ld + rows) of two column-major matrices
// intersect (the reference's matrix_overlaps, src/helpers.h:37-43).
bool spans_overlap(const void* a, int lda, int rows, int cols, const void* b, int ldb, std::size_t esize)
{
    if (!rows || !cols) return false;
    const auto a0 = reinterpret_cast<std::uintptr_t>(a), b0 = reinterpret_cast<std::uintptr_t>(b);
    const std::uintptr_t a1 = a0 + ((std::size_t)(cols - 1) * lda + rows) * esize;
    const std::uintptr_t b1 = b0 + ((std::size_t)(cols - 1) * ldb + rows) * esize;
    return a0 < b1 && b0 < a1;
}

}  // namespace

template <typename T>
void phegst(const DdlaHandle_t& handle, char uplo, int n, T* A, const int* descA, const T* factorB,
            const int* descB)
{
    if (handle == nullptr) throw std::runtime_error("phegst: null handle");
    detail::require_gpu(handle, "phegst");
    if (handle->nprocs > 1) throw std::invalid_argument("phegst: served on a 1x1 grid only");
    const char up = static_cast<char>(std::toupper(static_cast<unsigned char>(uplo)));
    if (n < 0 || n > INT_MAX / 8 || (up != 'L' && up != 'U'))
        throw std::invalid_argument("phegst: invalid order or triangle");
    detail::check_desc(descA, handle);
    detail::check_desc(descB, handle);
    const int block = descA[DDLA_MB_];
    for (const int* d : {descA, descB})
        if (d[DDLA_MB_] != block || d[DDLA_NB_] != block || d[DDLA_RSRC_] != 0 || d[DDLA_CSRC_] != 0 ||
            n > d[DDLA_M_] || n > d[DDLA_N_])
            throw std::invalid_argument("phegst: matching square source-zero descriptors required");
    // one rank holds the whole leading n x n
    if (n && (A == nullptr || factorB == nullptr)) throw std::invalid_argument("phegst: missing active matrix or factor");
    const int lda = descA[DDLA_LLD_], ldf = descB[DDLA_LLD_];
    if (spans_overlap(A, lda, n, n, factorB, ldf, sizeof(T)))
        throw std::invalid_argument("phegst: A and factor must be disjoint");
    if (n == 0) return;

    detail::cuda_check(cudaSetDevice(handle->device), "cudaSetDevice");
    cudaStream_t st = handle->stream;
    const char tc = hg_code<T>();
    const std::size_t wb = ddlak_potrs_workspace(n, n);
    detail::DeviceScratch w1(handle, wb), w2(handle, wb);  // one status word per solve
    detail::kernel_check(ddlak_herm_complete(tc, up, n, A, lda, st), "phegst: completion");
    detail::kernel_check(ddlak_forward_solve(tc, up, 'L', n, n, factorB, ldf, A, lda, w1.data(), wb, st),
                         "phegst: left solve");
    detail::kernel_check(ddlak_forward_solve(tc, up, 'R', n, n, factorB, ldf, A, lda, w2.data(), wb, st),
                         "phegst: right solve");
    detail::kernel_check(ddlak_herm_complete(tc, up, n, A, lda, st), "phegst: completion");
    detail::cuda_check(cudaMemcpyAsync(handle->host_word, w1.data(), sizeof(int), cudaMemcpyDeviceToHost, st),
                       "phegst: status");
    detail::cuda_check(cudaMemcpyAsync(handle->host_word + 1, w2.data(), sizeof(int), cudaMemcpyDeviceToHost, st),
                       "phegst: status");
    detail::cuda_check(cudaStreamSynchronize(st), "phegst: stream synchronisation");
    if (handle->host_word[0] != 0 || handle->host_word[1] != 0)
        throw std::runtime_error("phegst: a device wait of the triangular solve gave up");
}

#define DDLA_HG_INST(T) \
    template void phegst<T>(const DdlaHandle_t&, char, int, T*, const int*, const T*, const int*);
DDLA_HG_INST(float)
DDLA_HG_INST(double)
DDLA_HG_INST(std::complex<float>)
DDLA_HG_INST(std::complex<double>)
#undef DDLA_HG_INST

}  // namespace ddla
