// Variable-size batched GEMM: C_b = alpha op(A_b) op(B_b) + beta C_b for every
// b < batch, each with its own m, n, k and leading dimensions, all read from
// device arrays (the contract of the reference's gemmVbatched,
// include/ddla/ddla.h:1828-1849, src/BLAS/gemm_vbatched.cpp).
//
// ddlak_gemm_vbatched_check validates every entry on the device (negative
// sizes, leading dimensions below the rows of their matrix) and reduces the
// largest m, n, k, the reference's validate_and_max_dimensions
// (gemm_vbatched.cpp:72-106).  ddlak_gemm_vbatched then launches one CTA per
// 64 x 64 tile of C over a (ceil(max_m/64), ceil(max_n/64), batch) grid; a
// CTA whose tile lies outside its matrix returns at once.  Per CTA: 16-deep
// k slabs of op(A) and op(B) staged in shared memory (loads coalesced along
// the contiguous index for every transpose mode), a 4 x 4 register tile per
// thread on rows tx + 16 r and columns ty + 16 q (conflict-free shared reads,
// coalesced stores of C).  The edge cases follow the reference kernel
// (src/vbatched/gemm_template_kernel_vbatched.hpp:19-33, 77-91, and the
// stores of gemm_template_device.hpp:226-227): an empty m or n does nothing;
// k = 0 or alpha = 0 scales C by beta without reading A or B (beta = 1 leaves
// it, beta = 0 writes zeros without reading C); a null matrix pointer skips
// the entry; beta = 0 never reads C.  FP32/FP64 and complex arithmetic in the
// storage precision on the CUDA cores; the grid's batch dimension is walked in
// chunks of 65535.
#include <cuda_runtime.h>

#include <cstdint>

#include <ddla_kernels.h>

#include "common.cuh"
#include "profile.h"

namespace ddlak {
namespace {

constexpr int GB_M = 64, GB_N = 64, GB_K = 16, GB_NT = 256;

__device__ __forceinline__ float mulv(float a, float b) { return a * b; }
__device__ __forceinline__ double mulv(double a, double b) { return a * b; }
__device__ __forceinline__ cf32 mulv(cf32 a, cf32 b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__device__ __forceinline__ cf64 mulv(cf64 a, cf64 b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__device__ __forceinline__ bool is_zero(float a) { return a == 0.f; }
__device__ __forceinline__ bool is_zero(double a) { return a == 0.0; }
__device__ __forceinline__ bool is_zero(cf32 a) { return a.x == 0.f && a.y == 0.f; }
__device__ __forceinline__ bool is_zero(cf64 a) { return a.x == 0.0 && a.y == 0.0; }
__device__ __forceinline__ bool is_one(float a) { return a == 1.f; }
__device__ __forceinline__ bool is_one(double a) { return a == 1.0; }
__device__ __forceinline__ bool is_one(cf32 a) { return a.x == 1.f && a.y == 0.f; }
__device__ __forceinline__ bool is_one(cf64 a) { return a.x == 1.0 && a.y == 0.0; }

// element of a real or complex operand, as the output type (a real value
// widened to complex has no imaginary part, so 'C' on it is 'T')
template <class T, class E>
__device__ __forceinline__ T widen_to(E x)
{
    if constexpr (Traits<T>::cplx && !Traits<E>::cplx) return from_real<T>(x);
    else return x;
}

// op 0 'N', 1 'T', 2 'C'
template <class T, int OP>
__device__ __forceinline__ T opv(T v)
{
    if constexpr (OP == 2) return cj(v);
    else return v;
}

__global__ void __launch_bounds__(256) k_gemm_vbatched_check(int ta, int tb, const int* __restrict__ M,
                                                             const int* __restrict__ N, const int* __restrict__ K,
                                                             const int* __restrict__ LDA,
                                                             const int* __restrict__ LDB,
                                                             const int* __restrict__ LDC, int batch,
                                                             int* __restrict__ summary)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= batch) return;
    const int m = M[b], n = N[b], k = K[b];
    if (m < 0 || n < 0 || k < 0) {
        atomicCAS(summary + 3, 0, b + 1);
        return;
    }
    const int lda_need = ta == 0 ? (m > 1 ? m : 1) : (k > 1 ? k : 1);
    const int ldb_need = tb == 0 ? (k > 1 ? k : 1) : (n > 1 ? n : 1);
    const int ldc_need = m > 1 ? m : 1;
    if (LDA[b] < lda_need || LDB[b] < ldb_need || LDC[b] < ldc_need) {
        atomicCAS(summary + 3, 0, b + 1);
        return;
    }
    atomicMax(summary + 0, m);
    atomicMax(summary + 1, n);
    atomicMax(summary + 2, k);
}

template <class T, int TA, int TB, class EA = T, class EB = T>
__global__ void __launch_bounds__(GB_NT) k_gemm_vbatched(const int* __restrict__ M, const int* __restrict__ N,
                                                         const int* __restrict__ K, T alpha,
                                                         const EA* const* __restrict__ A, const int* __restrict__ LDA,
                                                         const EB* const* __restrict__ B, const int* __restrict__ LDB,
                                                         T beta, T* const* __restrict__ C,
                                                         const int* __restrict__ LDC, int batch0)
{
    __shared__ T sA[GB_K][GB_M + 1];
    __shared__ T sB[GB_K][GB_N + 1];
    const int b = batch0 + blockIdx.z;
    const int m = M[b], n = N[b], k = K[b];
    if (m <= 0 || n <= 0 || k < 0) return;
    const int i0 = blockIdx.x * GB_M, j0 = blockIdx.y * GB_N;
    if (i0 >= m || j0 >= n) return;
    T* c = C[b];
    const long long ldc = LDC[b];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;  // rows tx + 16 r, columns ty + 16 q
    if (k == 0 || is_zero(alpha)) {
        if (is_one(beta) || c == nullptr) return;
        for (int p = tid; p < GB_M * GB_N; p += GB_NT) {
            const int i = i0 + (p % GB_M), j = j0 + (p / GB_M);
            if (i < m && j < n) {
                T* e = c + i + j * ldc;
                *e = is_zero(beta) ? zero<T>() : mulv(beta, *e);
            }
        }
        return;
    }
    const EA* a = A[b];
    const EB* bm = B[b];
    if (a == nullptr || bm == nullptr || c == nullptr) return;
    const long long lda = LDA[b], ldb = LDB[b];
    T acc[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[r][q] = zero<T>();
    for (int k0 = 0; k0 < k; k0 += GB_K) {
        // op(A)(i, l): 'N' A[i + l lda], else A[l + i lda] (conjugated for 'C')
#pragma unroll
        for (int r = 0; r < GB_M * GB_K / GB_NT; ++r) {
            const int idx = tid + r * GB_NT;
            const int ii = TA == 0 ? idx % GB_M : idx / GB_K, kk = TA == 0 ? idx / GB_M : idx % GB_K;
            const int gi = i0 + ii, gk = k0 + kk;
            T v = zero<T>();
            if (gi < m && gk < k) v = opv<T, TA>(widen_to<T>(TA == 0 ? a[gi + gk * lda] : a[gk + gi * lda]));
            sA[kk][ii] = v;
        }
        // op(B)(l, j): 'N' B[l + j ldb], else B[j + l ldb] (conjugated for 'C')
#pragma unroll
        for (int r = 0; r < GB_N * GB_K / GB_NT; ++r) {
            const int idx = tid + r * GB_NT;
            const int kk = TB == 0 ? idx % GB_K : idx / GB_N, jj = TB == 0 ? idx / GB_K : idx % GB_N;
            const int gk = k0 + kk, gj = j0 + jj;
            T v = zero<T>();
            if (gk < k && gj < n) v = opv<T, TB>(widen_to<T>(TB == 0 ? bm[gk + gj * ldb] : bm[gj + gk * ldb]));
            sB[kk][jj] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GB_K; ++kk) {
            T av[4], bv[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) av[r] = sA[kk][tx + 16 * r];
#pragma unroll
            for (int q = 0; q < 4; ++q) bv[q] = sB[kk][ty + 16 * q];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[r][q] = fma_(acc[r][q], av[r], bv[q]);
        }
        __syncthreads();
    }
    const bool b0 = is_zero(beta);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = j0 + ty + 16 * q;
        if (j >= n) continue;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int i = i0 + tx + 16 * r;
            if (i >= m) continue;
            T* e = c + i + j * ldc;
            const T v = mulv(alpha, acc[r][q]);
            *e = b0 ? v : add(v, mulv(beta, *e));
        }
    }
}

int op_code(char t)
{
    if (t == 'N' || t == 'n') return 0;
    if (t == 'T' || t == 't') return 1;
    if (t == 'C' || t == 'c') return 2;
    return -1;
}

template <class T, int TA, int TB, class EA = T, class EB = T>
cudaError_t launch_t(int max_m, int max_n, const int* M, const int* N, const int* K, T alpha, const void* A,
                     const int* LDA, const void* B, const int* LDB, T beta, void* C, const int* LDC, int batch,
                     cudaStream_t st)
{
    const dim3 grid0((unsigned)ceil_div(max_m, GB_M), (unsigned)ceil_div(max_n, GB_N));
    if (grid0.y > 65535u) return cudaErrorInvalidValue;  // n above 4 194 240
    int launches = 0;
    for (int b0 = 0; b0 < batch; b0 += 65535) {
        const int nb = batch - b0 < 65535 ? batch - b0 : 65535;
        k_gemm_vbatched<T, TA, TB, EA, EB><<<dim3(grid0.x, grid0.y, (unsigned)nb), GB_NT, 0, st>>>(
            M, N, K, alpha, static_cast<const EA* const*>(A), LDA, static_cast<const EB* const*>(B), LDB, beta,
            static_cast<T* const*>(C), LDC, b0);
        ++launches;
    }
    note_launches(launches);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_typed(int ta, int tb, int max_m, int max_n, const int* M, const int* N, const int* K,
                         const void* alpha, const void* A, const int* LDA, const void* B, const int* LDB,
                         const void* beta, void* C, const int* LDC, int batch, cudaStream_t st)
{
    const T al = *static_cast<const T*>(alpha), be = *static_cast<const T*>(beta);
#define DDLAK_GV(TA_, TB_)                                                                                     \
    if (ta == TA_ && tb == TB_)                                                                                \
        return launch_t<T, TA_, TB_>(max_m, max_n, M, N, K, al, A, LDA, B, LDB, be, C, LDC, batch, st);
    DDLAK_GV(0, 0) DDLAK_GV(0, 1) DDLAK_GV(0, 2)
    DDLAK_GV(1, 0) DDLAK_GV(1, 1) DDLAK_GV(1, 2)
    DDLAK_GV(2, 0) DDLAK_GV(2, 1) DDLAK_GV(2, 2)
#undef DDLAK_GV
    return cudaErrorInvalidValue;
}

// one operand real (R), the other complex (T = complex<R>); 'C' on the real one is 'T'
template <class T, class EA, class EB>
cudaError_t launch_mixed(int ta, int tb, int max_m, int max_n, const int* M, const int* N, const int* K,
                         const void* alpha, const void* A, const int* LDA, const void* B, const int* LDB,
                         const void* beta, void* C, const int* LDC, int batch, cudaStream_t st)
{
    const T al = *static_cast<const T*>(alpha), be = *static_cast<const T*>(beta);
#define DDLAK_GVM(TA_, TB_)                                                                                    \
    if (ta == TA_ && tb == TB_)                                                                                \
        return launch_t<T, TA_, TB_, EA, EB>(max_m, max_n, M, N, K, al, A, LDA, B, LDB, be, C, LDC, batch, st);
    DDLAK_GVM(0, 0) DDLAK_GVM(0, 1) DDLAK_GVM(0, 2)
    DDLAK_GVM(1, 0) DDLAK_GVM(1, 1) DDLAK_GVM(1, 2)
    DDLAK_GVM(2, 0) DDLAK_GVM(2, 1) DDLAK_GVM(2, 2)
#undef DDLAK_GVM
    return cudaErrorInvalidValue;
}

// first entry whose product or scaling needs a matrix that is null (the reference's
// mixed_vbatched_pointer_check, src/BLAS/gemm_mixed.cpp:224-234): bad = 1 + its index
__global__ void __launch_bounds__(256) k_gemm_vbatched_pointers(const int* __restrict__ M, const int* __restrict__ N,
                                                                const int* __restrict__ K,
                                                                const void* const* __restrict__ A,
                                                                const void* const* __restrict__ B,
                                                                void* const* __restrict__ C, int alpha_zero,
                                                                int beta_one, int batch, int* __restrict__ bad)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= batch || M[q] == 0 || N[q] == 0) return;
    const bool product = !alpha_zero && K[q] != 0;
    if (!product && beta_one) return;
    if (!C[q] || (product && (!A[q] || !B[q]))) atomicCAS(bad, 0, q + 1);
}

// the C0 operand of stage 1 must be C0 as stage 0 writes it (the reference's
// mixed_vbatched_stage_check, src/BLAS/gemm_mixed.cpp:236-245): bad = 1 + index
__global__ void __launch_bounds__(256) k_gemm_vbatched_footprint(const int* __restrict__ M0, const int* __restrict__ N0,
                                                                 const int* __restrict__ LDC0,
                                                                 const int* __restrict__ M1, const int* __restrict__ N1,
                                                                 const int* __restrict__ K1,
                                                                 const int* __restrict__ LD1, int left, int trans,
                                                                 int batch, int* __restrict__ bad)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= batch || M1[q] == 0 || N1[q] == 0 || K1[q] == 0) return;
    const int rows = left ? (trans ? K1[q] : M1[q]) : (trans ? N1[q] : K1[q]);
    const int cols = left ? (trans ? M1[q] : K1[q]) : (trans ? K1[q] : N1[q]);
    if (rows != M0[q] || cols != N0[q] || LD1[q] != LDC0[q]) atomicCAS(bad, 0, q + 1);
}

}  // namespace
}  // namespace ddlak

extern "C" int ddlak_gemm_vbatched_footprint(const int* d_m0, const int* d_n0, const int* d_ldc0, const int* d_m1,
                                             const int* d_n1, const int* d_k1, const int* d_ld1, int left, int trans,
                                             int batch, int* d_bad, void* stream)
{
    using namespace ddlak;
    if (batch < 0 || !d_bad) return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(d_bad, 0, sizeof(int), st);
    if (e != cudaSuccess || batch == 0) return (int)e;
    k_gemm_vbatched_footprint<<<(unsigned)ceil_div(batch, 256), 256, 0, st>>>(d_m0, d_n0, d_ldc0, d_m1, d_n1, d_k1,
                                                                              d_ld1, left, trans, batch, d_bad);
    note_launches(1);
    return (int)cudaGetLastError();
}

extern "C" int ddlak_gemm_vbatched_pointers(const int* d_m, const int* d_n, const int* d_k, const void* const* d_A,
                                            const void* const* d_B, void* const* d_C, int alpha_zero, int beta_one,
                                            int batch, int* d_bad, void* stream)
{
    using namespace ddlak;
    if (batch < 0 || !d_bad) return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(d_bad, 0, sizeof(int), st);
    if (e != cudaSuccess || batch == 0) return (int)e;
    k_gemm_vbatched_pointers<<<(unsigned)ceil_div(batch, 256), 256, 0, st>>>(d_m, d_n, d_k, d_A, d_B, d_C, alpha_zero,
                                                                             beta_one, batch, d_bad);
    note_launches(1);
    return (int)cudaGetLastError();
}

extern "C" int ddlak_gemm_vbatched_mixed(char type, int complex_left, char transA, char transB, int max_m, int max_n,
                                         const int* d_m, const int* d_n, const int* d_k, const void* alpha,
                                         const void* d_A, const int* d_lda, const void* d_B, const int* d_ldb,
                                         const void* beta, void* d_C, const int* d_ldc, int batch, void* stream)
{
    using namespace ddlak;
    const int ta = op_code(transA), tb = op_code(transB);
    if (ta < 0 || tb < 0 || batch < 0 || !alpha || !beta) return (int)cudaErrorInvalidValue;
    if (batch == 0 || max_m <= 0 || max_n <= 0) return 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (type == 'c')
        return (int)(complex_left ? launch_mixed<cf32, cf32, float>(ta, tb, max_m, max_n, d_m, d_n, d_k, alpha, d_A,
                                                                     d_lda, d_B, d_ldb, beta, d_C, d_ldc, batch, st)
                                  : launch_mixed<cf32, float, cf32>(ta, tb, max_m, max_n, d_m, d_n, d_k, alpha, d_A,
                                                                     d_lda, d_B, d_ldb, beta, d_C, d_ldc, batch, st));
    if (type == 'z')
        return (int)(complex_left ? launch_mixed<cf64, cf64, double>(ta, tb, max_m, max_n, d_m, d_n, d_k, alpha, d_A,
                                                                      d_lda, d_B, d_ldb, beta, d_C, d_ldc, batch, st)
                                  : launch_mixed<cf64, double, cf64>(ta, tb, max_m, max_n, d_m, d_n, d_k, alpha, d_A,
                                                                      d_lda, d_B, d_ldb, beta, d_C, d_ldc, batch, st));
    return (int)cudaErrorInvalidValue;
}

extern "C" int ddlak_gemm_vbatched_check(char transA, char transB, const int* d_m, const int* d_n, const int* d_k,
                                         const int* d_lda, const int* d_ldb, const int* d_ldc, int batch,
                                         int* d_summary, void* stream)
{
    using namespace ddlak;
    const int ta = op_code(transA), tb = op_code(transB);
    if (ta < 0 || tb < 0 || batch < 0 || !d_summary) return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(d_summary, 0, 4 * sizeof(int), st);
    if (e != cudaSuccess || batch == 0) return (int)e;
    k_gemm_vbatched_check<<<(unsigned)ceil_div(batch, 256), 256, 0, st>>>(ta, tb, d_m, d_n, d_k, d_lda, d_ldb, d_ldc,
                                                                          batch, d_summary);
    note_launches(1);
    return (int)cudaGetLastError();
}

extern "C" int ddlak_gemm_vbatched(char type, char transA, char transB, int max_m, int max_n, const int* d_m,
                                   const int* d_n, const int* d_k, const void* alpha, const void* d_A,
                                   const int* d_lda, const void* d_B, const int* d_ldb, const void* beta, void* d_C,
                                   const int* d_ldc, int batch, void* stream)
{
    using namespace ddlak;
    const int ta = op_code(transA), tb = op_code(transB);
    if (ta < 0 || tb < 0 || batch < 0 || !alpha || !beta) return (int)cudaErrorInvalidValue;
    if (batch == 0 || max_m <= 0 || max_n <= 0) return 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (type) {
    case 's': return (int)launch_typed<float>(ta, tb, max_m, max_n, d_m, d_n, d_k, alpha, d_A, d_lda, d_B, d_ldb, beta,
                                              d_C, d_ldc, batch, st);
    case 'd': return (int)launch_typed<double>(ta, tb, max_m, max_n, d_m, d_n, d_k, alpha, d_A, d_lda, d_B, d_ldb,
                                               beta, d_C, d_ldc, batch, st);
    case 'c': return (int)launch_typed<cf32>(ta, tb, max_m, max_n, d_m, d_n, d_k, alpha, d_A, d_lda, d_B, d_ldb, beta,
                                             d_C, d_ldc, batch, st);
    case 'z': return (int)launch_typed<cf64>(ta, tb, max_m, max_n, d_m, d_n, d_k, alpha, d_A, d_lda, d_B, d_ldb, beta,
                                             d_C, d_ldc, batch, st);
    default: return (int)cudaErrorInvalidValue;
    }
}
