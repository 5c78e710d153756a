// Trailing update of the blocked Cholesky: C -= L21 * L21^H on lower tiles.
//
// This is the work the reference hands to cuSOLVER inside ?potrf
// (src/Cholesky/potrf.cpp:111) and, on multi-rank grids, to herk/gemm
// (src/Cholesky/ppotrf.cpp:212-238).  For double it runs on the FP64 tensor
// cores: mma.sync m8n8k4 f64 (DMMA).  Each CTA owns one 128x128 lower tile,
// streams the two 128 x nbk panel slices through a cp.async double buffer in
// 16-wide k chunks, and keeps its accumulators in registers (8 warps, each a
// 64x32 sub-tile = 8x4 DMMA fragments).  Diagonal tiles store only i >= j.
#include "common.cuh"
#include "ddla_kernels_internal.h"

namespace ddlak {

namespace {

constexpr int DM_BM = 128, DM_BK = 16, DM_LDS = DM_BM + 4;  // 132: conflict-free 8-byte fragment reads
constexpr int DM_STAGE = 2 * DM_BK * DM_LDS;                 // doubles per stage (A and B slices)

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int bytes = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ void tri_tile_idx(long long b, int& I, int& J)
{
    long long i = (long long)((sqrt(8.0 * (double)b + 1.0) - 1.0) * 0.5);
    while ((i + 1) * (i + 2) / 2 <= b) ++i;
    while (i * (i + 1) / 2 > b) --i;
    I = (int)i;
    J = (int)(b - i * (i + 1) / 2);
}

template <bool UP>
__device__ __forceinline__ void load_chunk(double* st, const double* __restrict__ A, long long lda, long long ri,
                                           long long rj, int kcol0, int kc, int nbk, int n)
{
    double* As = st;
    double* Bs = st + DM_BK * DM_LDS;
    // 2 operands x 128 rows x 16 k = 4096 elements, 16 per thread
    for (int idx = threadIdx.x; idx < DM_BM * DM_BK; idx += blockDim.x) {
        int i, k;
        if (UP) { k = idx % DM_BK; i = idx / DM_BK; } else { i = idx % DM_BM; k = idx / DM_BM; }
        const bool kin = kc + k < nbk;
        const long long col = (long long)kcol0 + kc + k;
        {
            const long long r = ri + i;
            const bool v = kin && r < n;
            const double* src = v ? (UP ? A + col + r * lda : A + r + col * lda) : A;
            cp_async8(&As[k * DM_LDS + i], src, v);
        }
        {
            const long long r = rj + i;
            const bool v = kin && r < n;
            const double* src = v ? (UP ? A + col + r * lda : A + r + col * lda) : A;
            cp_async8(&Bs[k * DM_LDS + i], src, v);
        }
    }
}

template <bool UP>
__global__ void __launch_bounds__(256, 1) k_syrk_dmma(double* __restrict__ A, long long lda, int k0, int nbk, int n,
                                                      const int* __restrict__ info)
{
    extern __shared__ __align__(16) double sm[];
    if (*(volatile const int*)info != 0) return;
    int I, J;
    tri_tile_idx(blockIdx.x, I, J);
    const long long t0 = (long long)k0 + nbk;
    const long long ri = t0 + (long long)I * DM_BM, rj = t0 + (long long)J * DM_BM;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = warp >> 2, wn = warp & 3;  // 2 x 4 warps, 64 x 32 each
    const int g = lane >> 2, q = lane & 3;

    double acc[8][4][2];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

    const int nchunks = (nbk + DM_BK - 1) / DM_BK;
    load_chunk<UP>(sm, A, lda, ri, rj, k0, 0, nbk, n);
    cp_async_commit();
    for (int c = 0; c < nchunks; ++c) {
        if (c + 1 < nchunks) load_chunk<UP>(sm + ((c + 1) & 1) * DM_STAGE, A, lda, ri, rj, k0, (c + 1) * DM_BK, nbk, n);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const double* As = sm + (c & 1) * DM_STAGE;
        const double* Bs = As + DM_BK * DM_LDS;
#pragma unroll
        for (int kk = 0; kk < DM_BK; kk += 4) {
            double af[8], bf[4];
#pragma unroll
            for (int a = 0; a < 8; ++a) af[a] = -As[(kk + q) * DM_LDS + wm * 64 + a * 8 + g];
#pragma unroll
            for (int b = 0; b < 4; ++b) bf[b] = Bs[(kk + q) * DM_LDS + wn * 32 + b * 8 + g];
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) dmma(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
        }
        __syncthreads();
    }
    cp_async_wait<0>();

    // epilogue: C += acc (acc already holds -L21*L21^T), lower part only on diagonal tiles
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const long long i = ri + wm * 64 + a * 8 + g;
            const long long j = rj + wn * 32 + b * 8 + 2 * q;
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const long long jj = j + e;
                if (i < n && jj < n && i >= jj) {
                    double* p = UP ? A + jj + i * lda : A + i + jj * lda;
                    *p += acc[a][b][e];
                }
            }
        }
}

template <bool UP>
cudaError_t trailing_update_dmma(double* A, long long lda, int k0, int nbk, int n, const int* dinfo, cudaStream_t st)
{
    const size_t smem = 2 * DM_STAGE * sizeof(double);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_syrk_dmma<UP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    const long long m = (long long)n - k0 - nbk;
    const long long t = ceil_div(m, DM_BM);
    k_syrk_dmma<UP><<<(unsigned)(t * (t + 1) / 2), 256, smem, st>>>(A, lda, k0, nbk, n, dinfo);
    return cudaSuccess;
}

}  // namespace

template <class T, bool UP>
cudaError_t trailing_update(T* A, long long lda, int k0, int nbk, int n, const int* dinfo, cudaStream_t st)
{
    if constexpr (std::is_same<T, double>::value) return trailing_update_dmma<UP>(A, lda, k0, nbk, n, dinfo, st);
    return trailing_update_simt<T, UP>(A, lda, k0, nbk, n, dinfo, st);
}

template cudaError_t trailing_update<float, false>(float*, long long, int, int, int, const int*, cudaStream_t);
template cudaError_t trailing_update<float, true>(float*, long long, int, int, int, const int*, cudaStream_t);
template cudaError_t trailing_update<double, false>(double*, long long, int, int, int, const int*, cudaStream_t);
template cudaError_t trailing_update<double, true>(double*, long long, int, int, int, const int*, cudaStream_t);
template cudaError_t trailing_update<cf32, false>(cf32*, long long, int, int, int, const int*, cudaStream_t);
template cudaError_t trailing_update<cf32, true>(cf32*, long long, int, int, int, const int*, cudaStream_t);
template cudaError_t trailing_update<cf64, false>(cf64*, long long, int, int, int, const int*, cudaStream_t);
template cudaError_t trailing_update<cf64, true>(cf64*, long long, int, int, int, const int*, cudaStream_t);

}  // namespace ddlak
