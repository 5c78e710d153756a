// Trailing update of the blocked Cholesky: C -= L21 * L21^H on lower tiles.
//
// This is the work the reference hands to cuSOLVER inside ?potrf
// (src/Cholesky/potrf.cpp:111) and, on multi-rank grids, to herk/gemm
// (src/Cholesky/ppotrf.cpp:212-238).  For double it runs on the FP64 tensor
// cores: mma.sync m8n8k4 f64 (DMMA).  Each CTA owns one 128x128 lower tile of
// the region, streams the two 128 x nbk panel slices through a cp.async
// 3-stage ring in 16-wide k chunks, and keeps its accumulators in registers
// (8 warps, each a 64x32 sub-tile = 8x4 DMMA fragments).  Diagonal tiles store
// only i >= j.  Other types use the SIMT kernel in potrf.cu.
#include "common.cuh"
#include "ddla_kernels_internal.h"
#include "profile.h"

namespace ddlak {

namespace {

constexpr int DM_BM = 128, DM_BK = 16, DM_LDS = DM_BM + 4;  // 132: conflict-free 8-byte fragment reads
constexpr int DM_STAGE = 2 * DM_BK * DM_LDS;                 // doubles per stage (A and B slices)
constexpr int DM_NSTAGE = 3;

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, int bytes)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int bytes)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// One k chunk (16 columns of the panel) of the A rows [ri, ri+128) and the B
// rows [rj, rj+128) into a stage: As[k][i], Bs[k][i].  Rows at or past their
// limit and columns past nbk are zero-filled.  VEC2: two consecutive rows per
// 16-byte copy (lower storage with even lda and a 16-byte aligned base).
template <bool UP, bool VEC2>
__device__ __forceinline__ void load_chunk(double* st, const double* __restrict__ A, long long lda, long long ri,
                                           long long rj, long long alim, long long blim, int kcol0, int kc, int nbk)
{
    double* As = st;
    double* Bs = st + DM_BK * DM_LDS;
    if (VEC2) {
        for (int idx = threadIdx.x; idx < (DM_BM / 2) * DM_BK; idx += blockDim.x) {
            const int i = 2 * (idx % (DM_BM / 2)), k = idx / (DM_BM / 2);
            const bool kin = kc + k < nbk;
            const long long col = (long long)kcol0 + kc + k;
            {
                const long long r = ri + i;
                const int bytes = (kin && r < alim) ? (r + 1 < alim ? 16 : 8) : 0;
                cp_async16(&As[k * DM_LDS + i], bytes ? A + r + col * lda : A, bytes);
            }
            {
                const long long r = rj + i;
                const int bytes = (kin && r < blim) ? (r + 1 < blim ? 16 : 8) : 0;
                cp_async16(&Bs[k * DM_LDS + i], bytes ? A + r + col * lda : A, bytes);
            }
        }
    } else {
        for (int idx = threadIdx.x; idx < DM_BM * DM_BK; idx += blockDim.x) {
            int i, k;
            if (UP) { k = idx % DM_BK; i = idx / DM_BK; } else { i = idx % DM_BM; k = idx / DM_BM; }
            const bool kin = kc + k < nbk;
            const long long col = (long long)kcol0 + kc + k;
            {
                const long long r = ri + i;
                const bool v = kin && r < alim;
                cp_async8(&As[k * DM_LDS + i], v ? (UP ? A + col + r * lda : A + r + col * lda) : A, v ? 8 : 0);
            }
            {
                const long long r = rj + i;
                const bool v = kin && r < blim;
                cp_async8(&Bs[k * DM_LDS + i], v ? (UP ? A + col + r * lda : A + r + col * lda) : A, v ? 8 : 0);
            }
        }
    }
}

template <bool UP, bool VEC2>
__global__ void __launch_bounds__(256, 1) k_syrk_dmma(double* __restrict__ A, long long lda, int k0, int nbk, int n,
                                                      long long t0, int cols, const int* __restrict__ info)
{
    extern __shared__ __align__(16) double sm[];
    if (*(volatile const int*)info != 0) return;
    int I, J;
    if (cols == 0) {
        tile_of_tri(blockIdx.x, I, J);
    } else {
        const int nct = (cols + DM_BM - 1) / DM_BM;
        J = blockIdx.x % nct;
        I = blockIdx.x / nct;
        if (I < J) return;
    }
    const long long cend = cols == 0 ? (long long)n : t0 + cols;
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
#pragma unroll
    for (int s = 0; s < DM_NSTAGE - 1; ++s) {
        if (s < nchunks) load_chunk<UP, VEC2>(sm + s * DM_STAGE, A, lda, ri, rj, n, cend, k0, s * DM_BK, nbk);
        cp_async_commit();
    }
    for (int c = 0; c < nchunks; ++c) {
        const int pre = c + DM_NSTAGE - 1;
        if (pre < nchunks)
            load_chunk<UP, VEC2>(sm + (pre % DM_NSTAGE) * DM_STAGE, A, lda, ri, rj, n, cend, k0, pre * DM_BK, nbk);
        cp_async_commit();
        cp_async_wait<DM_NSTAGE - 1>();
        __syncthreads();
        const double* As = sm + (c % DM_NSTAGE) * DM_STAGE;
        const double* Bs = As + DM_BK * DM_LDS;
#pragma unroll
        for (int kk = 0; kk < DM_BK; kk += 4) {
            double af[8], bf[4];
#pragma unroll
            for (int a = 0; a < 8; ++a) af[a] = As[(kk + q) * DM_LDS + wm * 64 + a * 8 + g];
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

    // epilogue: C -= acc, lower part of the region only.  The C values of two
    // fragment rows (16 per thread) are loaded together before any store, so
    // the loads overlap instead of serialising behind the stores.
#pragma unroll
    for (int a2 = 0; a2 < 8; a2 += 2) {
        double cv[2][4][2];
        bool ok[2][4][2];
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int b = 0; b < 4; ++b)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const long long i = ri + wm * 64 + (a2 + h) * 8 + g;
                    const long long jj = rj + wn * 32 + b * 8 + 2 * q + e;
                    ok[h][b][e] = i < n && jj < cend && i >= jj;
                    cv[h][b][e] = ok[h][b][e] ? __ldcg(UP ? A + jj + i * lda : A + i + jj * lda) : 0.0;
                }
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int b = 0; b < 4; ++b)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    if (!ok[h][b][e]) continue;
                    const long long i = ri + wm * 64 + (a2 + h) * 8 + g;
                    const long long jj = rj + wn * 32 + b * 8 + 2 * q + e;
                    double* p = UP ? A + jj + i * lda : A + i + jj * lda;
                    *p = cv[h][b][e] - acc[a2 + h][b][e];
                }
    }
}

template <bool UP, bool VEC2>
cudaError_t launch_dmma(double* A, long long lda, int k0, int nbk, int n, long long t0, int cols, const int* dinfo,
                        cudaStream_t st)
{
    const size_t smem = DM_NSTAGE * DM_STAGE * sizeof(double);
    if (cudaError_t e = smem_optin(k_syrk_dmma<UP, VEC2>, smem); e != cudaSuccess) return e;
    const long long m = (long long)n - t0;
    if (m <= 0) return cudaSuccess;
    const long long t = ceil_div(m, DM_BM);
    const long long grid = cols == 0 ? t * (t + 1) / 2 : t * ceil_div(cols, DM_BM);
    k_syrk_dmma<UP, VEC2><<<(unsigned)grid, 256, smem, st>>>(A, lda, k0, nbk, n, t0, cols, dinfo);
    return cudaGetLastError();
}

}  // namespace

template <class T, bool UP>
cudaError_t trailing_update(T* A, long long lda, int k0, int nbk, int n, long long t0, int cols, const int* dinfo,
                            cudaStream_t st)
{
    if constexpr (std::is_same<T, double>::value) {
        const bool vec2 = !UP && (lda % 2 == 0) && ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && (t0 % 2 == 0);
        if (vec2) return launch_dmma<false, true>(A, lda, k0, nbk, n, t0, cols, dinfo, st);
        return launch_dmma<UP, false>(A, lda, k0, nbk, n, t0, cols, dinfo, st);
    }
    return trailing_update_simt<T, UP>(A, lda, k0, nbk, n, t0, cols, dinfo, st);
}

#define DDLAK_INST_TU(T, UP)                                                                                        \
    template cudaError_t trailing_update<T, UP>(T*, long long, int, int, int, long long, int, const int*, cudaStream_t);
DDLAK_INST_TU(float, false)
DDLAK_INST_TU(float, true)
DDLAK_INST_TU(double, false)
DDLAK_INST_TU(double, true)
DDLAK_INST_TU(cf32, false)
DDLAK_INST_TU(cf32, true)
DDLAK_INST_TU(cf64, false)
DDLAK_INST_TU(cf64, true)
#undef DDLAK_INST_TU

}  // namespace ddlak
