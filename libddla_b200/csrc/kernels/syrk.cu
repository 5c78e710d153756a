// Trailing update of the blocked Cholesky: C -= L21 * L21^H on lower tiles.
//
// This is the work the reference hands to cuSOLVER inside ?potrf
// (src/Cholesky/potrf.cpp:111) and, on multi-rank grids, to herk/gemm
// (src/Cholesky/ppotrf.cpp:212-238).  For double it runs on the FP64 tensor
// cores: mma.sync m16n8k4 f64 (DMMA).  Each CTA owns one 128x128 lower tile of
// the region, streams the two 128 x nbk panel slices through a 3-stage ring in
// k chunks (cp.async, or TMA boxes), and keeps its accumulators in registers
// (8 warps, each a 64x32 sub-tile = 4x4 DMMA fragments of 16x8).  Diagonal tiles
// store only i >= j.  Complex double runs as two real DMMA products per
// fragment; float and complex float use the SIMT kernel in potrf.cu.
#include <cuda.h>

#include "common.cuh"
#include "ddla_kernels_internal.h"
#include "profile.h"
#include "tc_common.cuh"

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

// D += A B over k = 4 on the FP64 tensor cores, for two 8-row blocks at once
// (mma.sync m16n8k4 f64): lane (g = lane / 4, q = lane % 4) supplies A(g, q) and
// A(g + 8, q) -- the rows of its upper and lower 8-row block -- and B(q, g), and
// holds D(g, 2q + e) in u[e] and D(g + 8, 2q + e) in v[e].  The same fragments as
// two m8n8k4 products on the two blocks, in half the instructions.
__device__ __forceinline__ void dmma2(double (&u)[2], double (&v)[2], double a_up, double a_lo, double b)
{
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
                 : "+d"(u[0]), "+d"(u[1]), "+d"(v[0]), "+d"(v[1])
                 : "d"(a_up), "d"(a_lo), "d"(b));
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
            for (int a = 0; a < 8; a += 2)
#pragma unroll
                for (int b = 0; b < 4; ++b) dmma2(acc[a][b], acc[a + 1][b], af[a], af[a + 1], bf[b]);
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

// ---------------------------------------------------------------------------
// The same update with its operand slices delivered by TMA (lower storage, even
// leading dimension, 16-byte aligned base, K a multiple of 32): per stage one
// thread loads the A rows [ri, ri+132) and the B rows [rj, rj+132) of 32 panel
// columns as two 132 x 32 FP64 boxes (the 4 extra rows pad the leading dimension
// of the shared tile to 132, which keeps the fragment reads conflict free; rows
// past n arrive as zeros), so no thread spends issue slots on per-element copies.
// 3 stages of 66 KB.  No CTA barrier per stage: each warp releases a stage on
// its `empty` mbarrier when done with it, and the loading thread refills the
// stage of chunk c - 1 (long released by the other warps) after its own chunk c,
// so the warps drift freely and the DMMA pipe is not drained once per chunk.
// Every wait is bounded: if one gives up, the CTA records it in g_dmma_status,
// writes NaN into its tile (the factorization then stops at that column block
// with a failed pivot) and waits, bounded, for its copies still in flight
// before it exits.
// ---------------------------------------------------------------------------
constexpr int DT_BK = 32, DT_LDS = 132, DT_NS = 3;
constexpr int DT_BOX = DT_BK * DT_LDS;                                  // doubles per operand box
constexpr unsigned DT_BOX_BYTES = DT_BOX * 8u;                           // 33792
constexpr size_t DT_SMEM = (size_t)DT_NS * 2 * DT_BOX_BYTES + 128;      // + alignment slack

__device__ int g_dmma_status;

template <bool BATCH>  // BATCH: blockIdx.y is the matrix of a batch (3-D map, matrices astride apart)
__global__ void __launch_bounds__(256, 1) k_syrk_dmma_tma(const __grid_constant__ CUtensorMap amap,
                                                          double* __restrict__ A, long long lda, long long astride,
                                                          int k0, int nbk, int n, long long t0, int cols,
                                                          const int* __restrict__ info)
{
    extern __shared__ __align__(128) unsigned char dt_raw[];
    __shared__ __align__(8) uint64_t full[DT_NS], empty[DT_NS];
    const int z = BATCH ? (int)blockIdx.y : 0;
    A += (long long)z * astride;
    info += z;
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
    double* sm = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(dt_raw) + 127) & ~uintptr_t(127));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = warp >> 2, wn = warp & 3;
    const int g = lane >> 2, q = lane & 3;
    const int nchunks = nbk / DT_BK;

    auto issue = [&](int c) {
        const int s = c % DT_NS;
        double* st = sm + (size_t)s * 2 * DT_BOX;
        tc::mbar_expect_tx(&full[s], 2 * DT_BOX_BYTES);
        if (BATCH) {
            tc::tma_load_3d(st, &amap, &full[s], (int)ri, k0 + c * DT_BK, z);
            tc::tma_load_3d(st + DT_BOX, &amap, &full[s], (int)rj, k0 + c * DT_BK, z);
        } else {
            tc::tma_load_2d(st, &amap, &full[s], (int)ri, k0 + c * DT_BK);
            tc::tma_load_2d(st + DT_BOX, &amap, &full[s], (int)rj, k0 + c * DT_BK);
        }
    };
    if (threadIdx.x == 0) {
        for (int s = 0; s < DT_NS; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 256 / 32);  // one arrival per warp
        }
        tc::mbar_fence_init();
        tc::prefetch_tmap(&amap);
        for (int c = 0; c < DT_NS && c < nchunks; ++c) issue(c);
    }
    __syncthreads();

    double acc[8][4][2];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

    bool ok = true;
    int consumed = 0, issued = nchunks < DT_NS ? nchunks : DT_NS;  // issued: thread 0's count
    for (int c = 0; c < nchunks; ++c) {
        const int s = c % DT_NS;
        if (!tc::mbar_wait(&full[s], (uint32_t)((c / DT_NS) & 1), &g_dmma_status, 0x41)) {
            ok = false;
            break;
        }
        consumed = c + 1;
        const double* As = sm + (size_t)s * 2 * DT_BOX;
        const double* Bs = As + DT_BOX;
#pragma unroll
        for (int kk = 0; kk < DT_BK; kk += 4) {
            double af[8], bf[4];
#pragma unroll
            for (int a = 0; a < 8; ++a) af[a] = As[(kk + q) * DT_LDS + wm * 64 + a * 8 + g];
#pragma unroll
            for (int b = 0; b < 4; ++b) bf[b] = Bs[(kk + q) * DT_LDS + wn * 32 + b * 8 + g];
#pragma unroll
            for (int a = 0; a < 8; a += 2)
#pragma unroll
                for (int b = 0; b < 4; ++b) dmma2(acc[a][b], acc[a + 1][b], af[a], af[a + 1], bf[b]);
        }
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&empty[s]);  // this warp is done with stage s
        if (threadIdx.x == 0 && c >= 1 && c - 1 + DT_NS < nchunks) {
            const int cp = c - 1;  // refill chunk cp's stage with chunk cp + NS
            if (!tc::mbar_wait(&empty[cp % DT_NS], (uint32_t)((cp / DT_NS) & 1), &g_dmma_status, 0x44)) {
                ok = false;
                break;
            }
            issue(cp + DT_NS);
            issued = cp + DT_NS + 1;
        }
    }
    ok = __syncthreads_and(ok);
    if (!ok) {
        // copies issued for chunks consumed .. issued - 1 may still be in flight
        if (threadIdx.x == 0) {
            for (int c = consumed; c < issued; ++c)
                (void)tc::mbar_wait(&full[c % DT_NS], (uint32_t)((c / DT_NS) & 1), &g_dmma_status, 0x42);
        }
        __syncthreads();
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = nan;
    }

    // epilogue: C -= acc on the lower part of the region, loads of two fragment rows batched
#pragma unroll
    for (int a2 = 0; a2 < 8; a2 += 2) {
        double cv[2][4][2];
        bool in[2][4][2];
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int b = 0; b < 4; ++b)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const long long i = ri + wm * 64 + (a2 + h) * 8 + g;
                    const long long jj = rj + wn * 32 + b * 8 + 2 * q + e;
                    in[h][b][e] = i < n && jj < cend && i >= jj;
                    cv[h][b][e] = in[h][b][e] ? __ldcg(A + i + jj * lda) : 0.0;
                }
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int b = 0; b < 4; ++b)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    if (!in[h][b][e]) continue;
                    const long long i = ri + wm * 64 + (a2 + h) * 8 + g;
                    const long long jj = rj + wn * 32 + b * 8 + 2 * q + e;
                    A[i + jj * lda] = cv[h][b][e] - acc[a2 + h][b][e];
                }
    }
}

// The TMA variant when its conditions hold; false (nothing launched) otherwise.
bool launch_dmma_tma(double* A, long long lda, int k0, int nbk, int n, long long t0, int cols, const int* dinfo,
                     cudaStream_t st, cudaError_t* err)
{
    if ((lda & 1) || (reinterpret_cast<uintptr_t>(A) & 15) || (t0 & 1) || nbk % DT_BK != 0 || nbk <= 0) return false;
    const long long m = (long long)n - t0;
    if (m <= 0) {
        *err = cudaSuccess;
        return true;
    }
    CUtensorMap amap;
    if (!tc::encode_colmajor_2d(&amap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, A, n, n, lda, DT_LDS, DT_BK,
                                CU_TENSOR_MAP_SWIZZLE_NONE))
        return false;
    if ((*err = smem_optin(k_syrk_dmma_tma<false>, DT_SMEM)) != cudaSuccess) return true;
    const long long t = ceil_div(m, DM_BM);
    const long long grid = cols == 0 ? t * (t + 1) / 2 : t * ceil_div(cols, DM_BM);
    k_syrk_dmma_tma<false><<<(unsigned)grid, 256, DT_SMEM, st>>>(amap, A, lda, 0, k0, nbk, n, t0, cols, dinfo);
    *err = cudaGetLastError();
    return true;
}

}  // namespace

// The same over a batch of equal-order matrices (blockIdx.y = matrix, astride
// elements apart, info per matrix): the region from row / column t0, all of it
// (cols == 0) or its first cols columns.  False (nothing launched) when the TMA
// conditions do not hold.
bool launch_dmma_tma_batched(double* A, long long lda, long long astride, int batch, int k0, int nbk, int n,
                             long long t0, int cols, const int* dinfo, cudaStream_t st, cudaError_t* err)
{
    if ((lda & 1) || (astride & 1) || (reinterpret_cast<uintptr_t>(A) & 15) || (t0 & 1) || nbk % DT_BK != 0 ||
        nbk <= 0 || batch < 1 || batch > 65535)
        return false;
    const long long m = (long long)n - t0;
    if (m <= 0) {
        *err = cudaSuccess;
        return true;
    }
    CUtensorMap amap;
    if (!tc::encode_colmajor_3d(&amap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, A, n, n, lda, batch, astride, DT_LDS, DT_BK))
        return false;
    if ((*err = smem_optin(k_syrk_dmma_tma<true>, DT_SMEM)) != cudaSuccess) return true;
    const long long t = ceil_div(m, DM_BM);
    const dim3 grid((unsigned)(cols == 0 ? t * (t + 1) / 2 : t * ceil_div(cols, DM_BM)), (unsigned)batch);
    k_syrk_dmma_tma<true><<<grid, 256, DT_SMEM, st>>>(amap, A, lda, astride, k0, nbk, n, t0, cols, dinfo);
    *err = cudaGetLastError();
    return true;
}

namespace {

// ---------------------------------------------------------------------------
// Complex double (lower storage) on the FP64 tensor cores.  With K interleaved
// as k' = 2k + c (c = real, imaginary part) and b the conjugated operand,
//   Re C -= sum_k' A'(i, k') B'(k', j),  A'(i, 2k + c) = part c of a(i, k)
//   Im C -= sum_k' A''(i, k') B'(k', j), A''(i, 2k) = Im a(i, k), A''(i, 2k+1) = -Re a(i, k)
// with B'(2k + c, j) = part c of b(j, k): two real DMMA products per fragment
// pair, and one 16-byte shared load of a(i, k) gives a lane both its A' and A''
// values.  Tiles of 64 x 64 complex, 4 warps of 32 x 32, 16 complex k per stage
// by TMA over the matrix seen as 2n x n doubles (rows 2 ri .. 2 ri + 135: the 4
// extra complex rows pad the shared tile), 3 stages, bounded waits as above.
// ---------------------------------------------------------------------------
constexpr int ZT_BM = 64, ZT_BK = 16, ZT_LDS = 2 * (ZT_BM + 4), ZT_NS = 3;  // ZT_LDS in doubles (136)
constexpr int ZT_BOX = ZT_BK * ZT_LDS;
constexpr unsigned ZT_BOX_BYTES = ZT_BOX * 8u;                   // 17408
constexpr size_t ZT_SMEM = (size_t)ZT_NS * 2 * ZT_BOX_BYTES + 128;

__global__ void __launch_bounds__(128) k_herk_zmma_tma(const __grid_constant__ CUtensorMap amap,
                                                       cf64* __restrict__ A, long long lda, int k0, int nbk, int n,
                                                       long long t0, int cols, const int* __restrict__ info)
{
    extern __shared__ __align__(128) unsigned char zt_raw[];
    __shared__ __align__(8) uint64_t full[ZT_NS];
    if (*(volatile const int*)info != 0) return;
    int I, J;
    if (cols == 0) {
        tile_of_tri(blockIdx.x, I, J);
    } else {
        const int nct = (cols + ZT_BM - 1) / ZT_BM;
        J = blockIdx.x % nct;
        I = blockIdx.x / nct;
        if (I < J) return;
    }
    const long long cend = cols == 0 ? (long long)n : t0 + cols;
    const long long ri = t0 + (long long)I * ZT_BM, rj = t0 + (long long)J * ZT_BM;
    double* sm = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(zt_raw) + 127) & ~uintptr_t(127));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = warp >> 1, wn = warp & 1;  // 2 x 2 warps of 32 x 32
    const int g = lane >> 2, q = lane & 3;
    const int nchunks = nbk / ZT_BK;

    auto issue = [&](int c) {
        const int s = c % ZT_NS;
        double* st = sm + (size_t)s * 2 * ZT_BOX;
        tc::mbar_expect_tx(&full[s], 2 * ZT_BOX_BYTES);
        tc::tma_load_2d(st, &amap, &full[s], (int)(2 * ri), k0 + c * ZT_BK);
        tc::tma_load_2d(st + ZT_BOX, &amap, &full[s], (int)(2 * rj), k0 + c * ZT_BK);
    };
    if (threadIdx.x == 0) {
        for (int s = 0; s < ZT_NS; ++s) tc::mbar_init(&full[s], 1);
        tc::mbar_fence_init();
        tc::prefetch_tmap(&amap);
        for (int c = 0; c < ZT_NS && c < nchunks; ++c) issue(c);
    }
    __syncthreads();

    double re[4][4][2], im[4][4][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) re[a][b][0] = re[a][b][1] = im[a][b][0] = im[a][b][1] = 0.0;

    bool ok = true;
    int consumed = 0;
    const int part = q & 1;
    for (int c = 0; c < nchunks; ++c) {
        const int s = c % ZT_NS;
        ok = __syncthreads_and(tc::mbar_wait(&full[s], (uint32_t)((c / ZT_NS) & 1), &g_dmma_status, 0x43));
        if (!ok) break;
        consumed = c + 1;
        const double* As = sm + (size_t)s * 2 * ZT_BOX;
        const double* Bs = As + ZT_BOX;
#pragma unroll
        for (int kk = 0; kk < 2 * ZT_BK; kk += 4) {  // real k' = kk + q, complex k = kk/2 + q/2
            const int kc = kk / 2 + (q >> 1);
            double a1[4], a2[4], bf[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const double2 v = *reinterpret_cast<const double2*>(&As[kc * ZT_LDS + 2 * (wm * 32 + a * 8 + g)]);
                a1[a] = part ? v.y : v.x;   // A'
                a2[a] = part ? -v.x : v.y;  // A''
            }
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const double2 v = *reinterpret_cast<const double2*>(&Bs[kc * ZT_LDS + 2 * (wn * 32 + b * 8 + g)]);
                bf[b] = part ? v.y : v.x;
            }
#pragma unroll
            for (int a = 0; a < 4; a += 2)
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    dmma2(re[a][b], re[a + 1][b], a1[a], a1[a + 1], bf[b]);
                    dmma2(im[a][b], im[a + 1][b], a2[a], a2[a + 1], bf[b]);
                }
        }
        __syncthreads();
        if (threadIdx.x == 0 && c + ZT_NS < nchunks) issue(c + ZT_NS);
    }
    if (!ok) {
        if (threadIdx.x == 0) {
            for (int c = consumed; c < nchunks && c < consumed + ZT_NS; ++c)
                (void)tc::mbar_wait(&full[c % ZT_NS], (uint32_t)((c / ZT_NS) & 1), &g_dmma_status, 0x44);
        }
        __syncthreads();
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) re[a][b][0] = re[a][b][1] = im[a][b][0] = im[a][b][1] = nan;
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        cf64 cv[4][2];
        bool in[4][2];
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const long long i = ri + wm * 32 + a * 8 + g;
                const long long jj = rj + wn * 32 + b * 8 + 2 * q + e;
                in[b][e] = i < n && jj < cend && i >= jj;
                if (in[b][e]) {
                    const double2 v = __ldcg(reinterpret_cast<const double2*>(A + i + jj * lda));
                    cv[b][e] = {v.x, v.y};
                } else {
                    cv[b][e] = {0.0, 0.0};
                }
            }
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                if (!in[b][e]) continue;
                const long long i = ri + wm * 32 + a * 8 + g;
                const long long jj = rj + wn * 32 + b * 8 + 2 * q + e;
                A[i + jj * lda] = cf64{cv[b][e].x - re[a][b][e], cv[b][e].y - im[a][b][e]};
            }
    }
}

bool launch_zmma_tma(cf64* A, long long lda, int k0, int nbk, int n, long long t0, int cols, const int* dinfo,
                     cudaStream_t st, cudaError_t* err)
{
    if ((reinterpret_cast<uintptr_t>(A) & 15) || nbk % ZT_BK != 0 || nbk <= 0) return false;
    const long long m = (long long)n - t0;
    if (m <= 0) {
        *err = cudaSuccess;
        return true;
    }
    CUtensorMap amap;  // the complex matrix as 2n x n doubles, columns 2 lda doubles apart
    if (!tc::encode_colmajor_2d(&amap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, A, 2LL * n, n, 2 * lda, ZT_LDS, ZT_BK,
                                CU_TENSOR_MAP_SWIZZLE_NONE))
        return false;
    if ((*err = smem_optin(k_herk_zmma_tma, ZT_SMEM)) != cudaSuccess) return true;
    const long long t = ceil_div(m, ZT_BM);
    const long long grid = cols == 0 ? t * (t + 1) / 2 : t * ceil_div(cols, ZT_BM);
    k_herk_zmma_tma<<<(unsigned)grid, 128, ZT_SMEM, st>>>(amap, A, lda, k0, nbk, n, t0, cols, dinfo);
    *err = cudaGetLastError();
    return true;
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
        cudaError_t e = cudaSuccess;
        if (vec2 && launch_dmma_tma(A, lda, k0, nbk, n, t0, cols, dinfo, st, &e)) return e;
        if (vec2) return launch_dmma<false, true>(A, lda, k0, nbk, n, t0, cols, dinfo, st);
        return launch_dmma<UP, false>(A, lda, k0, nbk, n, t0, cols, dinfo, st);
    }
    if constexpr (std::is_same<T, cf64>::value && !UP) {
        cudaError_t e = cudaSuccess;
        if (launch_zmma_tma(A, lda, k0, nbk, n, t0, cols, dinfo, st, &e)) return e;
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
