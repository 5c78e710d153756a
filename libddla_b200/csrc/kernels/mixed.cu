// Mixed-precision Cholesky for ddla::pposv_mixed (no reference counterpart).
//
// The FP64 matrix A (lower) is copied to an FP32 working matrix W; W is
// factored with the blocked right-looking scheme of potrf.cu, but
//   * each diagonal block is factored in FP64 (FP32 storage widened in shared
//     memory, diag_factor.cuh) and rounded back to FP32;
//   * the panel solve runs in FP32 on W (k_trsm_panel<float>);
//   * the panel is packed into a K-contiguous operand copy P (BF16, or FP32
//     rounded to TF32) and the trailing update C -= P_I P_J^T runs on the
//     5th-generation tensor cores: one elected thread issues tcgen05.mma into a
//     128x128 FP32 accumulator in TMEM, operands arrive by TMA (128-byte
//     swizzled, no cluster multicast), and all four warps read the accumulator
//     back with tcgen05.ld for the FP32 read-modify-write of W.
// The FP64 residuals and the refinement live in mixed.cpp / potrs.cu; the
// symmetric residual R = B - A X (FP64, lower-stored A) is here too.
#include <cuda_bf16.h>

#include <mutex>
#include <vector>
#include <type_traits>

#include <ddla_kernels.h>

#include "common.cuh"
#include "ddla_kernels_internal.h"
#include "diag_factor.cuh"
#include "profile.h"
#include "tc_common.cuh"

namespace ddlak {

namespace {

constexpr int MX_NB = 128;  // block width of the mixed factorization (= UMMA tile)

// ---------------------------------------------------------------------------
// A (FP64, lower) -> W (FP32, lower); diagonal scaled by diag_scale;
// colsum[j] += sum_i |A(i,j)| over the full symmetric matrix (for ||A||_inf).
// One CTA per 64x64 lower tile.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_convert_lower(const double* __restrict__ A, long long lda,
                                                       float* __restrict__ W, long long ldw, int n, double diag_scale,
                                                       double* __restrict__ colsum, int jt0)
{
    // jt0 < 0: every lower 64 x 64 tile, one per block (triangle order); jt0 >= 0: the
    // tiles of tile columns jt0 + blockIdx.y, tile row J + blockIdx.x (a column panel)
    int I, J;
    if (jt0 < 0) {
        tile_of_tri(blockIdx.x, I, J);
    } else {
        J = jt0 + (int)blockIdx.y;
        I = J + (int)blockIdx.x;
        if ((long long)I * 64 >= n) return;
    }
    const long long ri = (long long)I * 64, rj = (long long)J * 64;
    __shared__ double csw[8][16];   // per warp: column sums of its 32 rows
    __shared__ double rsum[4][64];
    const int r = threadIdx.x & 63, cg = threadIdx.x >> 6;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double rs = 0.0;
    double vals[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
        const long long i = ri + r, j = rj + cg + 4 * u;
        vals[u] = (i < n && j < n && i >= j) ? A[i + j * lda] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 16; ++u) {
        const long long i = ri + r, j = rj + cg + 4 * u;
        const double a = vals[u];
        if (i < n && j < n && i >= j) {
            W[i + j * ldw] = (float)(i == j ? a * diag_scale : a);
            if (i != j) rs += fabs(a);
        }
        // column cg + 4u: sum of |a| over this warp's 32 rows
        double v = fabs(a);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) csw[warp][u] = v;
    }
    rsum[cg][r] = rs;
    __syncthreads();
    if (threadIdx.x < 64) {
        const int t = threadIdx.x, tcg = t & 3, tu = t >> 2;  // column t = tcg + 4 tu
        const double cs = csw[2 * tcg][tu] + csw[2 * tcg + 1][tu];
        if (rj + t < n && cs != 0.0) atomicAdd(&colsum[rj + t], cs);
        const double rt = rsum[0][t] + rsum[1][t] + rsum[2][t] + rsum[3][t];
        if (ri + t < n && rt != 0.0) atomicAdd(&colsum[ri + t], rt);
    }
}

// out[0] = max(v[0..n)), v >= 0
__global__ void __launch_bounds__(256) k_max_nonneg(const double* __restrict__ v, int n, double* out)
{
    double m = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = fmax(m, v[i]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<unsigned long long*>(out), __double_as_longlong(m));
}

// ---------------------------------------------------------------------------
// diagonal block: FP32 storage, FP64 arithmetic
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_potrf_diag_mixed(float* __restrict__ W, long long ldw, int k0, int nbk,
                                                          int* __restrict__ info)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* s = reinterpret_cast<double*>(smem_raw);
    const int ld = diag_block_ld<double>(nbk);
    if (*(volatile int*)info != 0) return;
    const int total = nbk * nbk;
    const float* Wb = W + k0 + (long long)k0 * ldw;
    if (nbk == 128) {
        // the full block by float4 columns (ldw and k0 are multiples of 4): 32 per column,
        // consecutive threads down a column; groups wholly above the diagonal are skipped
#pragma unroll 4
        for (int idx = threadIdx.x; idx < 128 * 32; idx += 256) {
            const int q = idx & 31, j = idx >> 5;
            if (4 * q + 3 < j) continue;
            const float4 v = *reinterpret_cast<const float4*>(Wb + 4 * q + (long long)j * ldw);
            double* d = s + 4 * q + j * ld;
            d[0] = v.x;
            d[1] = v.y;
            d[2] = v.z;
            d[3] = v.w;
        }
    } else {
        for (int base = 0; base < total; base += 16 * 256) {
            float v[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                const int idx = base + u * 256 + threadIdx.x;
                const int i = idx % nbk, j = idx / nbk;
                v[u] = (idx < total && i >= j) ? Wb[i + (long long)j * ldw] : 0.f;
            }
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                const int idx = base + u * 256 + threadIdx.x;
                if (idx < total) s[(idx % nbk) + (idx / nbk) * ld] = (double)v[u];
            }
        }
    }
    __syncthreads();
    const int fail = factor_block_smem<double>(s, ld, nbk);
    if (nbk == 128) {
        // float4 stores of the lower part; a group crossing the diagonal keeps its upper entries
        for (int idx = threadIdx.x; idx < 128 * 32; idx += 256) {
            const int q = idx & 31, j = idx >> 5;
            if (4 * q + 3 < j) continue;
            float* dst = W + k0 + 4 * q + (long long)(k0 + j) * ldw;
            const double* src = s + 4 * q + j * ld;
            if (4 * q >= j) {
                *reinterpret_cast<float4*>(dst) = make_float4((float)src[0], (float)src[1], (float)src[2], (float)src[3]);
            } else {
                for (int e = 0; e < 4; ++e)
                    if (4 * q + e >= j) dst[e] = (float)src[e];
            }
        }
    } else {
        for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
            const int i = idx % nbk, j = idx / nbk;
            if (i >= j) W[(k0 + i) + (long long)(k0 + j) * ldw] = (float)s[i + j * ld];
        }
    }
    if (fail && threadIdx.x == 0) *info = k0 + fail;
}

// ---------------------------------------------------------------------------
// panel rows [pr0, n) x columns [k0, k0+nbk) of W -> P, K-contiguous with row
// stride ldp: P[r*ldp + k] = round(W[(pr0+r) + (k0+k)*ldw]) (BF16, or FP32
// rounded to TF32)
// ---------------------------------------------------------------------------
template <bool TF32>
__global__ void __launch_bounds__(256) k_pack_panel(const float* __restrict__ W, long long ldw, int n, long long pr0,
                                                    int k0, int nbk, void* __restrict__ P, long long ldp,
                                                    const int* __restrict__ info)
{
    __shared__ float t[32][33];
    if (*(volatile int*)info != 0) return;
    const long long r0 = (long long)blockIdx.x * 32;
    const int kk0 = blockIdx.y * 32;
    for (int y = threadIdx.y; y < 32; y += 8) {
        const long long row = pr0 + r0 + threadIdx.x;
        t[y][threadIdx.x] = row < n ? W[row + (long long)(k0 + kk0 + y) * ldw] : 0.f;
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += 8) {
        const long long r = r0 + y;
        if (pr0 + r >= n) continue;
        const float x = t[threadIdx.x][y];
        const long long off = r * ldp + kk0 + threadIdx.x;
        if (TF32) {
            uint32_t b;
            asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(b) : "f"(x));
            reinterpret_cast<uint32_t*>(P)[off] = b;
        } else {
            reinterpret_cast<__nv_bfloat16*>(P)[off] = __float2bfloat16_rn(x);
        }
    }
}

// ---------------------------------------------------------------------------
// tcgen05 trailing update: W(i,j) -= sum_k P(i-pr0, k) P(j-pr0, k) on the lower
// entries of one 128x128 tile of the region (rows [t0,n), cols [t0,n) or
// [t0, t0+cols)).  128 threads: thread 0 issues TMA, thread 32 issues MMA,
// all four warps run the epilogue on their 32 TMEM lanes.
// ---------------------------------------------------------------------------
constexpr int MU_STAGES = 2;  // 3 stages measured no faster, 4 slower (one CTA per SM)
constexpr int MU_TILE_BYTES = 128 * 128;  // 128 rows x 128 bytes
constexpr size_t MU_SMEM = (size_t)MU_STAGES * 2 * MU_TILE_BYTES + 1024;

enum : int { MU_ERR_EMPTY = 0x21, MU_ERR_FULL = 0x22, MU_ERR_DONE = 0x23, MU_ERR_CTILE = 0x24 };

template <bool TF32>
__global__ void __launch_bounds__(128, 3) k_mixed_update(const __grid_constant__ CUtensorMap pmap,
                                                         const __grid_constant__ CUtensorMap wmap,
                                                         float* __restrict__ W, long long ldw, int n, long long t0,
                                                         long long pr0, int cols, int nkb,
                                                         const int* __restrict__ info, int* __restrict__ status)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[MU_STAGES], empty[MU_STAGES], done, cbar;
    __shared__ uint32_t s_tmem;
    if (*(volatile const int*)info != 0) return;
    int I, J;
    if (cols == 0) {
        tile_of_tri(blockIdx.x, I, J);
    } else {
        const int nct = (cols + 127) / 128;
        J = blockIdx.x % nct;
        I = blockIdx.x / nct;
        if (I < J) return;
    }
    const long long ri = t0 + (long long)I * 128, rj = t0 + (long long)J * 128;
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < MU_STAGES; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        tc::mbar_init(&done, 1);
        tc::mbar_init(&cbar, 1);
        tc::mbar_fence_init();
    }
    if (warp == 0) tc::tmem_alloc(&s_tmem, 128);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = s_tmem;

    if (threadIdx.x == 0) {
        tc::prefetch_tmap(&pmap);
        // the panel is read by every tile of its row and column: keep it in L2 ahead of the
        // W tiles, which stream through once (evict_first on their load and store)
        const uint64_t keep = tc::l2_policy_evict_last();
        for (int kb = 0; kb < nkb; ++kb) {
            const int s = kb % MU_STAGES;
            if (kb >= MU_STAGES && !tc::mbar_wait(&empty[s], ((kb / MU_STAGES) - 1) & 1, status, MU_ERR_EMPTY)) break;
            unsigned char* sa = base + (size_t)s * 2 * MU_TILE_BYTES;
            tc::mbar_expect_tx(&full[s], 2 * MU_TILE_BYTES);
            const int x = kb * (TF32 ? 32 : 64);
            tc::tma_load_2d_hint(sa, &pmap, &full[s], x, (int)(ri - pr0), keep);
            tc::tma_load_2d_hint(sa + MU_TILE_BYTES, &pmap, &full[s], x, (int)(rj - pr0), keep);
        }
    } else if (threadIdx.x == 32) {
        constexpr uint32_t idesc = tc::idesc_m128_n128<TF32>();
        bool ok = true;
        for (int kb = 0; kb < nkb && ok; ++kb) {
            const int s = kb % MU_STAGES;
            ok = tc::mbar_wait(&full[s], (kb / MU_STAGES) & 1, status, MU_ERR_FULL);
            if (!ok) break;
            tc::tc_fence_after();
            const unsigned char* sa = base + (size_t)s * 2 * MU_TILE_BYTES;
            const uint64_t ad = tc::smem_desc_sw128(sa), bd = tc::smem_desc_sw128(sa + MU_TILE_BYTES);
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)  // four K steps of 32 bytes per 128-byte row
                tc::umma<TF32>(tmem, ad + 2 * kk, bd + 2 * kk, idesc, (kb | kk) != 0 ? 1u : 0u);
            tc::umma_commit(&empty[s]);
        }
        tc::umma_commit(&done);
    }
    __syncwarp();

    // epilogue: once the MMAs are done the operand stages are free; the 128 x 128
    // FP32 tile of W comes in by TMA (64 KB, one request), the accumulator is
    // subtracted in shared memory and the tile goes back by a TMA bulk store.
    // Out-of-range rows and columns are zero-filled on the load and clipped on
    // the store; the upper triangle of a diagonal tile is written too (W's upper
    // triangle is scratch nothing reads).
    bool ok = tc::mbar_wait(&done, 0, status, MU_ERR_DONE);
    ok = __all_sync(0xffffffffu, ok);
    tc::tc_fence_after();
    float* ct = reinterpret_cast<float*>(base);  // [128 cols][128 rows]
    if (__syncthreads_and(ok)) {
        if (threadIdx.x == 0) {
            tc::mbar_expect_tx(&cbar, 128 * 128 * 4);
            tc::tma_load_2d_hint(ct, &wmap, &cbar, (int)ri, (int)rj, tc::l2_policy_evict_first());
        }
        ok = tc::mbar_wait(&cbar, 0, status, MU_ERR_CTILE);
        ok = __all_sync(0xffffffffu, ok);
        if (ok) {
            const int r = 32 * warp + lane;
#pragma unroll 1
            for (int c = 0; c < 4; ++c) {
                float v[32];
                tc::tmem_ld_32x32b_x32(tmem + ((uint32_t)(32 * warp) << 16) + 32 * c, v);
#pragma unroll
                for (int e = 0; e < 32; ++e) ct[(32 * c + e) * 128 + r] -= v[e];
            }
            tc::fence_proxy_async_smem();
        }
        if (__syncthreads_and(ok) && threadIdx.x == 0) {
            tc::tma_store_2d_hint(&wmap, ct, (int)ri, (int)rj, tc::l2_policy_evict_first());
            tc::tma_store_wait_read();
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, 128);
    }
}

// ---------------------------------------------------------------------------
// The same update over the whole region from t0 by pairs of tiles (I, 2P) and
// (I, 2P + 1) of one tile row: one 128 x 256 MMA accumulator (TMEM columns
// 0..255), the A rows loaded once for both tiles, so each C tile costs 3/4 of
// the operand bytes of the single-tile kernel; two CTAs per SM (96 KB of
// operand stages each).  The epilogue runs the two C tiles one after the other
// through the freed stages; a pair whose second tile lies above the diagonal
// computes it (the MMA is 256 wide) but neither loads nor stores it.
// ---------------------------------------------------------------------------
constexpr int MP_STAGES = 2;
constexpr int MP_STAGE_BYTES = 3 * MU_TILE_BYTES;  // A (128 rows) + B (256 rows) of 128 bytes
constexpr size_t MP_SMEM = (size_t)MP_STAGES * MP_STAGE_BYTES + 1024;

// first pair of tile row I: rows 0..I-1 hold floor(i / 2) + 1 pairs each
__host__ __device__ __forceinline__ long long pair_start(long long I)
{
    return (I & 1) ? ((I + 1) / 2) * ((I + 1) / 2) : (I / 2) * (I / 2 + 1);
}
__host__ __device__ __forceinline__ void pair_of(long long b, int& I, int& P)
{
    long long i = (long long)(2.0 * sqrt((double)b)) - 1;
    if (i < 0) i = 0;
    while (pair_start(i + 1) <= b) ++i;
    while (i > 0 && pair_start(i) > b) --i;
    I = (int)i;
    P = (int)(b - pair_start(i));
}

// The C tiles one CTA of a whole-region update writes: tile row `row`, tile
// columns col0 .. col0 + ntiles - 1 (128-wide tiles from the region's start).
struct UpdateTiles {
    long long row, col0;
    int ntiles;
};
// pair CTA b: tiles (I, 2P) and, when it lies on or below the diagonal, (I, 2P + 1)
__host__ __device__ __forceinline__ UpdateTiles pair_tiles(long long b)
{
    int I, P;
    pair_of(b, I, P);
    return {I, 2LL * P, (2 * P + 1 <= I) ? 2 : 1};
}

template <bool TF32>
__global__ void __launch_bounds__(128, 2) k_mixed_update_pair(const __grid_constant__ CUtensorMap pmap,
                                                              const __grid_constant__ CUtensorMap wmap, int n,
                                                              long long t0, long long pr0, int nkb,
                                                              const int* __restrict__ info, int* __restrict__ status)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[MP_STAGES], empty[MP_STAGES], done, cbar;
    __shared__ uint32_t s_tmem;
    if (*(volatile const int*)info != 0) return;
    const UpdateTiles tl = pair_tiles(blockIdx.x);
    const long long ri = t0 + tl.row * 128, rj = t0 + tl.col0 * 128;
    const int halves = tl.ntiles;
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < MP_STAGES; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        tc::mbar_init(&done, 1);
        tc::mbar_init(&cbar, 1);
        tc::mbar_fence_init();
    }
    if (warp == 0) tc::tmem_alloc(&s_tmem, 256);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = s_tmem;

    if (threadIdx.x == 0) {
        tc::prefetch_tmap(&pmap);
        const uint64_t keep = tc::l2_policy_evict_last();
        for (int kb = 0; kb < nkb; ++kb) {
            const int s = kb % MP_STAGES;
            if (kb >= MP_STAGES && !tc::mbar_wait(&empty[s], ((kb / MP_STAGES) - 1) & 1, status, MU_ERR_EMPTY)) break;
            unsigned char* sa = base + (size_t)s * MP_STAGE_BYTES;
            tc::mbar_expect_tx(&full[s], MP_STAGE_BYTES);
            const int x = kb * (TF32 ? 32 : 64);
            tc::tma_load_2d_hint(sa, &pmap, &full[s], x, (int)(ri - pr0), keep);
            tc::tma_load_2d_hint(sa + MU_TILE_BYTES, &pmap, &full[s], x, (int)(rj - pr0), keep);
            tc::tma_load_2d_hint(sa + 2 * MU_TILE_BYTES, &pmap, &full[s], x, (int)(rj + 128 - pr0), keep);
        }
    } else if (threadIdx.x == 32) {
        constexpr uint32_t idesc = tc::idesc_m128_n256<TF32>();
        bool ok = true;
        for (int kb = 0; kb < nkb && ok; ++kb) {
            const int s = kb % MP_STAGES;
            ok = tc::mbar_wait(&full[s], (kb / MP_STAGES) & 1, status, MU_ERR_FULL);
            if (!ok) break;
            tc::tc_fence_after();
            const unsigned char* sa = base + (size_t)s * MP_STAGE_BYTES;
            const uint64_t ad = tc::smem_desc_sw128(sa), bd = tc::smem_desc_sw128(sa + MU_TILE_BYTES);
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)  // four K steps of 32 bytes per 128-byte row
                tc::umma<TF32>(tmem, ad + 2 * kk, bd + 2 * kk, idesc, (kb | kk) != 0 ? 1u : 0u);
            tc::umma_commit(&empty[s]);
        }
        tc::umma_commit(&done);
    }
    __syncwarp();

    // epilogue: the two C tiles in turn through the freed stages (64 KB each)
    bool ok = tc::mbar_wait(&done, 0, status, MU_ERR_DONE);
    ok = __all_sync(0xffffffffu, ok);
    tc::tc_fence_after();
    float* ct = reinterpret_cast<float*>(base);  // [128 cols][128 rows]
    const uint64_t stream_once = tc::l2_policy_evict_first();
    for (int h = 0; h < halves; ++h) {
        if (!__syncthreads_and(ok)) break;
        if (threadIdx.x == 0) {
            if (h > 0) tc::tma_store_wait_read();  // the first tile's store has left the buffer
            tc::mbar_expect_tx(&cbar, 128 * 128 * 4);
            tc::tma_load_2d_hint(ct, &wmap, &cbar, (int)ri, (int)(rj + 128 * h), stream_once);
        }
        ok = tc::mbar_wait(&cbar, (uint32_t)h, status, MU_ERR_CTILE);
        ok = __all_sync(0xffffffffu, ok);
        if (ok) {
            const int r = 32 * warp + lane;
#pragma unroll 1
            for (int c = 0; c < 4; ++c) {
                float v[32];
                tc::tmem_ld_32x32b_x32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(128 * h + 32 * c), v);
#pragma unroll
                for (int e = 0; e < 32; ++e) ct[(32 * c + e) * 128 + r] -= v[e];
            }
            tc::fence_proxy_async_smem();
        }
        if (__syncthreads_and(ok) && threadIdx.x == 0)
            tc::tma_store_2d_hint(&wmap, ct, (int)ri, (int)(rj + 128 * h), stream_once);
    }
    if (threadIdx.x == 0) tc::tma_store_wait_read();
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, 256);
    }
}

// ---------------------------------------------------------------------------
// The same update over the whole region from t0 by 256 x 256 blocks (I2, J2),
// J2 <= I2, on CTA pairs: a cluster of two CTAs runs one 256 x 256 MMA
// (tcgen05 cta_group::2).  CTA v of the pair loads rows
// 128 v .. 128 v + 127 of the block's A rows and of its B rows, holds the
// 128 x 256 accumulator of its A rows in its own TMEM and writes their C tiles.
// Each C tile costs half the operand bytes of the single-tile kernel, and with
// 256 TMEM columns and 96 KB of stages per CTA two CTAs share an SM, so one
// CTA's C-tile epilogue runs under the other's MMAs.  Both CTAs always run the
// whole protocol (no early exit on a failed pivot): the leader counts the
// peer's operand bytes on its own barriers and the MMA completions arrive on
// both CTAs' barriers, so neither may leave while the other can still signal it.
// ---------------------------------------------------------------------------
constexpr long long MC_MIN_TILES = 32;  // smaller regions keep the pair kernel (more CTAs)

// block b of the lower triangle of 256-blocks, row by row: rows 0..I2-1 hold I2 (I2 + 1) / 2
__host__ __device__ __forceinline__ void block256_of(long long b, int& I2, int& J2)
{
    long long i = (long long)((sqrt(8.0 * (double)b + 1.0) - 1.0) * 0.5);
    while (i > 0 && i * (i + 1) / 2 > b) --i;
    while ((i + 1) * (i + 2) / 2 <= b) ++i;
    I2 = (int)i;
    J2 = (int)(b - i * (i + 1) / 2);
}
// CTA c of the CTA-pair update over t tile rows: block c / 2, rows 128 (c mod 2)
// .. of it (c mod 2 is the CTA's rank in its cluster); its tiles (row, 2 J2) and
// (row, 2 J2 + 1) where they lie on or below the diagonal, none past the last row
// the form of a whole-region update over t tile rows: 2 CTA pairs, 1 tile pairs,
// 0 single tiles; *ctas its grid
inline int region_update_kind(long long t, long long* ctas)
{
    const long long t2 = (t + 1) / 2;
    const int kind = t >= MC_MIN_TILES ? 2 : (t >= 4 ? 1 : 0);
    *ctas = kind == 2 ? t2 * (t2 + 1) : (kind == 1 ? pair_start(t) : t * (t + 1) / 2);
    return kind;
}
__host__ __device__ __forceinline__ UpdateTiles cta2_tiles(long long c, long long t)
{
    int I2, J2;
    block256_of(c >> 1, I2, J2);
    const long long row = 2LL * I2 + (c & 1);
    return {row, 2LL * J2, row >= t ? 0 : (2LL * J2 + 1 <= row ? 2 : 1)};
}

constexpr int MC_STAGES = 3;
constexpr int MC_STAGE_BYTES = 2 * MU_TILE_BYTES;  // this CTA's 128 A rows + 128 B rows of 128 bytes
constexpr size_t MC_SMEM = (size_t)MC_STAGES * MC_STAGE_BYTES + 1024;
static_assert(MC_STAGES * MC_STAGE_BYTES >= 128 * 128 * 4, "the stages hold one FP32 C tile");

template <bool TF32>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(128, 2)
    k_mixed_update_cta2(const __grid_constant__ CUtensorMap pmap, const __grid_constant__ CUtensorMap wmap,
                        long long t0, long long pr0, int t, int nkb, int* __restrict__ status)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[MC_STAGES], empty[MC_STAGES], done, cbar;
    __shared__ uint32_t s_tmem;
    const uint32_t v = tc::cluster_ctarank();  // 0: the leader, which issues the MMAs
    const UpdateTiles tl = cta2_tiles(blockIdx.x, t);  // blockIdx.x mod 2 == v (clusters of 2 along x)
    const long long ri = t0 + tl.row * 128, rj = t0 + tl.col0 * 128;
    const int halves = tl.ntiles;
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < MC_STAGES; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        tc::mbar_init(&done, 1);
        tc::mbar_init(&cbar, 1);
        tc::mbar_fence_init();
    }
    if (warp == 0) tc::tmem_alloc_pair(&s_tmem, 256);
    tc::tc_fence_before();
    tc::cluster_sync();  // both CTAs' barriers initialised and their TMEM allocated
    tc::tc_fence_after();
    const uint32_t tmem = s_tmem;

    if (threadIdx.x == 0) {
        tc::prefetch_tmap(&pmap);
        const uint64_t keep = tc::l2_policy_evict_last();
        bool ok = true;
        int issued = 0;
        for (int kb = 0; kb < nkb; ++kb) {
            const int s = kb % MC_STAGES;
            if (kb >= MC_STAGES && !(ok = tc::mbar_wait(&empty[s], ((kb / MC_STAGES) - 1) & 1, status, MU_ERR_EMPTY)))
                break;
            unsigned char* sa = base + (size_t)s * MC_STAGE_BYTES;
            const uint32_t fb = tc::mapa_shared(tc::smem_u32(&full[s]), 0);
            if (v == 0) tc::mbar_expect_tx(&full[s], 2 * MC_STAGE_BYTES);  // both CTAs' bytes
            const int x = kb * (TF32 ? 32 : 64);
            tc::tma_load_2d_pair(sa, &pmap, fb, x, (int)(ri - pr0), keep);
            tc::tma_load_2d_pair(sa + MU_TILE_BYTES, &pmap, fb, x, (int)(rj + 128 * v - pr0), keep);
            issued = kb + 1;
        }
        // every release of this CTA's stages has arrived before it may leave
        for (int kb = issued > MC_STAGES ? issued - MC_STAGES : 0; ok && kb < issued; ++kb)
            ok = tc::mbar_wait(&empty[kb % MC_STAGES], (kb / MC_STAGES) & 1, status, MU_ERR_EMPTY);
    } else if (threadIdx.x == 32 && v == 0) {
        constexpr uint32_t idesc = tc::idesc_m256_n256<TF32>();
        bool ok = true;
        for (int kb = 0; kb < nkb && ok; ++kb) {
            const int s = kb % MC_STAGES;
            ok = tc::mbar_wait(&full[s], (kb / MC_STAGES) & 1, status, MU_ERR_FULL);
            if (!ok) break;
            tc::tc_fence_after();
            const unsigned char* sa = base + (size_t)s * MC_STAGE_BYTES;
            const uint64_t ad = tc::smem_desc_sw128(sa), bd = tc::smem_desc_sw128(sa + MU_TILE_BYTES);
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)  // four K steps of 32 bytes per 128-byte row
                tc::umma_pair<TF32>(tmem, ad + 2 * kk, bd + 2 * kk, idesc, (kb | kk) != 0 ? 1u : 0u);
            tc::umma_commit_pair(&empty[s]);
        }
        tc::umma_commit_pair(&done);
    }
    __syncwarp();

    // epilogue: this CTA's C tiles in turn through its freed stages (64 KB each)
    bool ok = tc::mbar_wait(&done, 0, status, MU_ERR_DONE);
    ok = __all_sync(0xffffffffu, ok);
    tc::tc_fence_after();
    float* ct = reinterpret_cast<float*>(base);  // [128 cols][128 rows]
    const uint64_t stream_once = tc::l2_policy_evict_first();
    for (int h = 0; h < halves; ++h) {
        if (!__syncthreads_and(ok)) break;
        if (threadIdx.x == 0) {
            if (h > 0) tc::tma_store_wait_read();  // the first tile's store has left the buffer
            tc::mbar_expect_tx(&cbar, 128 * 128 * 4);
            tc::tma_load_2d_hint(ct, &wmap, &cbar, (int)ri, (int)(rj + 128 * h), stream_once);
        }
        ok = tc::mbar_wait(&cbar, (uint32_t)h, status, MU_ERR_CTILE);
        ok = __all_sync(0xffffffffu, ok);
        if (ok) {
            const int r = 32 * warp + lane;
#pragma unroll 1
            for (int c = 0; c < 4; ++c) {
                float vv[32];
                tc::tmem_ld_32x32b_x32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(128 * h + 32 * c), vv);
#pragma unroll
                for (int e = 0; e < 32; ++e) ct[(32 * c + e) * 128 + r] -= vv[e];
            }
            tc::fence_proxy_async_smem();
        }
        if (__syncthreads_and(ok) && threadIdx.x == 0)
            tc::tma_store_2d_hint(&wmap, ct, (int)ri, (int)(rj + 128 * h), stream_once);
    }
    if (threadIdx.x == 0) tc::tma_store_wait_read();
    tc::tc_fence_before();
    tc::cluster_sync();  // neither CTA frees TMEM or leaves while the pair is still working
    if (warp == 0) {
        tc::tc_fence_after();
        tc::tmem_dealloc_pair(tmem, 256);
    }
}

// ---------------------------------------------------------------------------
// R = B - A X for symmetric A stored in its lower triangle (FP64), NC (8 or 16)
// right-hand sides per chunk (grid.y).  Every lower tile A(I, J), I >= J, is
// read from HBM once and used twice: A(I,J) X(J) goes to R(I) and A(I,J)^T X(I)
// to R(J).  CTA (J, c) walks tiles I = J + c*SR_CPT .. of column strip J through
// a double-buffered cp.async ring: the first product is folded into R(I) with
// atomics after each tile, the second accumulates in registers and is folded
// into R(J) at the end (R holds B on entry).  The tile is stored rotated,
// element (r, col) at T[col][(r + col) mod 64], so both the row walk of the
// first product and the column walk of the second are conflict free.  The
// atomics make the last bits of R depend on the order the tiles finish.
// ---------------------------------------------------------------------------
constexpr int SR = 64;
constexpr int SR_CPT = 8;  // tiles per CTA

template <int NC>
constexpr size_t symm_residual_smem()
{
    return sizeof(double) * (2 * SR * SR + 3 * SR * (NC + 1));
}

template <int NC>
__global__ void __launch_bounds__(256) k_symm_residual(const double* __restrict__ A, long long lda, int n, int nrhs,
                                                       const double* __restrict__ X, long long ldx,
                                                       double* __restrict__ R, long long ldr, int chunks)
{
    constexpr int QN = NC / 4;  // columns per thread
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* Tb = reinterpret_cast<double*>(smem_raw);                       // [2][SR cols][SR]
    double (*XJ)[NC + 1] = reinterpret_cast<double (*)[NC + 1]>(Tb + 2 * SR * SR);
    double (*XI)[SR][NC + 1] = reinterpret_cast<double (*)[SR][NC + 1]>(Tb + 2 * SR * SR + SR * (NC + 1));
    const int N = (int)ceil_div(n, SR);
    const int J = blockIdx.x / chunks, c = blockIdx.x % chunks;
    if (J >= N) return;
    const int tbeg = J + c * SR_CPT;
    if (tbeg >= N) return;
    const int tend = (tbeg + SR_CPT) < N ? (tbeg + SR_CPT) : N;
    const long long j0 = (long long)J * SR;
    const int ncols = (int)((n - j0) < SR ? (n - j0) : SR);
    const int r0 = blockIdx.y * NC;
    const int nr = nrhs - r0 < NC ? nrhs - r0 : NC;
    const int tr = threadIdx.x & 63, tg = threadIdx.x >> 6;

    auto issue = [&](int I, int buf) {
        const long long i0 = (long long)I * SR;
        const int nrows = (int)((n - i0) < SR ? (n - i0) : SR);
        double* T = Tb + buf * SR * SR;
        for (int idx = threadIdx.x; idx < SR * SR; idx += blockDim.x) {
            const int r = idx & 63, col = idx >> 6;
            const bool valid = r < nrows && col < ncols && (I != J || r >= col);
            cp_async_elem<8>(&T[col * SR + ((r + col) & 63)], valid ? A + (i0 + r) + (j0 + col) * lda : A, valid);
        }
        for (int idx = threadIdx.x; idx < SR * NC; idx += blockDim.x) {
            const int k = idx % SR, q = idx / SR;
            const bool valid = k < nrows && q < nr;
            cp_async_elem<8>(&XI[buf][k][q], valid ? X + (i0 + k) + (r0 + q) * ldx : X, valid);
        }
    };
    for (int idx = threadIdx.x; idx < SR * NC; idx += blockDim.x) {
        const int k = idx % SR, q = idx / SR;
        XJ[k][q] = (k < ncols && q < nr) ? X[(j0 + k) + (r0 + q) * ldx] : 0.0;
    }
    issue(tbeg, 0);
    cp_group_commit();
    double accb[QN], accb2[QN];
#pragma unroll
    for (int q = 0; q < QN; ++q) accb[q] = accb2[q] = 0.0;
    for (int I = tbeg; I < tend; ++I) {
        const int buf = (I - tbeg) & 1;
        if (I + 1 < tend) issue(I + 1, buf ^ 1);
        cp_group_commit();
        cp_group_wait<1>();
        __syncthreads();
        const double* T = Tb + buf * SR * SR;
        double acca[QN], acca2[QN];
#pragma unroll
        for (int q = 0; q < QN; ++q) acca[q] = acca2[q] = 0.0;
        if (I != J) {
            // R(I) -= A(I,J) X(J)  (row tr);  R(J) -= A(I,J)^T X(I)  (column tr)
#pragma unroll 4
            for (int k = 0; k < SR; k += 2) {
                const double a0 = T[k * SR + ((tr + k) & 63)], a1 = T[(k + 1) * SR + ((tr + k + 1) & 63)];
                const double b0 = T[tr * SR + ((k + tr) & 63)], b1 = T[tr * SR + ((k + 1 + tr) & 63)];
#pragma unroll
                for (int q = 0; q < QN; ++q) {
                    const int col = tg + 4 * q;
                    acca[q] = fma(a0, XJ[k][col], acca[q]);
                    acca2[q] = fma(a1, XJ[k + 1][col], acca2[q]);
                    accb[q] = fma(b0, XI[buf][k][col], accb[q]);
                    accb2[q] = fma(b1, XI[buf][k + 1][col], accb2[q]);
                }
            }
        } else {
            // diagonal tile: the symmetric product from its lower half, into R(J) only
#pragma unroll 4
            for (int k = 0; k < SR; ++k) {
                const double a = tr >= k ? T[k * SR + ((tr + k) & 63)] : T[tr * SR + ((k + tr) & 63)];
#pragma unroll
                for (int q = 0; q < QN; ++q) acca[q] = fma(a, XJ[k][tg + 4 * q], acca[q]);
            }
        }
        const long long i0 = (long long)I * SR;
        if (i0 + tr < n)
#pragma unroll
            for (int q = 0; q < QN; ++q) {
                const int col = tg + 4 * q;
                if (col < nr) atomicAdd(&R[(i0 + tr) + (r0 + col) * ldr], -(acca[q] + acca2[q]));
            }
        __syncthreads();
    }
    cp_group_wait<0>();
    if (tr < ncols)
#pragma unroll
        for (int q = 0; q < QN; ++q) {
            const int col = tg + 4 * q;
            const double v = accb[q] + accb2[q];
            if (col < nr && v != 0.0) atomicAdd(&R[(j0 + tr) + (r0 + col) * ldr], -v);
        }
}

// The same residual with the tiles of A and the blocks of X brought in by TMA
// (one 32 KB request per tile instead of 4096 element copies); the tile stays
// unrotated in shared memory, element (r, col) at T[col*64 + r], and the column
// walk of the transposed product visits row (k + col) mod 64 at step k so that
// the threads of a warp still hit different banks.  Requires A and X with even
// leading dimensions and 16-byte aligned (the host falls back otherwise).  If a
// tile's arrival wait gives up, NaN is folded into the affected rows of R, which
// the refinement treats as a failed residual.
__device__ int g_sr_status;

template <int NC>
constexpr size_t symm_residual_tma_smem()
{
    return 1024 + sizeof(double) * (2 * SR * SR + 2 * NC * SR + SR * (NC + 1));
}

template <int NC>
__global__ void __launch_bounds__(256, 2) k_symm_residual_tma(const __grid_constant__ CUtensorMap amap,
                                                              const __grid_constant__ CUtensorMap xmap, int n,
                                                              int nrhs, const double* __restrict__ X, long long ldx,
                                                              double* __restrict__ R, long long ldr, int chunks)
{
    constexpr int QN = NC / 4;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[2];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    double* Tb = reinterpret_cast<double*>(base);  // [2][64 cols][64 rows]
    double* XIb = Tb + 2 * SR * SR;                // [2][NC][64]
    double (*XJ)[NC + 1] = reinterpret_cast<double (*)[NC + 1]>(XIb + 2 * NC * SR);
    const int N = (int)ceil_div(n, SR);
    const int J = blockIdx.x / chunks, c = blockIdx.x % chunks;
    if (J >= N) return;
    const int tbeg = J + c * SR_CPT;
    if (tbeg >= N) return;
    const int tend = (tbeg + SR_CPT) < N ? (tbeg + SR_CPT) : N;
    const long long j0 = (long long)J * SR;
    const int ncols = (int)((n - j0) < SR ? (n - j0) : SR);
    const int r0 = blockIdx.y * NC;
    const int nr = nrhs - r0 < NC ? nrhs - r0 : NC;
    const int tr = threadIdx.x & 63, tg = threadIdx.x >> 6;
    if (threadIdx.x == 0) {
        tc::mbar_init(&full[0], 1);
        tc::mbar_init(&full[1], 1);
        tc::mbar_fence_init();
    }
    for (int idx = threadIdx.x; idx < SR * NC; idx += blockDim.x) {
        const int k = idx % SR, q = idx / SR;
        XJ[k][q] = (k < ncols && q < nr) ? X[(j0 + k) + (r0 + q) * ldx] : 0.0;
    }
    __syncthreads();
    constexpr uint32_t bytes = (uint32_t)(sizeof(double) * (SR * SR + NC * SR));
    auto issue = [&](int I, int buf) {
        if (threadIdx.x == 0) {
            tc::mbar_expect_tx(&full[buf], bytes);
            tc::tma_load_2d(Tb + buf * SR * SR, &amap, &full[buf], I * SR, (int)j0);
            tc::tma_load_2d(XIb + buf * NC * SR, &xmap, &full[buf], I * SR, r0);
        }
    };
    issue(tbeg, 0);
    double accb[QN], accb2[QN];
#pragma unroll
    for (int q = 0; q < QN; ++q) accb[q] = accb2[q] = 0.0;
    bool all_ok = true;
    for (int I = tbeg; I < tend; ++I) {
        const int k_ = I - tbeg, buf = k_ & 1;
        if (I + 1 < tend) issue(I + 1, buf ^ 1);
        const bool ok = __syncthreads_and(tc::mbar_wait(&full[buf], (k_ >> 1) & 1, &g_sr_status, 0x31));
        all_ok = all_ok && ok;
        const double* T = Tb + buf * SR * SR;
        const double* XI = XIb + buf * NC * SR;
        double acca[QN], acca2[QN];
#pragma unroll
        for (int q = 0; q < QN; ++q) acca[q] = acca2[q] = 0.0;
        if (!ok) {
#pragma unroll
            for (int q = 0; q < QN; ++q) acca[q] = __longlong_as_double(0x7ff8000000000000LL);
        } else if (I != J) {
            // R(I) -= A(I,J) X(J)  (row tr);  R(J) -= A(I,J)^T X(I)  (column tr, rows visited rotated)
#pragma unroll 4
            for (int k = 0; k < SR; k += 2) {
                const double a0 = T[k * SR + tr], a1 = T[(k + 1) * SR + tr];
                const int kr0 = (k + tr) & 63, kr1 = (k + 1 + tr) & 63;
                const double b0 = T[tr * SR + kr0], b1 = T[tr * SR + kr1];
#pragma unroll
                for (int q = 0; q < QN; ++q) {
                    const int col = tg + 4 * q;
                    acca[q] = fma(a0, XJ[k][col], acca[q]);
                    acca2[q] = fma(a1, XJ[k + 1][col], acca2[q]);
                    accb[q] = fma(b0, XI[col * SR + kr0], accb[q]);
                    accb2[q] = fma(b1, XI[col * SR + kr1], accb2[q]);
                }
            }
        } else {
            // diagonal tile: the symmetric product from its lower half, into R(J) only
#pragma unroll 4
            for (int k = 0; k < SR; ++k) {
                const double a = tr >= k ? T[k * SR + tr] : T[tr * SR + k];
#pragma unroll
                for (int q = 0; q < QN; ++q) acca[q] = fma(a, XJ[k][tg + 4 * q], acca[q]);
            }
        }
        const long long i0 = (long long)I * SR;
        if (i0 + tr < n)
#pragma unroll
            for (int q = 0; q < QN; ++q) {
                const int col = tg + 4 * q;
                if (col < nr) atomicAdd(&R[(i0 + tr) + (r0 + col) * ldr], -(acca[q] + acca2[q]));
            }
        __syncthreads();
    }
    if (tr < ncols)
#pragma unroll
        for (int q = 0; q < QN; ++q) {
            const int col = tg + 4 * q;
            const double v = all_ok ? accb[q] + accb2[q] : __longlong_as_double(0x7ff8000000000000LL);
            if (col < nr && v != 0.0) atomicAdd(&R[(j0 + tr) + (r0 + col) * ldr], -v);
        }
}

// The residual for up to 8 right-hand sides on the FP64 tensor cores
// (mma.sync m8n8k4 f64): with n = 8 = the right-hand sides, A(I,J) X(J) is
// 8 x 16 fragments of the tile times the 16 fragments of X(J), and
// A(I,J)^T X(I) the transposed fragments times those of X(I); the k sum runs
// inside the instruction, so no partial sums cross threads.  Warp w owns rows
// 8w..8w+7 of the first product (accumulated per tile, folded into R(I) with
// atomics) and columns 8w..8w+7 of the second (accumulated over the CTA's tiles,
// folded into R(J) at the end); X(J)'s fragments stay in registers for the
// CTA's life.  The tile arrives by one TMA load of a 68 x 64 box: its column
// stride of 68 doubles (4 rows beyond the tile, never read) puts the 32
// elements of every fragment of either orientation, and of X(I)'s fragments, on
// 16 distinct 8-byte bank pairs, two wavefronts per load, where the dense
// 64-double stride gives 4-way (row walk) and 8-way (column walk) conflicts.
// Two stages per CTA, two CTAs per SM.  Same preconditions and timeout
// behaviour as k_symm_residual_tma.
// ---------------------------------------------------------------------------
constexpr int SRD_LD = SR + 4;                                      // smem column stride (doubles)
constexpr int SRD_TILE = SRD_LD * SR;                               // A tile, doubles
constexpr int SRD_XI = SRD_LD * 8;                                  // X(I) block, doubles
constexpr int SRD_STAGE = ((SRD_TILE + SRD_XI) * 8 + 1023) / 1024 * 1024;  // bytes, 1024-aligned
constexpr int SRD_NSTAGE = 2;
constexpr size_t symm_residual_dmma_smem() { return 1024 + (size_t)SRD_NSTAGE * SRD_STAGE; }

__device__ __forceinline__ void dmma_f64(double& d0, double& d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(256, 2) k_symm_residual_dmma(const __grid_constant__ CUtensorMap amap,
                                                               const __grid_constant__ CUtensorMap xmap, int n,
                                                               int nrhs, const double* __restrict__ X, long long ldx,
                                                               double* __restrict__ R, long long ldr, int chunks)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[SRD_NSTAGE];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int N = (int)ceil_div(n, SR);
    const int J = blockIdx.x / chunks, c = blockIdx.x % chunks;
    if (J >= N) return;
    const int tbeg = J + c * SR_CPT;
    if (tbeg >= N) return;
    const int tend = (tbeg + SR_CPT) < N ? (tbeg + SR_CPT) : N;
    const long long j0 = (long long)J * SR;
    const int r0 = blockIdx.y * 8;
    const int nr = nrhs - r0 < 8 ? nrhs - r0 : 8;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, q = lane & 3;  // fragment row / column within the 8x4 (4x8) block
    if (threadIdx.x == 0) {
        for (int s = 0; s < SRD_NSTAGE; ++s) tc::mbar_init(&full[s], 1);
        tc::mbar_fence_init();
    }
    __syncthreads();
    constexpr uint32_t bytes = (uint32_t)(sizeof(double) * (SRD_TILE + SRD_XI));
    auto issue = [&](int I, int s) {
        if (threadIdx.x == 0) {
            double* T = reinterpret_cast<double*>(base + s * SRD_STAGE);
            tc::mbar_expect_tx(&full[s], bytes);
            tc::tma_load_2d(T, &amap, &full[s], I * SR, (int)j0);
            tc::tma_load_2d(T + SRD_TILE, &xmap, &full[s], I * SR, r0);
        }
    };
    for (int s = 0; s < SRD_NSTAGE && tbeg + s < tend; ++s) issue(tbeg + s, s);
    // B fragments of X(J): element (k = 4kb + q, rhs = g)
    double xj[16];
#pragma unroll
    for (int kb = 0; kb < 16; ++kb) {
        const long long row = j0 + 4 * kb + q;
        xj[kb] = (row < n && g < nr) ? X[row + (r0 + g) * ldx] : 0.0;
    }
    double cb0 = 0.0, cb1 = 0.0, cb2 = 0.0, cb3 = 0.0;  // second product, rows 8w+g of R(J), two k parities
    bool all_ok = true;
    for (int I = tbeg; I < tend; ++I) {
        const int k_ = I - tbeg, s = k_ % SRD_NSTAGE;
        const bool ok = __syncthreads_and(tc::mbar_wait(&full[s], (k_ / SRD_NSTAGE) & 1, &g_sr_status, 0x32));
        all_ok = all_ok && ok;
        const double* T = reinterpret_cast<const double*>(base + s * SRD_STAGE);
        const double* XI = T + SRD_TILE;
        double ca0 = 0.0, ca1 = 0.0, ca2 = 0.0, ca3 = 0.0;
        if (I != J) {
            // A(I,J) X(J): A fragment (row 8w+g, k 4kb+q) at T[k*68 + row]
            // A(I,J)^T X(I): A fragment (col 8w+g, k 4kb+q) at T[col*68 + k], B fragment X(I)(4kb+q, g)
#pragma unroll
            for (int kb = 0; kb < 16; kb += 2) {
                const double a0 = T[(4 * kb + q) * SRD_LD + 8 * w + g];
                const double a1 = T[(4 * kb + 4 + q) * SRD_LD + 8 * w + g];
                const double t0 = T[(8 * w + g) * SRD_LD + 4 * kb + q];
                const double t1 = T[(8 * w + g) * SRD_LD + 4 * kb + 4 + q];
                const double x0 = XI[g * SRD_LD + 4 * kb + q];
                const double x1 = XI[g * SRD_LD + 4 * kb + 4 + q];
                dmma_f64(ca0, ca1, a0, xj[kb]);
                dmma_f64(ca2, ca3, a1, xj[kb + 1]);
                dmma_f64(cb0, cb1, t0, x0);
                dmma_f64(cb2, cb3, t1, x1);
            }
        } else {
            // diagonal tile: the symmetric product from its lower half, into R(J) only
#pragma unroll
            for (int kb = 0; kb < 16; kb += 2) {
                const int r = 8 * w + g, k0 = 4 * kb + q, k1 = k0 + 4;
                const double a0 = r >= k0 ? T[k0 * SRD_LD + r] : T[r * SRD_LD + k0];
                const double a1 = r >= k1 ? T[k1 * SRD_LD + r] : T[r * SRD_LD + k1];
                dmma_f64(ca0, ca1, a0, xj[kb]);
                dmma_f64(ca2, ca3, a1, xj[kb + 1]);
            }
        }
        __syncthreads();  // stage s consumed by every warp
        if (I + SRD_NSTAGE < tend) issue(I + SRD_NSTAGE, s);
        // C fragment: row 8w+g, right-hand sides 2q and 2q+1
        const long long row = (long long)I * SR + 8 * w + g;
        const double nanv = __longlong_as_double(0x7ff8000000000000LL);
        const double v0 = ok ? ca0 + ca2 : nanv, v1 = ok ? ca1 + ca3 : nanv;
        if (row < n) {
            if (2 * q < nr) atomicAdd(&R[row + (r0 + 2 * q) * ldr], -v0);
            if (2 * q + 1 < nr) atomicAdd(&R[row + (r0 + 2 * q + 1) * ldr], -v1);
        }
    }
    const long long row = j0 + 8 * w + g;
    if (row < n) {
        const double nanv = __longlong_as_double(0x7ff8000000000000LL);
        const double v0 = all_ok ? cb0 + cb2 : nanv, v1 = all_ok ? cb1 + cb3 : nanv;
        if (2 * q < nr && v0 != 0.0) atomicAdd(&R[row + (r0 + 2 * q) * ldr], -v0);
        if (2 * q + 1 < nr && v1 != 0.0) atomicAdd(&R[row + (r0 + 2 * q + 1) * ldr], -v1);
    }
}

// out[j] = max_i |M(i,j)| (out zeroed by the caller; atomics on the bit pattern of non-negative doubles)
__global__ void __launch_bounds__(256) k_colmax(const double* __restrict__ M, long long ld, int n, int ncol,
                                                double* __restrict__ out)
{
    const int j = blockIdx.y;
    double m = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = fmax(m, fabs(M[i + j * ld]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && j < ncol)
        atomicMax(reinterpret_cast<unsigned long long*>(out + j), __double_as_longlong(m));
}

// Y += alpha * X (n x ncol, column-major)
__global__ void __launch_bounds__(256) k_axpy(int n, int ncol, double alpha, const double* __restrict__ X,
                                              long long ldx, double* __restrict__ Y, long long ldy)
{
    const long long total = (long long)n * ncol;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long i = t % n, j = t / n;
        Y[i + j * ldy] += alpha * X[i + j * ldx];
    }
}

// ---------------------------------------------------------------------------
// GMRES helpers on column blocks (n x ncol, column-major, ld = n).  Vectors
// V_0..V_{nv-1} are stored vstride doubles apart.
// ---------------------------------------------------------------------------
// out[i*ncol + c] = <V_i(:,c), w(:,c)>, one CTA per (i, c), fixed reduction order
__global__ void __launch_bounds__(256) k_multidot(const double* __restrict__ V, long long vstride, int nv,
                                                  const double* __restrict__ w, int n, int ncol,
                                                  double* __restrict__ out)
{
    const int i = blockIdx.x, c = blockIdx.y;
    const double* v = V + i * vstride + (long long)c * n;
    const double* x = w + (long long)c * n;
    double s = 0.0;
    for (int r = threadIdx.x; r < n; r += blockDim.x) s = fma(v[r], x[r], s);
    __shared__ double part[8];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += part[k];
        out[i * ncol + c] = t;
    }
}

// w(:,c) -= sum_i coef[i*ncol + c] V_i(:,c)
__global__ void __launch_bounds__(256) k_multi_axpy(const double* __restrict__ V, long long vstride, int nv,
                                                    const double* __restrict__ coef, double* __restrict__ w, int n,
                                                    int ncol)
{
    const long long total = (long long)n * ncol;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(t / n);
        double acc = w[t];
        for (int i = 0; i < nv; ++i) acc = fma(-coef[i * ncol + c], V[i * vstride + t], acc);
        w[t] = acc;
    }
}

// y(:,c) = alpha * x(:,c) / sqrt(nrm2[c])  (nrm2 == nullptr: y = alpha * x)
__global__ void __launch_bounds__(256) k_scale_cols(const double* __restrict__ x, double* __restrict__ y, int n,
                                                    int ncol, double alpha, const double* __restrict__ nrm2)
{
    const long long total = (long long)n * ncol;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(t / n);
        double s = alpha;
        if (nrm2) {
            const double q = nrm2[c];
            s = q > 0.0 ? alpha / sqrt(q) : 0.0;
        }
        y[t] = s * x[t];
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encode_fn()
{
    static EncodeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeFn>(p);
    });
    return fn;
}

// P: rows x kp elements, K contiguous, row stride ldp elements; box = 128 rows x
// 128 bytes, 128-byte swizzle
bool encode_panel_map(CUtensorMap* map, const void* P, long long rows, int kp, long long ldp, bool tf32)
{
    EncodeFn fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t esize = tf32 ? 4 : 2;
    const cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ldp * esize};
    const cuuint32_t box[2] = {(cuuint32_t)(128 / esize), 128u};
    const cuuint32_t estr[2] = {1u, 1u};
    const CUresult r = fn(map, tf32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                          const_cast<void*>(P), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// W (FP32, n x n, leading dimension ldw, a multiple of 4) as 128 x 128 tiles, no swizzle
bool encode_w_map(CUtensorMap* map, const float* W, int n, long long ldw)
{
    EncodeFn fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)n, (cuuint64_t)n};
    const cuuint64_t strides[1] = {(cuuint64_t)ldw * 4};
    const cuuint32_t box[2] = {128u, 128u};
    const cuuint32_t estr[2] = {1u, 1u};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(W), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// FP64 column-major matrix (rows x cols, leading dimension ld, even) as box_rows x
// box_cols tiles, no swizzle; out-of-range elements read as zero
bool encode_f64_map(CUtensorMap* map, const double* P, long long rows, long long cols, long long ld, int box_rows,
                    int box_cols)
{
    EncodeFn fn = encode_fn();
    if (!fn || (ld & 1) || (reinterpret_cast<uintptr_t>(P) & 15)) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)rows, (cuuint64_t)cols};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 8};
    const cuuint32_t box[2] = {(cuuint32_t)box_rows, (cuuint32_t)box_cols};
    const cuuint32_t estr[2] = {1u, 1u};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(P), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

struct MixedStreams {
    cudaStream_t hi = nullptr;
    cudaEvent_t start = nullptr, panel = nullptr, rest = nullptr;
};
MixedStreams& mixed_streams()
{
    static thread_local MixedStreams res[64];
    int dev = 0;
    cudaGetDevice(&dev);
    MixedStreams& r = res[dev & 63];
    if (r.hi == nullptr) {
        int least = 0, greatest = 0;
        cudaDeviceGetStreamPriorityRange(&least, &greatest);
        cudaStreamCreateWithPriority(&r.hi, cudaStreamNonBlocking, greatest);
        cudaEventCreateWithFlags(&r.start, cudaEventDisableTiming);
        cudaEventCreateWithFlags(&r.panel, cudaEventDisableTiming);
        cudaEventCreateWithFlags(&r.rest, cudaEventDisableTiming);
    }
    return r;
}

template <bool TF32>
cudaError_t mixed_update(float* W, long long ldw, int n, long long t0, long long pr0, int cols, const void* P,
                         long long ldp, int nbk, const int* dinfo, int* status, cudaStream_t st)
{
    const long long m = (long long)n - t0;
    if (m <= 0 || nbk <= 0) return cudaSuccess;
    if (cudaError_t e = smem_optin(k_mixed_update<TF32>, MU_SMEM); e != cudaSuccess) return e;
    CUtensorMap map;
    if (!encode_panel_map(&map, P, (long long)n - pr0, nbk, ldp, TF32)) return cudaErrorInvalidValue;
    CUtensorMap wmap;
    if (!encode_w_map(&wmap, W, n, ldw)) return cudaErrorInvalidValue;
    const long long t = ceil_div(m, 128);
    long long grid = t * ceil_div(cols, 128);
    const int kind = cols == 0 ? region_update_kind(t, &grid) : 0;
    const int nkb = nbk / (TF32 ? 32 : 64);
    const double md = (double)m, cw = cols ? (double)cols : md;
    const double fl = cols ? 2.0 * nbk * (md * cw - cw * (cw - 1) / 2) : md * (md + 1) * nbk;
    ProfScope ps(PK_MIXED_UPDATE, st, fl, 4.0 * (cols ? 2.0 * md * cw : md * (md + 1)));
    if (kind == 2) {
        // the whole trailing region by 256 x 256 blocks, one per CTA pair
        if (cudaError_t e = smem_optin(k_mixed_update_cta2<TF32>, MC_SMEM); e != cudaSuccess) return e;
        k_mixed_update_cta2<TF32><<<(unsigned)grid, 128, MC_SMEM, st>>>(map, wmap, t0, pr0, (int)t, nkb, status);
        note_launches(1);
        return cudaGetLastError();
    }
    if (kind == 1) {
        // the whole trailing region by pairs of tiles sharing their A rows
        if (cudaError_t e = smem_optin(k_mixed_update_pair<TF32>, MP_SMEM); e != cudaSuccess) return e;
        k_mixed_update_pair<TF32><<<(unsigned)grid, 128, MP_SMEM, st>>>(map, wmap, n, t0, pr0, nkb, dinfo, status);
        note_launches(1);
        return cudaGetLastError();
    }
    k_mixed_update<TF32><<<(unsigned)grid, 128, MU_SMEM, st>>>(map, wmap, W, ldw, n, t0, pr0, cols, nkb, dinfo,
                                                               status);
    note_launches(1);
    return cudaGetLastError();
}

// Right-looking factorization in super-steps of G block columns (K = 128 G):
// within a super-step the chain on the high-priority stream factors its
// blocks one after the other (block g first takes the update from blocks
// 0..g-1 of the super-step, left-looking, K = 128 g), then packs the G
// finished panels into one K = 128 G operand, updates the next super-step's
// G block columns with it (look-ahead), and hands it to the caller's stream,
// which updates everything to the right of those in one pass.  The FP32
// trailing matrix is therefore read and written once per super-step instead
// of once per block column: G = 2 halves that traffic.  Per super-step the
// caller's stream waits for the packed panel, the chain waits for the previous
// super-step's trailing update before its look-ahead update, and the two
// touch disjoint tiles.
// P0 / P1: two slots of ddlak_mixed_panel_bytes(n) bytes; a slot holds the
// packed super-step panel (n x 128 G) and the left-looking operand (n x 128 (G-1)).
template <bool TF32>
cudaError_t potrf_mixed_enqueue(float* W, long long ldw, int n, int G, void* P0, void* P1, int* dinfo, int* status,
                                cudaStream_t st)
{
    constexpr int NB = MX_NB;
    const size_t diag_smem = (size_t)NB * diag_block_ld<double>(NB) * sizeof(double);
    if (cudaError_t e = smem_optin(k_potrf_diag_mixed, diag_smem); e != cudaSuccess) return e;
    MixedStreams& L = mixed_streams();
    cudaStream_t hi = L.hi;
    void* P[2] = {P0, P1};
    const long long SW = (long long)G * NB;  // super-step width

    auto diag_trsm = [&](int k0, cudaStream_t s) -> cudaError_t {
        const int nbk = n - k0 < NB ? n - k0 : NB;
        {
            ProfScope ps(PK_MIXED_OTHER, s, (double)nbk * nbk * nbk / 3.0, 4.0 * nbk * (nbk + 1));
            k_potrf_diag_mixed<<<1, 256, (size_t)nbk * diag_block_ld<double>(nbk) * sizeof(double), s>>>(W, ldw, k0, nbk, dinfo);
        }
        note_launches(1);
        if ((long long)n - k0 - nbk <= 0) return cudaGetLastError();
        return launch_trsm_panel<float, false>(W, ldw, k0, nbk, n, dinfo, s);
    };
    // rows [pr0, n) x columns [k0, k0 + kw) of W -> K-contiguous operand at Pbuf
    auto pack = [&](long long pr0, int k0, int kw, void* Pbuf, cudaStream_t s) -> cudaError_t {
        const long long m = (long long)n - pr0;
        dim3 grid((unsigned)ceil_div(m, 32), kw / 32);
        {
            ProfScope ps(PK_MIXED_OTHER, s, 0.0, (double)m * kw * (4.0 + (TF32 ? 4.0 : 2.0)));
            k_pack_panel<TF32><<<grid, dim3(32, 8), 0, s>>>(W, ldw, n, pr0, k0, kw, Pbuf, kw, dinfo);
        }
        note_launches(1);
        return cudaGetLastError();
    };

    cudaEventRecord(L.start, st);
    cudaStreamWaitEvent(hi, L.start, 0);
    bool have_rest = false, have_panel = false;
    int step = 0;
    cudaError_t e = cudaSuccess;
    for (long long k0 = 0; k0 < n; k0 += SW, ++step) {
        unsigned char* slot = static_cast<unsigned char*>(P[step & 1]);
        void* Ppanel = slot;
        void* Pleft = slot + ((size_t)n * SW * 4 + 255) / 256 * 256;
        // the chain: the super-step's block columns, each after the left-looking
        // update from the ones before it
        for (int g = 0; g < G; ++g) {
            const long long kg = k0 + (long long)g * NB;
            if (kg >= n) break;
            if (g > 0) {
                if ((e = pack(kg, (int)k0, g * NB, Pleft, hi)) != cudaSuccess) return e;
                const int cols = (long long)n - kg < NB ? (int)(n - kg) : NB;
                if ((e = mixed_update<TF32>(W, ldw, n, kg, kg, cols, Pleft, g * NB, g * NB, dinfo, status, hi)) !=
                    cudaSuccess)
                    return e;
            }
            if ((e = diag_trsm((int)kg, hi)) != cudaSuccess) return e;
        }
        const long long t0 = k0 + SW;  // first row / column after the super-step
        if (t0 >= n) break;
        // all G panels are final: one K = 128 G operand for the updates to the right
        if ((e = pack(t0, (int)k0, (int)SW, Ppanel, hi)) != cudaSuccess) return e;
        cudaEventRecord(L.panel, hi);
        have_panel = true;
        // look-ahead: the next super-step's block columns, after the previous
        // super-step's trailing update has reached them
        if (have_rest) cudaStreamWaitEvent(hi, L.rest, 0);
        const int la_cols = (long long)n - t0 < SW ? (int)(n - t0) : (int)SW;
        if ((e = mixed_update<TF32>(W, ldw, n, t0, t0, la_cols, Ppanel, SW, (int)SW, dinfo, status, hi)) != cudaSuccess)
            return e;
        // the rest of the trailing matrix on the caller's stream
        have_rest = false;
        if (t0 + SW < n) {
            cudaStreamWaitEvent(st, L.panel, 0);
            if ((e = mixed_update<TF32>(W, ldw, n, t0 + SW, t0, 0, Ppanel, SW, (int)SW, dinfo, status, st)) !=
                cudaSuccess)
                return e;
            cudaEventRecord(L.rest, st);
            have_rest = true;
        }
    }
    (void)have_panel;
    cudaEventRecord(L.panel, hi);
    cudaStreamWaitEvent(st, L.panel, 0);
    return cudaGetLastError();
}

// Left-looking factorization fed from host memory, one super-step panel at a
// time (the end-to-end form of pposv_mixed).  The copy stream cs brings the
// lower part of A in column panels of SW = 128 G columns (rows [c0, n) of
// columns [c0, c0 + SW), the part uplo 'L' references) into Ad; on the
// compute stream st, panel c waits only for its own arrival, so the copies of
// the later panels overlap the factorization of the earlier ones:
//   1. W(panel) = fl32(A(panel)), column / row sums for ||A||_inf;
//   2. the panel takes the update from every earlier column,
//      W(i, j) -= sum_{k < c0} Lk(i, k) Lk(j, k), from Lk, the K-contiguous
//      low-precision copy of L the factorization appends to (row stride ldk),
//      in launches of 1024 columns of K (each subtracts its partial sum in FP32):
//      the columns of panels 0 .. c-2 on the compute stream while the previous
//      panel's chain still runs on a high-priority stream (look-ahead), those
//      of panel c-1 on that stream once its chain is done;
//   3. its G block columns are factored one after the other, block g after the
//      update from blocks 0..g-1 of the panel (from Lk as well), with the FP64
//      diagonal block and the panel solve of the right-looking form, and each
//      finished block column is rounded into Lk.
// No part of W to the right of the panel is touched before it arrives.  The
// trailing updates of the right-looking form read and write the FP32 trailing
// matrix once per super-step; here each panel is written once and the factor
// is read (in TF32/BF16) once per later panel.
template <bool TF32>
cudaError_t potrf_mixed_stream_enqueue(int n, int G, const double* Ah, long long ldah, double* Ad, long long ldad,
                                       float* W, long long ldw, void* Lk, long long ldk, double* colsum,
                                       double* anrm, int* dinfo, int* status, cudaStream_t cs, cudaStream_t st)
{
    constexpr int NB = MX_NB;
    const size_t diag_smem = (size_t)NB * diag_block_ld<double>(NB) * sizeof(double);
    if (cudaError_t e = smem_optin(k_potrf_diag_mixed, diag_smem); e != cudaSuccess) return e;
    const long long SW = (long long)G * NB;
    const size_t esz = TF32 ? 4 : 2;
    const int S = (int)ceil_div(n, SW);
    auto lk_at = [&](long long row, long long k) -> void* {
        return static_cast<unsigned char*>(Lk) + (size_t)(row * ldk + k) * esz;
    };
    // events: each panel's arrival, the end of its update from the earlier panels (on st)
    // and the end of its chain (on the high-priority stream)
    std::vector<cudaEvent_t> ev((size_t)3 * S, nullptr);
    cudaError_t e = cudaSuccess;
    for (size_t i = 0; i < ev.size() && e == cudaSuccess; ++i)
        e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
    auto release = [&] {
        for (cudaEvent_t x : ev)
            if (x) cudaEventDestroy(x);  // resources go once the recorded work is done
    };
    if (e != cudaSuccess) {
        release();
        return e;
    }
    cudaEvent_t* arrive = ev.data();
    cudaEvent_t* big = ev.data() + S;
    cudaEvent_t* chained = ev.data() + 2 * S;
    MixedStreams& MS = mixed_streams();
    cudaStream_t hs = MS.hi;
    for (int c = 0; c < S && e == cudaSuccess; ++c) {
        const long long c0 = (long long)c * SW, w = std::min<long long>(SW, n - c0);
        e = cudaMemcpy2DAsync(Ad + c0 + c0 * ldad, (size_t)ldad * 8, Ah + c0 + c0 * ldah, (size_t)ldah * 8,
                              (size_t)(n - c0) * 8, (size_t)w, cudaMemcpyHostToDevice, cs);
        if (e == cudaSuccess) e = cudaEventRecord(arrive[c], cs);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(colsum, 0, sizeof(double) * n, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(anrm, 0, sizeof(double), st);
    if (e == cudaSuccess) e = cudaEventRecord(MS.start, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(hs, MS.start, 0);
    // Look-ahead: on st, panel c is converted and takes the update from the panels
    // 0 .. c-2 (whose chains are done) while the high-priority stream still runs the
    // chain of panel c-1; then, on that stream, panel c takes the update from panel
    // c-1 and its own chain runs.  The two streams write disjoint panels of W and
    // disjoint columns of Lk.
    constexpr long long KL = 1024;
    for (int c = 0; c < S && e == cudaSuccess; ++c) {
        const long long c0 = (long long)c * SW, w = std::min<long long>(SW, n - c0);
        if ((e = cudaStreamWaitEvent(st, arrive[c], 0)) != cudaSuccess) break;
        {
            const long long jt = c0 / 64, jts = ceil_div(c0 + w, 64) - jt, its = ceil_div(n - c0, 64);
            ProfScope ps(PK_MIXED_OTHER, st, 0.0, 6.0 * (double)(n - c0) * w);
            k_convert_lower<<<dim3((unsigned)its, (unsigned)jts), 256, 0, st>>>(Ad, ldad, W, ldw, n, 1.0, colsum,
                                                                                (int)jt);
        }
        note_launches(1);
        // the update from the columns of panels 0 .. c-2, in launches of at most KL columns:
        // each launch's partial sum is subtracted from W in FP32 by the epilogue, as the
        // right-looking form does per super-step (one tensor-core accumulation over the
        // whole of K, up to n, measured a less accurate factor: more refinement sweeps)
        const long long kfar = c0 - SW;
        if (kfar > 0 && (e = cudaStreamWaitEvent(st, chained[c - 2], 0)) != cudaSuccess) break;
        for (long long k0 = 0; k0 < kfar && e == cudaSuccess; k0 += KL)
            e = mixed_update<TF32>(W, ldw, n, c0, 0, (int)w, lk_at(0, k0), ldk, (int)std::min(KL, kfar - k0), dinfo,
                                   status, st);
        if (e == cudaSuccess) e = cudaEventRecord(big[c], st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(hs, big[c], 0);
        if (e != cudaSuccess) break;
        // on the chain's stream: the update from panel c-1, then the panel's block columns
        if (c0 > 0 && (e = mixed_update<TF32>(W, ldw, n, c0, 0, (int)w, lk_at(0, c0 - SW), ldk, (int)SW, dinfo,
                                              status, hs)) != cudaSuccess)
            break;
        for (int g = 0; g < G && e == cudaSuccess; ++g) {
            const long long kg = c0 + (long long)g * NB;
            if (kg >= n) break;
            const int nbk = (long long)n - kg < NB ? (int)(n - kg) : NB;
            if (g > 0 && (e = mixed_update<TF32>(W, ldw, n, kg, 0, nbk, lk_at(0, c0), ldk, g * NB, dinfo, status,
                                                 hs)) != cudaSuccess)
                break;
            {
                ProfScope ps(PK_MIXED_OTHER, hs, (double)nbk * nbk * nbk / 3.0, 4.0 * nbk * (nbk + 1));
                k_potrf_diag_mixed<<<1, 256, (size_t)nbk * diag_block_ld<double>(nbk) * sizeof(double), hs>>>(W, ldw, (int)kg, nbk,
                                                                                             dinfo);
            }
            note_launches(1);
            if (kg + nbk >= n) break;  // the last block column: nothing to its right
            if ((e = launch_trsm_panel<float, false>(W, ldw, (int)kg, nbk, n, dinfo, hs)) != cudaSuccess) break;
            {
                const long long m = (long long)n - kg;
                ProfScope ps(PK_MIXED_OTHER, hs, 0.0, (double)m * NB * (4.0 + (TF32 ? 4.0 : 2.0)));
                k_pack_panel<TF32><<<dim3((unsigned)ceil_div(m, 32), NB / 32), dim3(32, 8), 0, hs>>>(
                    W, ldw, n, kg, (int)kg, NB, lk_at(kg, kg), ldk, dinfo);
            }
            note_launches(1);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaEventRecord(chained[c], hs);
    }
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, chained[S - 1], 0);
    if (e == cudaSuccess) {
        k_max_nonneg<<<148, 256, 0, st>>>(colsum, n, anrm);
        note_launches(1);
        e = cudaGetLastError();
    }
    release();
    return e;
}

}  // namespace
}  // namespace ddlak

extern "C" unsigned long long ddlak_mixed_panel_bytes(int n)
{
    // one slot for super-steps of up to DDLAK_MIXED_MAX_GROUP block columns: the packed
    // panel (n x 128 G) and the left-looking operand (n x 128 (G - 1)), FP32 (the larger
    // operand type), each 256-byte aligned
    const unsigned long long rows = (unsigned long long)(n > 0 ? n : 0);
    const unsigned long long G = DDLAK_MIXED_MAX_GROUP;
    return (rows * G * ddlak::MX_NB * 4 + 255) / 256 * 256 + (rows * (G - 1) * ddlak::MX_NB * 4 + 255) / 256 * 256;
}

extern "C" int ddlak_mixed_update_grid(int t, int* kind, long long* ctas)
{
    using namespace ddlak;
    if (t < 1 || !kind || !ctas) return (int)cudaErrorInvalidValue;
    *kind = region_update_kind(t, ctas);
    return 0;
}

extern "C" int ddlak_mixed_update_cta_tiles(int t, long long c, long long* row, long long* col0, int* ntiles)
{
    using namespace ddlak;
    int kind = 0;
    long long ctas = 0;
    if (ddlak_mixed_update_grid(t, &kind, &ctas) != 0 || kind == 0 || c < 0 || c >= ctas || !row || !col0 || !ntiles)
        return (int)cudaErrorInvalidValue;
    const UpdateTiles tl = kind == 2 ? cta2_tiles(c, t) : pair_tiles(c);
    *row = tl.row;
    *col0 = tl.col0;
    *ntiles = tl.ntiles;
    return 0;
}

extern "C" int ddlak_convert_lower(int n, const void* A, long long lda, void* W, long long ldw, double diag_scale,
                                   void* colsum, void* anrm, void* stream)
{
    using namespace ddlak;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n <= 0) return 0;
    cudaError_t e = cudaMemsetAsync(colsum, 0, sizeof(double) * n, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(anrm, 0, sizeof(double), st);
    if (e != cudaSuccess) return (int)e;
    const long long t = ceil_div(n, 64);
    {
        ProfScope ps(PK_MIXED_OTHER, st, 0.0, 6.0 * (double)n * n);
        k_convert_lower<<<(unsigned)(t * (t + 1) / 2), 256, 0, st>>>(static_cast<const double*>(A), lda,
                                                                     static_cast<float*>(W), ldw, n, diag_scale,
                                                                     static_cast<double*>(colsum), -1);
        k_max_nonneg<<<148, 256, 0, st>>>(static_cast<const double*>(colsum), n, static_cast<double*>(anrm));
    }
    note_launches(2);
    return (int)cudaGetLastError();
}

extern "C" int ddlak_potrf_mixed_grouped(char precision, int group, int n, void* W, long long ldw, void* P0,
                                         void* P1, int* dinfo, int* status, void* stream)
{
    using namespace ddlak;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(dinfo, 0, sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(status, 0, sizeof(int), st);
    if (e != cudaSuccess) return (int)e;
    if (n <= 0) return 0;
    if (ldw % 4 != 0) return (int)cudaErrorInvalidValue;  // keeps every W column 16-byte aligned
    float* w = static_cast<float*>(W);
    if (group < 1 || group > DDLAK_MIXED_MAX_GROUP) return (int)cudaErrorInvalidValue;
    if (precision == 'T') return (int)potrf_mixed_enqueue<true>(w, ldw, n, group, P0, P1, dinfo, status, st);
    if (precision == 'B') return (int)potrf_mixed_enqueue<false>(w, ldw, n, group, P0, P1, dinfo, status, st);
    return (int)cudaErrorInvalidValue;
}

extern "C" int ddlak_potrf_mixed(char precision, int n, void* W, long long ldw, void* P0, void* P1, int* dinfo,
                                 int* status, void* stream)
{
    return ddlak_potrf_mixed_grouped(precision, DDLAK_MIXED_GROUP, n, W, ldw, P0, P1, dinfo, status, stream);
}

extern "C" int ddlak_symm_residual(int n, int nrhs, const void* A, long long lda, const void* X, long long ldx,
                                   const void* B, long long ldb, void* R, long long ldr, void* stream)
{
    using namespace ddlak;
    if (n <= 0 || nrhs <= 0) return 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (R != B) {
        const cudaError_t e = cudaMemcpy2DAsync(R, ldr * sizeof(double), B, ldb * sizeof(double), n * sizeof(double),
                                                nrhs, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return (int)e;
    }
    const int N = (int)ceil_div(n, SR);
    const int chunks = (int)ceil_div(N, SR_CPT);
    if (nrhs <= 8) {
        CUtensorMap amap, xmap;
        if (encode_f64_map(&amap, static_cast<const double*>(A), n, n, lda, SRD_LD, SR) &&
            encode_f64_map(&xmap, static_cast<const double*>(X), n, nrhs, ldx, SRD_LD, 8)) {
            const size_t smem = symm_residual_dmma_smem();
            if (cudaError_t e = smem_optin(k_symm_residual_dmma, smem); e != cudaSuccess) return (int)e;
            ProfScope ps(PK_SYMM_RESIDUAL, st, 2.0 * (double)n * n * nrhs, 4.0 * (double)n * (n + 1));
            k_symm_residual_dmma<<<dim3((unsigned)(N * chunks), 1), 256, smem, st>>>(
                amap, xmap, n, nrhs, static_cast<const double*>(X), ldx, static_cast<double*>(R), ldr, chunks);
            note_launches(1);
            return (int)cudaGetLastError();
        }
    }
    auto launch = [&](auto nc_tag) -> void {
        constexpr int NC = decltype(nc_tag)::value;
        CUtensorMap amap, xmap;
        if (encode_f64_map(&amap, static_cast<const double*>(A), n, n, lda, SR, SR) &&
            encode_f64_map(&xmap, static_cast<const double*>(X), n, nrhs, ldx, SR, NC)) {
            const size_t smem = symm_residual_tma_smem<NC>();
            smem_optin(k_symm_residual_tma<NC>, smem);  // a failed raise shows as the launch's error
            dim3 grid((unsigned)(N * chunks), (unsigned)ceil_div(nrhs, NC));
            ProfScope ps(PK_SYMM_RESIDUAL, st, 2.0 * (double)n * n * nrhs, 4.0 * (double)n * (n + 1));
            k_symm_residual_tma<NC><<<grid, 256, smem, st>>>(amap, xmap, n, nrhs, static_cast<const double*>(X),
                                                              ldx, static_cast<double*>(R), ldr, chunks);
            return;
        }
        const size_t smem = symm_residual_smem<NC>();
        smem_optin(k_symm_residual<NC>, smem);  // a failed raise shows as the launch's error
        dim3 grid((unsigned)(N * chunks), (unsigned)ceil_div(nrhs, NC));
        ProfScope ps(PK_SYMM_RESIDUAL, st, 2.0 * (double)n * n * nrhs, 4.0 * (double)n * (n + 1));
        k_symm_residual<NC><<<grid, 256, smem, st>>>(static_cast<const double*>(A), lda, n, nrhs,
                                                    static_cast<const double*>(X), ldx, static_cast<double*>(R), ldr,
                                                    chunks);
    };
    if (nrhs <= 8)
        launch(std::integral_constant<int, 8>{});
    else
        launch(std::integral_constant<int, 16>{});
    note_launches(1);
    return (int)cudaGetLastError();
}

extern "C" int ddlak_colmax(int n, int ncol, const void* M, long long ld, void* out, void* stream)
{
    using namespace ddlak;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double) * (ncol > 0 ? ncol : 0), st);
    if (e != cudaSuccess || n <= 0 || ncol <= 0) return (int)e;
    dim3 grid((unsigned)(ceil_div(n, 256) < 64 ? ceil_div(n, 256) : 64), (unsigned)ncol);
    k_colmax<<<grid, 256, 0, st>>>(static_cast<const double*>(M), ld, n, ncol, static_cast<double*>(out));
    note_launches(1);
    return (int)cudaGetLastError();
}

extern "C" int ddlak_multidot(const void* V, long long vstride, int nv, const void* w, int n, int ncol, void* out,
                              void* stream)
{
    using namespace ddlak;
    if (nv <= 0 || n <= 0 || ncol <= 0) return 0;
    k_multidot<<<dim3(nv, ncol), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const double*>(V), vstride, nv, static_cast<const double*>(w), n, ncol, static_cast<double*>(out));
    note_launches(1);
    return (int)cudaGetLastError();
}

extern "C" int ddlak_multi_axpy(const void* V, long long vstride, int nv, const void* coef, void* w, int n, int ncol,
                                void* stream)
{
    using namespace ddlak;
    if (nv <= 0 || n <= 0 || ncol <= 0) return 0;
    const long long total = (long long)n * ncol;
    const long long grid = ceil_div(total, 256) < 1184 ? ceil_div(total, 256) : 1184;
    k_multi_axpy<<<(unsigned)grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const double*>(V), vstride, nv, static_cast<const double*>(coef), static_cast<double*>(w), n,
        ncol);
    note_launches(1);
    return (int)cudaGetLastError();
}

extern "C" int ddlak_scale_cols(const void* x, void* y, int n, int ncol, double alpha, const void* nrm2, void* stream)
{
    using namespace ddlak;
    if (n <= 0 || ncol <= 0) return 0;
    const long long total = (long long)n * ncol;
    const long long grid = ceil_div(total, 256) < 1184 ? ceil_div(total, 256) : 1184;
    k_scale_cols<<<(unsigned)grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const double*>(x), static_cast<double*>(y), n, ncol, alpha, static_cast<const double*>(nrm2));
    note_launches(1);
    return (int)cudaGetLastError();
}

extern "C" int ddlak_axpy(int n, int ncol, double alpha, const void* X, long long ldx, void* Y, long long ldy,
                          void* stream)
{
    using namespace ddlak;
    if (n <= 0 || ncol <= 0) return 0;
    const long long total = (long long)n * ncol;
    const long long grid = ceil_div(total, 256) < 1184 ? ceil_div(total, 256) : 1184;
    k_axpy<<<(unsigned)grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(n, ncol, alpha,
                                                                         static_cast<const double*>(X), ldx,
                                                                         static_cast<double*>(Y), ldy);
    note_launches(1);
    return (int)cudaGetLastError();
}

extern "C" unsigned long long ddlak_mixed_lk_bytes(char precision, int n, long long* ldk)
{
    // the K-contiguous copy of L: n rows of ldk elements, ldk a multiple of 64 (TMA row strides
    // and the 128-byte boxes stay aligned)
    const long long ld = ((long long)(n > 0 ? n : 1) + 63) / 64 * 64;
    if (ldk) *ldk = ld;
    return (unsigned long long)ld * (unsigned long long)(n > 0 ? n : 0) * (precision == 'B' ? 2u : 4u);
}

extern "C" int ddlak_potrf_mixed_stream(char precision, int group, int n, const void* A_host, long long lda_host,
                                        void* A, long long lda, void* W, long long ldw, void* Lk, long long ldk,
                                        void* colsum, void* anrm, int* dinfo, int* status, void* copy_stream,
                                        void* stream)
{
    using namespace ddlak;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(dinfo, 0, sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(status, 0, sizeof(int), st);
    if (e != cudaSuccess) return (int)e;
    if (n <= 0) return 0;
    if (ldw % 4 != 0 || ldk % 64 != 0 || ldk < n || lda < n || lda_host < n || group < 1 ||
        group > DDLAK_MIXED_MAX_GROUP || (reinterpret_cast<uintptr_t>(Lk) & 255))
        return (int)cudaErrorInvalidValue;
    const double* ah = static_cast<const double*>(A_host);
    double* ad = static_cast<double*>(A);
    float* w = static_cast<float*>(W);
    cudaStream_t cs = static_cast<cudaStream_t>(copy_stream);
    double* cols = static_cast<double*>(colsum);
    double* an = static_cast<double*>(anrm);
    if (precision == 'T')
        return (int)potrf_mixed_stream_enqueue<true>(n, group, ah, lda_host, ad, lda, w, ldw, Lk, ldk, cols, an, dinfo,
                                                     status, cs, st);
    if (precision == 'B')
        return (int)potrf_mixed_stream_enqueue<false>(n, group, ah, lda_host, ad, lda, w, ldw, Lk, ldk, cols, an,
                                                      dinfo, status, cs, st);
    return (int)cudaErrorInvalidValue;
}
