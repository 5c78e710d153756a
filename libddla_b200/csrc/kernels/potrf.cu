// Blocked right-looking Cholesky with look-ahead (ddla::ppotrf / ddla::potrf on
// a 1x1 grid).
//
// Replaces the vendor call the reference makes at src/Cholesky/potrf.cpp:106-113
// (cusolverDn?potrf).  Per block column k of width NB:
//   1. k_potrf_diag   -- the NB x NB diagonal block in shared memory, factored in
//                        32-wide steps (diag_factor.cuh); info detected in-kernel;
//   2. k_trsm_panel   -- L21 = A21 * L11^{-H}: warps own rows, lanes own columns,
//                        each solved entry broadcast with a warp shuffle;
//   3. trailing update -- C -= L21 * L21^H on lower tiles (FP64 DMMA for double,
//                        syrk.cu; register-tiled SIMT for the other types).
// Look-ahead: the update of block column k+1 plus the diagonal block and panel
// of k+1 run on a high-priority internal stream while the update of the rest
// of the trailing matrix runs on the caller's stream; events order the two so
// that no tile is touched by both at once.
// info follows LAPACK ?potrf: the order of the first leading minor that is not
// positive definite (diagonal value <= 0 or NaN), 0 on success.  Every kernel
// returns immediately once info is set, so the first failure is the one kept.
#include <mutex>
#include <type_traits>

#include <ddla_kernels.h>

#include "common.cuh"
#include "ddla_kernels_internal.h"
#include "diag_factor.cuh"
#include "profile.h"
#include "tc_common.cuh"

namespace ddlak {

// ---------------------------------------------------------------------------
// 1. diagonal block
// ---------------------------------------------------------------------------
template <class T, bool UP>
__global__ void __launch_bounds__(256) k_potrf_diag(T* __restrict__ A, long long lda, long long astride, int k0,
                                                    int nbk, int* __restrict__ info)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* s = reinterpret_cast<T*>(smem_raw);
    const int ld = diag_block_ld<T>(nbk);
    A += (long long)blockIdx.x * astride;  // blockIdx.x: the matrix of a batch (grid 1 for one matrix)
    info += blockIdx.x;
    if (*(volatile int*)info != 0) return;
    load_lview_block<T, UP>(s, ld, A, lda, k0, k0, nbk, nbk, nbk, nbk, true);
    const int fail = factor_block_smem<T>(s, ld, nbk);
    if (nbk == 128) {  // the full block: index arithmetic by shifts
        for (int idx = threadIdx.x; idx < 128 * 128; idx += blockDim.x) {
            const int i = UP ? idx >> 7 : idx & 127, j = UP ? idx & 127 : idx >> 7;
            if (i >= j) lview_st<T, UP>(A, lda, k0 + i, k0 + j, s[i + j * ld]);
        }
    } else {
        for (int idx = threadIdx.x; idx < nbk * nbk; idx += blockDim.x) {
            const int i = idx % nbk, j = idx / nbk;
            if (i >= j) lview_st<T, UP>(A, lda, k0 + i, k0 + j, s[i + j * ld]);
        }
    }
    if (fail && threadIdx.x == 0) *info = k0 + fail;
}

// ---------------------------------------------------------------------------
// 2. panel: X * L11^H = A21 for the rows below the diagonal block.
//    Each warp owns PR rows; lane l owns columns l, l+32, ... of those rows.
// ---------------------------------------------------------------------------
template <class T, bool UP, int NQ, int PR>
__global__ void __launch_bounds__(256) k_trsm_panel(T* __restrict__ A, long long lda, int k0, int nbk, int n,
                                                    const int* __restrict__ info)
{
    using R = real_t<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* l11 = reinterpret_cast<T*>(smem_raw);  // [c + j*ldl], c,j < NQ*32, zero outside nbk
    const int ldl = NQ * 32 + 1;
    __shared__ R s_rinv[NQ * 32];
    if (*(volatile int*)info != 0) return;

    load_lview_block<T, UP>(l11, ldl, A, lda, k0, k0, nbk, nbk, NQ * 32, NQ * 32, true);
    // multiply by reciprocal pivots, as reference BLAS ?trsm does for side 'R'
    for (int j = threadIdx.x; j < NQ * 32; j += blockDim.x) s_rinv[j] = j < nbk ? R(1) / re(l11[j + j * ldl]) : R(0);
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // persistent over row groups of 8 warps x PR rows: L11 is loaded once per CTA
    const long long ngroups = ceil_div((long long)n - k0 - nbk, 8LL * PR);
    for (long long grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
        const long long row0 = (long long)k0 + nbk + (grp * (blockDim.x >> 5) + warp) * PR;
        if (row0 >= n) continue;
        T p[PR][NQ];
#pragma unroll
        for (int r = 0; r < PR; ++r)
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                const long long i = row0 + r;
                const int c = q * 32 + lane;
                p[r][q] = (i < n && c < nbk) ? lview_ld<T, UP>(A, lda, i, k0 + c) : zero<T>();
            }

#pragma unroll
        for (int qj = 0; qj < NQ; ++qj) {
            for (int jj = 0; jj < 32; ++jj) {
                const int j = qj * 32 + jj;
                if (j >= nbk) break;
                const R rjj = s_rinv[j];
                T x[PR];
#pragma unroll
                for (int r = 0; r < PR; ++r) {
                    const T v = scal(p[r][qj], rjj);
                    if (lane == jj) p[r][qj] = v;
                    x[r] = shfl(v, jj);
                }
#pragma unroll
                for (int q = qj; q < NQ; ++q) {
                    const int c = q * 32 + lane;
                    if (c > j) {
                        const T lcj = cj(l11[c + j * ldl]);
#pragma unroll
                        for (int r = 0; r < PR; ++r) p[r][q] = fms(p[r][q], x[r], lcj);
                    }
                }
            }
        }
#pragma unroll
        for (int r = 0; r < PR; ++r)
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                const long long i = row0 + r;
                const int c = q * 32 + lane;
                if (i < n && c < nbk) lview_st<T, UP>(A, lda, i, k0 + c, p[r][q]);
            }
    }
}

// Grid of the panel solve: every row group once, at most as many CTAs as fit on
// the device at once (the kernel loops over row groups).
template <class K>
long long trsm_grid(K* kernel, size_t smem, long long groups)
{
    static std::mutex mu;
    static int cap[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return groups;
    std::lock_guard<std::mutex> lk(mu);
    if (cap[dev] == 0) {
        int sms = 148, per = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, 256, smem);
        cap[dev] = sms * (per > 0 ? per : 1);
    }
    return groups < cap[dev] ? groups : cap[dev];
}

// ---------------------------------------------------------------------------
// 3. generic trailing update (SIMT; every type).  64x64 tiles, 16-wide k
//    chunks through shared memory, 4x4 per thread.  Region: rows [t0, n) and
//    columns [t0, n) (cols == 0, lower triangle of tiles) or [t0, t0+cols).
// ---------------------------------------------------------------------------
template <class T, bool UP>
__global__ void __launch_bounds__(256) k_syrk_simt(T* __restrict__ A, long long lda, int k0, int nbk, int n,
                                                   long long t0, int cols, const int* __restrict__ info)
{
    constexpr int BT = 64, BK = 16;
    __shared__ T As[BK][BT + 1];
    __shared__ T Bs[BK][BT + 1];
    if (*(volatile int*)info != 0) return;
    int I, J;
    if (cols == 0) {
        tile_of_tri(blockIdx.x, I, J);
    } else {
        const int nct = (cols + BT - 1) / BT;
        J = blockIdx.x % nct;
        I = blockIdx.x / nct;
        if (I < J) return;
    }
    const long long cend = cols == 0 ? (long long)n : t0 + cols;
    const long long ri = t0 + (long long)I * BT, rj = t0 + (long long)J * BT;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    T acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = zero<T>();

    for (int kc = 0; kc < nbk; kc += BK) {
        for (int idx = threadIdx.x; idx < BT * BK; idx += 256) {
            int i, k;
            if (UP) { k = idx % BK; i = idx / BK; } else { i = idx % BT; k = idx / BT; }
            const bool kin = kc + k < nbk;
            As[k][i] = (kin && ri + i < n) ? lview_ld<T, UP>(A, lda, ri + i, k0 + kc + k) : zero<T>();
            Bs[k][i] = (kin && rj + i < cend) ? lview_ld<T, UP>(A, lda, rj + i, k0 + kc + k) : zero<T>();
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < BK; ++k) {
            T av[4], bv[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) av[a] = As[k][tx + 16 * a];
#pragma unroll
            for (int b = 0; b < 4; ++b) bv[b] = cj(Bs[k][ty + 16 * b]);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b] = fma_(acc[a][b], av[a], bv[b]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const long long i = ri + tx + 16 * a, j = rj + ty + 16 * b;
            if (i < n && j < cend && i >= j) {
                T c = lview_ld<T, UP>(A, lda, i, j);
                lview_st<T, UP>(A, lda, i, j, sub(c, acc[a][b]));
            }
        }
}

template <class T, bool UP>
cudaError_t trailing_update_simt(T* A, long long lda, int k0, int nbk, int n, long long t0, int cols, const int* dinfo,
                                 cudaStream_t st)
{
    const long long m = (long long)n - t0;
    if (m <= 0) return cudaSuccess;
    const long long t = ceil_div(m, 64);
    const long long grid = cols == 0 ? t * (t + 1) / 2 : t * ceil_div(cols, 64);
    k_syrk_simt<T, UP><<<(unsigned)grid, 256, 0, st>>>(A, lda, k0, nbk, n, t0, cols, dinfo);
    return cudaGetLastError();
}

#define DDLAK_INST_SIMT(T, UP)                                                                                      \
    template cudaError_t trailing_update_simt<T, UP>(T*, long long, int, int, int, long long, int, const int*,     \
                                                     cudaStream_t);
DDLAK_INST_SIMT(float, false)
DDLAK_INST_SIMT(float, true)
DDLAK_INST_SIMT(double, false)
DDLAK_INST_SIMT(double, true)
DDLAK_INST_SIMT(cf32, false)
DDLAK_INST_SIMT(cf32, true)
DDLAK_INST_SIMT(cf64, false)
DDLAK_INST_SIMT(cf64, true)
#undef DDLAK_INST_SIMT

// ---------------------------------------------------------------------------
// host-side enqueue of the whole factorization
// ---------------------------------------------------------------------------
template <class T> constexpr int potrf_nb() { return sizeof(T) == 16 ? 64 : 128; }

// ---------------------------------------------------------------------------
// The FP32 panel of the mixed factorization (lower storage, nbk <= 128): one
// thread per row.  X L11^T = A21 along the row, in two halves of 64 columns so
// that at most 64 of the row's values are live in registers:
//   1. x1 = row[0:64] solved against L11[0:64, 0:64] (x_j *= 1 / l_jj,
//      x_k -= x_j l_kj for k > j), written back and staged in shared memory;
//   2. x2 = row[64:128] - x1 L11[64:128, 0:64]^T, then solved against
//      L11[64:128, 64:128], written back.
// Columns of L11 are read from shared memory as float4 broadcasts (every thread
// of the warp reads the same address); the row loads and stores are coalesced
// (consecutive threads, consecutive rows of the column-major panel), and no
// shuffle sits on the per-column chain.
// ---------------------------------------------------------------------------
constexpr int TRR_NT = 128;
constexpr size_t TRR_SMEM = (128 * 128 + 64 * TRR_NT) * sizeof(float);

// a shared-memory float4 load kept in program order (the unrolled substitution would
// otherwise hoist hundreds of them ahead of their use and run out of registers)
__device__ __forceinline__ float4 ld_shared_f4(const float4* p)
{
    float4 v;
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
    return v;
}

// x (64 values at column offset c0) against the 64 x 64 diagonal part of L11 at (c0, c0)
__device__ __forceinline__ void trr_solve64(float (&x)[64], const float* l11, const float* rinv, int c0)
{
#pragma unroll
    for (int j = 0; j < 64; ++j) {
        x[j] *= rinv[c0 + j];
        const float4* col = reinterpret_cast<const float4*>(&l11[(c0 + j) * 128 + c0]);
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            if (4 * q + 3 > j) {
                const float4 l = ld_shared_f4(col + q);
                if (4 * q + 0 > j) x[4 * q + 0] = fmaf(-x[j], l.x, x[4 * q + 0]);
                if (4 * q + 1 > j) x[4 * q + 1] = fmaf(-x[j], l.y, x[4 * q + 1]);
                if (4 * q + 2 > j) x[4 * q + 2] = fmaf(-x[j], l.z, x[4 * q + 2]);
                if (4 * q + 3 > j) x[4 * q + 3] = fmaf(-x[j], l.w, x[4 * q + 3]);
            }
        }
    }
}

__device__ int g_trsm_status;  // a TMA wait that gave up (never expected): the panel is NaN-poisoned

// TMA: L11 staged by one 128 x 128 TMA box (nbk = 128; the solve reads only entries
// below the diagonal, so the block's upper half comes in unmasked); otherwise by loads.
template <bool TMA>
__global__ void __launch_bounds__(TRR_NT) k_trsm_panel_rows(const __grid_constant__ CUtensorMap amap,
                                                            float* __restrict__ A, long long lda, int k0, int nbk,
                                                            int n, const int* __restrict__ info)
{
    extern __shared__ __align__(128) float trr_smem[];
    float* l11 = trr_smem;               // l11[j * 128 + k] = L(k0 + k, k0 + j) (zero for k < j or k >= nbk by loads)
    float* xs = trr_smem + 128 * 128;    // xs[j * TRR_NT + t]: thread t's solved first half
    __shared__ float rinv[128];
    __shared__ __align__(8) uint64_t l11_bar;
    if (*(volatile const int*)info != 0) return;
    bool staged = true;
    if constexpr (TMA) {
        if (threadIdx.x == 0) {
            tc::mbar_init(&l11_bar, 1);
            tc::mbar_fence_init();
            tc::prefetch_tmap(&amap);
            tc::mbar_expect_tx(&l11_bar, 128 * 128 * 4);
            tc::tma_load_2d(l11, &amap, &l11_bar, k0, k0);
        }
        __syncthreads();
        staged = __syncthreads_and(tc::mbar_wait(&l11_bar, 0, &g_trsm_status, 0x53));
        if (!staged && threadIdx.x == 0) (void)tc::mbar_wait(&l11_bar, 0, &g_trsm_status, 0x54);
    } else {
        const float* Ad = A + k0 + (long long)k0 * lda;
        for (int idx = threadIdx.x; idx < 128 * 32; idx += TRR_NT) {
            const int j = idx >> 5, k4 = (idx & 31) * 4;
            float v[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int k = k4 + e;
                v[e] = (j < nbk && k < nbk && k >= j) ? Ad[k + (long long)j * lda] : 0.f;
            }
            *reinterpret_cast<float4*>(&l11[j * 128 + k4]) = make_float4(v[0], v[1], v[2], v[3]);
        }
        __syncthreads();
    }
    rinv[threadIdx.x] = threadIdx.x < nbk ? 1.f / l11[threadIdx.x * 129] : 0.f;
    __syncthreads();
    const int t = threadIdx.x;
    const long long row = (long long)k0 + nbk + (long long)blockIdx.x * TRR_NT + t;
    const bool live = row < n;
    float* Ar = A + (live ? row : (long long)k0) + (long long)k0 * lda;
    if (!staged) {  // L11 never arrived: poison the rows (the next diagonal block reports a NaN pivot)
        if (live)
            for (int c = 0; c < nbk; ++c) Ar[(long long)c * lda] = __int_as_float(0x7fc00000);
        return;
    }
    // the two 64-column halves through one rolled loop, so that the unrolled solve exists once
    // in the instruction stream (the kernel is bound by instruction fetch, not arithmetic)
#pragma unroll 1
    for (int half = 0; half < 2; ++half) {
        const int c0 = 64 * half;
        if (c0 >= nbk) break;  // uniform
        float x[64];
        {
            const float* p = Ar + (long long)c0 * lda;
#pragma unroll
            for (int c = 0; c < 64; ++c) x[c] = (live && c0 + c < nbk) ? p[(long long)c * lda] : 0.f;
        }
        if (half == 1) {
            // x -= x1 L11[64:128, 0:64]^T, x1 = this thread's solved first half
#pragma unroll 4
            for (int j = 0; j < 64; ++j) {
                const float xj = xs[j * TRR_NT + t];
                const float4* col = reinterpret_cast<const float4*>(&l11[j * 128 + 64]);
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const float4 l = ld_shared_f4(col + q);
                    x[4 * q + 0] = fmaf(-xj, l.x, x[4 * q + 0]);
                    x[4 * q + 1] = fmaf(-xj, l.y, x[4 * q + 1]);
                    x[4 * q + 2] = fmaf(-xj, l.z, x[4 * q + 2]);
                    x[4 * q + 3] = fmaf(-xj, l.w, x[4 * q + 3]);
                }
            }
        }
        trr_solve64(x, l11, rinv, c0);
        {
            // the row's addresses are recomputed here rather than kept live through the solve
            float* p = Ar + (long long)c0 * lda;
            long long ld = lda;
            asm volatile("" : "+l"(p), "+l"(ld));
#pragma unroll
            for (int c = 0; c < 64; ++c) {
                if (live && c0 + c < nbk) p[(long long)c * ld] = x[c];
                if (half == 0) xs[c * TRR_NT + t] = x[c];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// The FP64 panel (lower storage, nbk <= 128): L11 staged in shared memory by TMA
// (ten 32 x 32 boxes, one mbarrier) when lda is even, then one thread per row, in
// four chunks of 32 columns so that 32 of the row's values are live in registers.
// Chunk C: x = row[32C : 32C + 32]; x -= x_J L11[32C.., 32J..]^T for the
// chunks J < C (their solved values re-read from the row this thread already
// wrote); then x is solved against the diagonal block (x_j *= 1 / l_jj,
// x_k -= x_j l_kj for k > j) and written back.  Every entry receives the
// updates of its columns in increasing order, as in the column-by-column
// substitution.  L11's lower part is held as ten 32 x 32 blocks (80 KB, two
// CTAs per SM) read as 16-byte broadcasts; the row loads and stores are
// coalesced (consecutive threads, consecutive rows).
// ---------------------------------------------------------------------------
constexpr int TRD_NT = 128;
constexpr size_t TRD_SMEM = 10 * 32 * 32 * sizeof(double);

__device__ __forceinline__ double2 ld_shared_d2(const double2* p)
{
    double2 v;
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a));
    return v;
}

// TMA_DIMS: 0 = L11 staged by plain loads (any lda, any nbk); 2 = by ten 32 x 32 TMA
// boxes from a 2-D map over A; 3 = the same from a 3-D map over a batch (z = matrix).
// The TMA forms need nbk = 128: they load whole boxes, so the diagonal blocks'
// upper halves come in unmasked (the solve reads only entries below the diagonal).

template <int TMA_DIMS>
__global__ void __launch_bounds__(TRD_NT) k_trsm_panel_rows_f64(const __grid_constant__ CUtensorMap amap,
                                                                double* __restrict__ A, long long lda,
                                                                long long astride, int k0, int nbk, int n,
                                                                const int* __restrict__ info)
{
    // block (C, J), J <= C, at trd_smem + (C (C + 1) / 2 + J) * 1024, element [j * 32 + i]
    // = L(k0 + 32 C + i, k0 + 32 J + j) (zero above the diagonal and past nbk when staged by loads)
    extern __shared__ __align__(128) double trd_smem[];
    __shared__ double rinv[128];
    __shared__ __align__(8) uint64_t l11_bar;
    A += (long long)blockIdx.y * astride;  // blockIdx.y: the matrix of a batch
    info += blockIdx.y;
    if (*(volatile const int*)info != 0) return;
    bool staged = true;
    if constexpr (TMA_DIMS == 0) {
        const double* Ad = A + k0 + (long long)k0 * lda;
        for (int idx = threadIdx.x; idx < 10 * 1024; idx += TRD_NT) {
            const int b = idx >> 10, e = idx & 1023, j = e >> 5, i = e & 31;
            const int C = b >= 6 ? 3 : b >= 3 ? 2 : b >= 1 ? 1 : 0;
            const int J = b - C * (C + 1) / 2;
            const int r = 32 * C + i, c = 32 * J + j;
            trd_smem[idx] = (r < nbk && c < nbk && r >= c) ? Ad[r + (long long)c * lda] : 0.0;
        }
        __syncthreads();
    } else {
        if (threadIdx.x == 0) {
            tc::mbar_init(&l11_bar, 1);
            tc::mbar_fence_init();
            tc::prefetch_tmap(&amap);
            tc::mbar_expect_tx(&l11_bar, 10 * 32 * 32 * 8);
            for (int C = 0, b = 0; C < 4; ++C)
                for (int J = 0; J <= C; ++J, ++b) {
                    if constexpr (TMA_DIMS == 2)
                        tc::tma_load_2d(trd_smem + b * 1024, &amap, &l11_bar, k0 + 32 * C, k0 + 32 * J);
                    else
                        tc::tma_load_3d(trd_smem + b * 1024, &amap, &l11_bar, k0 + 32 * C, k0 + 32 * J,
                                        (int)blockIdx.y);
                }
        }
        __syncthreads();
        staged = __syncthreads_and(tc::mbar_wait(&l11_bar, 0, &g_trsm_status, 0x51));
        if (!staged && threadIdx.x == 0)  // give the copies a second bounded chance to land before the exit
            (void)tc::mbar_wait(&l11_bar, 0, &g_trsm_status, 0x52);
    }
    {
        const int t = threadIdx.x, C = t >> 5, i = t & 31;
        rinv[t] = t < nbk ? 1.0 / trd_smem[(C * (C + 1) / 2 + C) * 1024 + i * 32 + i] : 0.0;
    }
    __syncthreads();
    const long long row = (long long)k0 + nbk + (long long)blockIdx.x * TRD_NT + threadIdx.x;
    const bool live = row < n;
    double* Ar = A + (live ? row : (long long)k0) + (long long)k0 * lda;
    if (!staged) {  // L11 never arrived: poison the rows (the next diagonal block reports a NaN pivot)
        if (live)
            for (int c = 0; c < nbk; ++c) Ar[(long long)c * lda] = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    const int nch = (nbk + 31) >> 5;
    for (int C = 0; C < nch; ++C) {
        double x[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) x[i] = (live && 32 * C + i < nbk) ? Ar[(long long)(32 * C + i) * lda] : 0.0;
        for (int J = 0; J < C; ++J) {
            const double* blk = trd_smem + (C * (C + 1) / 2 + J) * 1024;
            const double* xs = Ar + (long long)(32 * J) * lda;
#pragma unroll 4
            for (int j = 0; j < 32; ++j) {
                const double xj = live ? xs[(long long)j * lda] : 0.0;
                const double2* col = reinterpret_cast<const double2*>(blk + j * 32);
#pragma unroll
                for (int h = 0; h < 16; ++h) {
                    const double2 l = ld_shared_d2(col + h);
                    x[2 * h] = fma(-xj, l.x, x[2 * h]);
                    x[2 * h + 1] = fma(-xj, l.y, x[2 * h + 1]);
                }
            }
        }
        const double* dblk = trd_smem + (C * (C + 1) / 2 + C) * 1024;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            x[j] *= rinv[32 * C + j];
            const double2* col = reinterpret_cast<const double2*>(dblk + j * 32);
#pragma unroll
            for (int h = 0; h < 16; ++h) {
                if (2 * h + 1 > j) {
                    const double2 l = ld_shared_d2(col + h);
                    if (2 * h > j) x[2 * h] = fma(-x[j], l.x, x[2 * h]);
                    x[2 * h + 1] = fma(-x[j], l.y, x[2 * h + 1]);
                }
            }
        }
#pragma unroll
        for (int i = 0; i < 32; ++i)
            if (live && 32 * C + i < nbk) Ar[(long long)(32 * C + i) * lda] = x[i];
    }
}

template <class T, bool UP>
cudaError_t launch_trsm_panel(T* A, long long lda, int k0, int nbk, int n, const int* dinfo, cudaStream_t s)
{
    if constexpr (std::is_same<T, float>::value && !UP) {
        const long long m = (long long)n - k0 - nbk;
        if (m <= 0) return cudaSuccess;
        const double md = (double)m, b = nbk;
        ProfScope ps(PK_TRSM_PANEL, s, md * b * b, sizeof(T) * (2.0 * md * b + b * (b + 1) / 2));
        const unsigned grid = (unsigned)ceil_div(m, TRR_NT);
        CUtensorMap amap{};
        if (nbk == 128 && (lda % 4) == 0 &&
            tc::encode_colmajor_2d(&amap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, A, n, n, lda, 128, 128,
                                   CU_TENSOR_MAP_SWIZZLE_NONE)) {
            if (cudaError_t e = smem_optin(k_trsm_panel_rows<true>, TRR_SMEM); e != cudaSuccess) return e;
            k_trsm_panel_rows<true><<<grid, TRR_NT, TRR_SMEM, s>>>(amap, A, lda, k0, nbk, n, dinfo);
        } else {
            if (cudaError_t e = smem_optin(k_trsm_panel_rows<false>, TRR_SMEM); e != cudaSuccess) return e;
            k_trsm_panel_rows<false><<<grid, TRR_NT, TRR_SMEM, s>>>(amap, A, lda, k0, nbk, n, dinfo);
        }
        note_launches(1);
        return cudaGetLastError();
    }
    if constexpr (std::is_same<T, double>::value && !UP) {
        const long long m = (long long)n - k0 - nbk;
        if (m <= 0) return cudaSuccess;
        const double md = (double)m, b = nbk;
        ProfScope ps(PK_TRSM_PANEL, s, md * b * b, sizeof(T) * (2.0 * md * b + b * (b + 1) / 2));
        const unsigned grid = (unsigned)ceil_div(m, TRD_NT);
        CUtensorMap amap{};
        if (nbk == 128 && !(lda & 1) &&
            tc::encode_colmajor_2d(&amap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, A, n, n, lda, 32, 32,
                                   CU_TENSOR_MAP_SWIZZLE_NONE)) {
            if (cudaError_t e = smem_optin(k_trsm_panel_rows_f64<2>, TRD_SMEM); e != cudaSuccess) return e;
            k_trsm_panel_rows_f64<2><<<grid, TRD_NT, TRD_SMEM, s>>>(amap, A, lda, 0, k0, nbk, n, dinfo);
        } else {
            if (cudaError_t e = smem_optin(k_trsm_panel_rows_f64<0>, TRD_SMEM); e != cudaSuccess) return e;
            k_trsm_panel_rows_f64<0><<<grid, TRD_NT, TRD_SMEM, s>>>(amap, A, lda, 0, k0, nbk, n, dinfo);
        }
        note_launches(1);
        return cudaGetLastError();
    }
    constexpr int NQ = potrf_nb<T>() / 32;
    constexpr int PR = sizeof(T) >= 16 ? 4 : 8;
    const size_t panel_smem = (size_t)(NQ * 32) * (NQ * 32 + 1) * sizeof(T);
    const long long m = (long long)n - k0 - nbk;
    if (m <= 0) return cudaSuccess;
    if (cudaError_t e = smem_optin(k_trsm_panel<T, UP, NQ, PR>, panel_smem); e != cudaSuccess) return e;
    const double cf = Traits<T>::cplx ? 4.0 : 1.0, md = (double)m, b = nbk;
    ProfScope ps(PK_TRSM_PANEL, s, cf * md * b * b, sizeof(T) * (2.0 * md * b + b * (b + 1) / 2));
    const long long grid = trsm_grid(k_trsm_panel<T, UP, NQ, PR>, panel_smem, ceil_div(m, 8 * PR));
    k_trsm_panel<T, UP, NQ, PR><<<(unsigned)grid, 256, panel_smem, s>>>(A, lda, k0, nbk, n, dinfo);
    note_launches(1);
    return cudaGetLastError();
}
template cudaError_t launch_trsm_panel<float, false>(float*, long long, int, int, int, const int*, cudaStream_t);

namespace {
struct LookaheadRes {
    cudaStream_t hi = nullptr;
    cudaEvent_t start = nullptr, panel = nullptr, rest = nullptr;
};
LookaheadRes& lookahead_res()
{
    static thread_local LookaheadRes res[64];
    int dev = 0;
    cudaGetDevice(&dev);
    LookaheadRes& r = res[dev & 63];
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
}  // namespace

template <class T, bool UP>
static cudaError_t potrf_enqueue(T* A, long long lda, int n, int G, int* dinfo, cudaStream_t st)
{
    constexpr int NB = potrf_nb<T>();
    constexpr int NQ = NB / 32;
    constexpr int PR = sizeof(T) >= 16 ? 4 : 8;
    const size_t diag_smem = (size_t)NB * diag_block_ld<T>(NB) * sizeof(T);
    const size_t panel_smem = (size_t)(NQ * 32) * (NQ * 32 + 1) * sizeof(T);
    if (cudaError_t e = smem_optin(k_potrf_diag<T, UP>, diag_smem); e != cudaSuccess) return e;
    if (cudaError_t e = smem_optin(k_trsm_panel<T, UP, NQ, PR>, panel_smem); e != cudaSuccess) return e;
    const double cf = Traits<T>::cplx ? 4.0 : 1.0;  // real flops per multiply-add relative to a real one
    LookaheadRes& L = lookahead_res();
    cudaStream_t hi = L.hi;

    cudaError_t panel_err = cudaSuccess;
    auto diag_and_panel = [&](int k0, cudaStream_t s) {
        const int nbk = n - k0 < NB ? n - k0 : NB;
        const double b = nbk;
        {
            ProfScope ps(PK_POTRF_DIAG, s, cf * b * b * b / 3.0, sizeof(T) * b * (b + 1));
            k_potrf_diag<T, UP><<<1, 256, (size_t)nbk * diag_block_ld<T>(nbk) * sizeof(T), s>>>(A, lda, 0, k0, nbk,
                                                                                              dinfo);
        }
        note_launches(1);
        const long long m = (long long)n - k0 - nbk;
        if (m <= 0) return;
        if constexpr ((std::is_same<T, double>::value || std::is_same<T, float>::value) && !UP) {
            const cudaError_t pe = launch_trsm_panel<T, UP>(A, lda, k0, nbk, n, dinfo, s);  // one thread per row
            if (pe != cudaSuccess && panel_err == cudaSuccess) panel_err = pe;
            return;
        }
        const double md = (double)m;
        {
            ProfScope ps(PK_TRSM_PANEL, s, cf * md * b * b, sizeof(T) * (2.0 * md * b + b * (b + 1) / 2));
            const long long grid = trsm_grid(k_trsm_panel<T, UP, NQ, PR>, panel_smem, ceil_div(m, 8 * PR));
            k_trsm_panel<T, UP, NQ, PR><<<(unsigned)grid, 256, panel_smem, s>>>(A, lda, k0, nbk, n, dinfo);
        }
        note_launches(1);
    };
    // C -= L(:, k0 : k0 + kw) L(:, k0 : k0 + kw)^H on the region from row / column t0
    auto update = [&](int k0, int kw, long long t0, int cols, cudaStream_t s) -> cudaError_t {
        const double md = (double)(n - t0), b = kw;
        const double cw = cols ? (double)cols : md;
        const double fl = cols ? cf * 2.0 * b * (md * cw - cw * (cw - 1) / 2) : cf * md * (md + 1) * b;
        ProfScope ps(PK_SYRK_UPDATE, s, fl, sizeof(T) * ((cols ? 2.0 * md * cw : md * (md + 1)) + md * b));
        const cudaError_t e = trailing_update<T, UP>(A, lda, k0, kw, n, t0, cols, dinfo, s);
        note_launches(1);
        return e;
    };

    // Super-steps of G block columns: the chain on the high-priority stream factors
    // them one after the other (block g first takes the left-looking update from
    // blocks 0..g-1 of the super-step), then updates the next super-step's G block
    // columns (look-ahead); the caller's stream updates everything to their right
    // with K = G NB in one pass, so the trailing matrix is read and written once
    // per G block columns.  The caller's stream waits for the super-step's panels;
    // the chain waits for the previous trailing update before its look-ahead; the
    // two touch disjoint tiles.
    const long long SW = (long long)G * NB;
    cudaEventRecord(L.start, st);
    cudaStreamWaitEvent(hi, L.start, 0);
    bool have_rest = false;
    cudaError_t e = cudaSuccess;
    for (long long k0 = 0; k0 < n; k0 += SW) {
        for (int g = 0; g < G; ++g) {
            const long long kg = k0 + (long long)g * NB;
            if (kg >= n) break;
            if (g > 0) {
                const int cols = (long long)n - kg < NB ? (int)(n - kg) : NB;
                if ((e = update((int)k0, g * NB, kg, cols, hi)) != cudaSuccess) return e;
            }
            diag_and_panel((int)kg, hi);
        }
        const long long t0 = k0 + SW;
        if (t0 >= n) break;
        cudaEventRecord(L.panel, hi);
        if (have_rest) cudaStreamWaitEvent(hi, L.rest, 0);
        const int la_cols = (long long)n - t0 < SW ? (int)(n - t0) : (int)SW;
        if ((e = update((int)k0, (int)SW, t0, la_cols, hi)) != cudaSuccess) return e;
        have_rest = false;
        if (t0 + SW < n) {
            cudaStreamWaitEvent(st, L.panel, 0);
            if ((e = update((int)k0, (int)SW, t0 + SW, 0, st)) != cudaSuccess) return e;
            cudaEventRecord(L.rest, st);
            have_rest = true;
        }
    }
    // join
    cudaEventRecord(L.panel, hi);
    cudaStreamWaitEvent(st, L.panel, 0);
    if (panel_err != cudaSuccess) return panel_err;
    return cudaGetLastError();
}

template <class T>
static cudaError_t potrf_typed(char uplo, int n, int G, void* A, long long lda, int* dinfo, cudaStream_t st)
{
    if (uplo == 'U') return potrf_enqueue<T, true>(static_cast<T*>(A), lda, n, G, dinfo, st);
    return potrf_enqueue<T, false>(static_cast<T*>(A), lda, n, G, dinfo, st);
}

}  // namespace ddlak

// ---------------------------------------------------------------------------
// L L^T x = b for a batch of factored equal-order FP64 matrices (lower, order
// <= 1024, one right-hand side each), one CTA per matrix with x in shared
// memory; log det = 2 sum log l_ii on the way.  Forward, by 32-row blocks: warp
// 0 solves the block (lane i owns row i; x_j = x_j / l_jj, then broadcast),
// every thread updates its rows below with the block's 32 columns (coalesced
// column reads).  Backward, by 32-row blocks from the end: each warp forms the
// dot products of some of the block's columns with the solved x below
// (coalesced, warp sums), then warp 0 solves the transposed block from a
// shared copy.  A matrix with info != 0 keeps b and gets log det = NaN.
// ---------------------------------------------------------------------------
constexpr int PB_NT = 256, PB_NMAX = 1024;

__global__ void __launch_bounds__(PB_NT) k_potrs_batched_f64(int n, const double* __restrict__ Lg, long long lda,
                                                             long long astride, double* __restrict__ Bg,
                                                             long long bstride, const int* __restrict__ info,
                                                             double* __restrict__ logdet)
{
    __shared__ double x[PB_NMAX];
    __shared__ double blk[32][33];
    __shared__ double s_ld;
    const int m = blockIdx.x, t = threadIdx.x, warp = t >> 5, lane = t & 31;
    if (info[m] != 0) {
        if (t == 0 && logdet) logdet[m] = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    const double* L = Lg + (long long)m * astride;
    double* B = Bg + (long long)m * bstride;
    for (int i = t; i < n; i += PB_NT) x[i] = B[i];
    double ld = 0.0;  // warp 0: sum of log l_ii over the rows its lanes own
    __syncthreads();
    for (int b0 = 0; b0 < n; b0 += 32) {
        const int w = n - b0 < 32 ? n - b0 : 32;
        // the block's lower triangle into shared memory first (all warps, coalesced), so that
        // warp 0's chain reads no global memory
        for (int e = t; e < 32 * 32; e += PB_NT) {
            const int r = e & 31, c = e >> 5;
            blk[r][c] = (r < w && c <= r) ? L[(b0 + r) + (long long)(b0 + c) * lda] : 0.0;
        }
        __syncthreads();
        if (warp == 0) {
            double xi = lane < w ? x[b0 + lane] : 0.0;
            for (int j = 0; j < w; ++j) {
                if (lane == j) {
                    const double d = blk[j][j];
                    xi = xi / d;
                    ld += log(d);
                }
                const double xj = __shfl_sync(0xffffffffu, xi, j);
                if (lane > j && lane < w) xi = fma(-blk[lane][j], xj, xi);
            }
            if (lane < w) x[b0 + lane] = xi;
        }
        __syncthreads();
        for (int r = b0 + 32 + t; r < n; r += PB_NT) {
            double acc = x[r];
            const double* lr = L + r + (long long)b0 * lda;
            for (int j = 0; j < w; ++j) acc = fma(-lr[(long long)j * lda], x[b0 + j], acc);
            x[r] = acc;
        }
        __syncthreads();
    }
    if (warp == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ld += __shfl_xor_sync(0xffffffffu, ld, o);
        if (lane == 0) s_ld = 2.0 * ld;
    }
    for (int b0 = ((n - 1) / 32) * 32; b0 >= 0; b0 -= 32) {
        const int w = n - b0 < 32 ? n - b0 : 32;
        // x_i -= sum_{r >= b0 + 32} l(r, b0 + i) x_r for the block's columns i
        for (int i = warp; i < w; i += PB_NT / 32) {
            const double* lc = L + (long long)(b0 + i) * lda;
            double acc = 0.0;
            for (int r = b0 + 32 + lane; r < n; r += 32) acc = fma(lc[r], x[r], acc);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) x[b0 + i] -= acc;
        }
        for (int e = t; e < 32 * 32; e += PB_NT) {  // the block itself, for the transposed solve
            const int r = e & 31, c = e >> 5;
            blk[r][c] = (r < w && c <= r) ? L[(b0 + r) + (long long)(b0 + c) * lda] : 0.0;
        }
        __syncthreads();
        if (warp == 0) {
            double xi = lane < w ? x[b0 + lane] : 0.0;
            for (int j = w - 1; j >= 0; --j) {
                if (lane == j) xi = xi / blk[j][j];
                const double xj = __shfl_sync(0xffffffffu, xi, j);
                if (lane < j) xi = fma(-blk[j][lane], xj, xi);
            }
            if (lane < w) x[b0 + lane] = xi;
        }
        __syncthreads();
    }
    for (int i = t; i < n; i += PB_NT) B[i] = x[i];
    if (t == 0 && logdet) logdet[m] = s_ld;
}

// A batch of equal-order FP64 matrices (lower), right-looking by super-steps of
// G block columns of 128, each step one launch per kernel over the whole batch:
// the diagonal blocks (one CTA per matrix), the panels (row-per-thread solve,
// grid.y = matrix) and the updates (TMA DMMA tiles, grid.y = matrix).  In a
// super-step, block column g first takes the update of its own 128 columns by
// block columns 0 .. g-1 (K = 128 g), and the rest of the trailing matrix is
// updated once with K = 128 G, so the trailing matrix is read and written once
// per 128 G columns and the update tiles run long K.
#ifndef BATCHED_POTRF_GROUP
#define BATCHED_POTRF_GROUP 4
#endif
extern "C" int ddlak_potrf_batched_f64(int batch, int n, void* A_, long long lda, long long astride, int* dinfo,
                                       void* stream)
{
    using namespace ddlak;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double* A = static_cast<double*>(A_);
    if (batch < 0 || n < 0 || (batch > 0 && (!A || !dinfo || lda < n || astride < lda * (long long)n)))
        return (int)cudaErrorInvalidValue;
    if (batch == 0) return 0;
    if (batch > 65535 || (lda & 1) || (astride & 1) || (reinterpret_cast<uintptr_t>(A) & 15))
        return (int)cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(dinfo, 0, sizeof(int) * (size_t)batch, st);
    if (e != cudaSuccess || n == 0) return (int)e;
    constexpr int NB = 128, G = BATCHED_POTRF_GROUP;
    const size_t diag_smem = (size_t)NB * diag_block_ld<double>(NB) * sizeof(double);
    if ((e = smem_optin(k_potrf_diag<double, false>, diag_smem)) != cudaSuccess) return (int)e;
    if ((e = smem_optin(k_trsm_panel_rows_f64<3>, TRD_SMEM)) != cudaSuccess) return (int)e;
    if ((e = smem_optin(k_trsm_panel_rows_f64<0>, TRD_SMEM)) != cudaSuccess) return (int)e;
    // L11 of every matrix by TMA boxes of 32 x 32 (lda and astride even, A 16-byte aligned: checked above)
    CUtensorMap amap{};
    const bool tma = tc::encode_colmajor_3d(&amap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, A, n, n, lda, batch, astride,
                                            32, 32);
    const double nb3 = (double)batch;
    auto diag_and_panel = [&](int k0) -> cudaError_t {
        const int nbk = n - k0 < NB ? n - k0 : NB;
        const double b = nbk;
        {
            ProfScope ps(PK_POTRF_DIAG, st, nb3 * b * b * b / 3.0, nb3 * 8.0 * b * (b + 1));
            k_potrf_diag<double, false><<<(unsigned)batch, 256, (size_t)nbk * diag_block_ld<double>(nbk) * 8, st>>>(
                A, lda, astride, k0, nbk, dinfo);
        }
        note_launches(1);
        const long long m = (long long)n - k0 - nbk;
        if (m > 0) {
            const double md = (double)m;
            ProfScope ps(PK_TRSM_PANEL, st, nb3 * md * b * b, nb3 * 8.0 * (2.0 * md * b + b * (b + 1) / 2));
            const dim3 grid((unsigned)ceil_div(m, TRD_NT), (unsigned)batch);
            if (tma && nbk == 128)
                k_trsm_panel_rows_f64<3><<<grid, TRD_NT, TRD_SMEM, st>>>(amap, A, lda, astride, k0, nbk, n, dinfo);
            else
                k_trsm_panel_rows_f64<0><<<grid, TRD_NT, TRD_SMEM, st>>>(amap, A, lda, astride, k0, nbk, n, dinfo);
            note_launches(1);
        }
        return cudaGetLastError();
    };
    // C -= L(:, k0 : k0 + kw) L(:, k0 : k0 + kw)^T on the region from t0 (all of it, or cols columns)
    auto update = [&](int k0, int kw, long long t0, int cols) -> cudaError_t {
        const double md = (double)(n - t0), b = kw;
        const double cw = cols ? (double)cols : md;
        const double fl = cols ? 2.0 * b * (md * cw - cw * (cw - 1) / 2) : md * (md + 1) * b;
        ProfScope ps(PK_SYRK_UPDATE, st, nb3 * fl, nb3 * 8.0 * ((cols ? 2.0 * md * cw : md * (md + 1)) + md * b));
        cudaError_t ue = cudaSuccess;
        if (!launch_dmma_tma_batched(A, lda, astride, batch, k0, kw, n, t0, cols, dinfo, st, &ue))
            return cudaErrorInvalidValue;
        note_launches(1);
        return ue;
    };
    for (int k0 = 0; k0 < n; k0 += G * NB) {
        if ((e = diag_and_panel(k0)) != cudaSuccess) return (int)e;
        // block column g of the super-step: the update of its own columns by block columns
        // 0 .. g-1 of the super-step (left-looking, K = 128 g), then its factor
        for (int g = 1; g < G; ++g) {
            const int kg = k0 + g * NB;
            if (kg >= n) break;
            const int cg = n - kg < NB ? n - kg : NB;
            if ((e = update(k0, g * NB, kg, cg)) != cudaSuccess) return (int)e;
            if ((e = diag_and_panel(kg)) != cudaSuccess) return (int)e;
        }
        const long long t0 = (long long)k0 + G * NB;
        if (t0 >= n) break;
        if ((e = update(k0, G * NB, t0, 0)) != cudaSuccess) return (int)e;
    }
    return (int)cudaGetLastError();
}

extern "C" int ddlak_potrs_batched_f64(int batch, int n, const void* L, long long lda, long long astride, void* B,
                                       long long bstride, const int* dinfo, double* logdet, void* stream)
{
    using namespace ddlak;
    if (batch < 0 || n < 0 || n > PB_NMAX) return (int)cudaErrorInvalidValue;
    if (batch == 0 || n == 0) return 0;
    if (!L || !B || !dinfo || lda < n || astride < lda * (long long)n || bstride < n)
        return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const double nn = n;
    ProfScope ps(PK_POTRS_FUSED, st, 2.0 * batch * nn * nn, 8.0 * batch * nn * (nn + 1));
    k_potrs_batched_f64<<<(unsigned)batch, PB_NT, 0, st>>>(n, static_cast<const double*>(L), lda, astride,
                                                         static_cast<double*>(B), bstride, dinfo, logdet);
    note_launches(1);
    return (int)cudaGetLastError();
}

extern "C" int ddlak_potrf_grouped(char type, char uplo, int group, int n, void* A, long long lda, int* dinfo,
                                   void* stream)
{
    using namespace ddlak;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (group < 1 || group > DDLAK_POTRF_MAX_GROUP) return (int)cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(dinfo, 0, sizeof(int), st);
    if (e != cudaSuccess) return (int)e;
    if (n <= 0) return 0;
    switch (type) {
    case 's': e = potrf_typed<float>(uplo, n, group, A, lda, dinfo, st); break;
    case 'd': e = potrf_typed<double>(uplo, n, group, A, lda, dinfo, st); break;
    case 'c': e = potrf_typed<cf32>(uplo, n, group, A, lda, dinfo, st); break;
    case 'z': e = potrf_typed<cf64>(uplo, n, group, A, lda, dinfo, st); break;
    default: return (int)cudaErrorInvalidValue;
    }
    return (int)e;
}

extern "C" int ddlak_potrf(char type, char uplo, int n, void* A, long long lda, int* dinfo, void* stream)
{
    return ddlak_potrf_grouped(type, uplo, DDLAK_POTRF_GROUP, n, A, lda, dinfo, stream);
}
