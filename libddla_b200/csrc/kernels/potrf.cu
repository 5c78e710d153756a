// Blocked right-looking Cholesky (ddla::ppotrf / ddla::potrf on a 1x1 grid).
//
// Replaces the vendor call the reference makes at src/Cholesky/potrf.cpp:106-113
// (cusolverDn?potrf) with three kernels per block column k:
//   1. k_potrf_diag   -- the nb x nb diagonal block factored in shared memory,
//                        one __syncthreads per column, info detected in-kernel;
//   2. k_trsm_panel   -- L21 = A21 * L11^{-H}, row blocks owned by warps, columns
//                        by lanes, warp-shuffle broadcast of each solved entry;
//   3. trailing update -- C -= L21 * L21^H on the lower tiles of the trailing
//                        matrix (FP64 DMMA tiles for double, see syrk.cu).
// info follows LAPACK ?potrf: the order of the first leading minor that is not
// positive definite (diagonal value <= 0 or NaN), 0 on success.  Every kernel
// returns immediately once info is set, so the first failure is the one kept.
#include "common.cuh"
#include "ddla_kernels_internal.h"
#include "profile.h"

namespace ddlak {

// ---------------------------------------------------------------------------
// 1. diagonal block
// ---------------------------------------------------------------------------
template <class T, bool UP>
__global__ void __launch_bounds__(256) k_potrf_diag(T* __restrict__ A, long long lda, int k0, int nbk,
                                                    int* __restrict__ info)
{
    using R = real_t<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* s = reinterpret_cast<T*>(smem_raw);
    const int ld = nbk + 1;
    if (*(volatile int*)info != 0) return;

    for (int idx = threadIdx.x; idx < nbk * nbk; idx += blockDim.x) {
        const int i = idx % nbk, j = idx / nbk;
        if (i >= j) s[i + j * ld] = lview_ld<T, UP>(A, lda, k0 + i, k0 + j);
    }
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    int fail = 0;
    R dprev = R(1);
    for (int j = 0; j < nbk; ++j) {
        const R d = re(s[j + j * ld]);
        // Column j-1 was last read by the previous iteration's update: scale it now.
        if (j > 0) {
            const R inv = R(1) / sqrt(dprev);
            for (int i = j + threadIdx.x; i < nbk; i += blockDim.x) s[i + (j - 1) * ld] = scal(s[i + (j - 1) * ld], inv);
            if (threadIdx.x == 0) s[(j - 1) + (j - 1) * ld] = from_real<T>(sqrt(dprev));
        }
        if (!(d > R(0))) { fail = j + 1; break; }
        const R invd = R(1) / d;
        for (int k = j + 1 + warp; k < nbk; k += nw) {
            const T lkj = scal(cj(s[k + j * ld]), invd);
            for (int i = k + lane; i < nbk; i += 32) s[i + k * ld] = fms(s[i + k * ld], s[i + j * ld], lkj);
        }
        dprev = d;
        __syncthreads();
    }
    if (!fail) {
        const int j = nbk;
        const R inv = R(1) / sqrt(dprev);
        for (int i = j + threadIdx.x; i < nbk; i += blockDim.x) s[i + (j - 1) * ld] = scal(s[i + (j - 1) * ld], inv);
        if (threadIdx.x == 0) s[(j - 1) + (j - 1) * ld] = from_real<T>(sqrt(dprev));
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < nbk * nbk; idx += blockDim.x) {
        const int i = idx % nbk, j = idx / nbk;
        if (i >= j) lview_st<T, UP>(A, lda, k0 + i, k0 + j, s[i + j * ld]);
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
    if (*(volatile int*)info != 0) return;

    for (int idx = threadIdx.x; idx < NQ * 32 * NQ * 32; idx += blockDim.x) {
        const int c = idx % (NQ * 32), j = idx / (NQ * 32);
        T v = zero<T>();
        if (c < nbk && j < nbk && c >= j) v = lview_ld<T, UP>(A, lda, k0 + c, k0 + j);
        l11[c + j * ldl] = v;
    }
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long row0 = (long long)k0 + nbk + ((long long)blockIdx.x * (blockDim.x >> 5) + warp) * PR;
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
            const R djj = re(l11[j + j * ldl]);
            T x[PR];
#pragma unroll
            for (int r = 0; r < PR; ++r) {
                T v = divr(p[r][qj], djj);
                if (lane == jj) p[r][qj] = v;
                if constexpr (Traits<T>::cplx) {
                    v.x = __shfl_sync(0xffffffffu, v.x, jj);
                    v.y = __shfl_sync(0xffffffffu, v.y, jj);
                } else {
                    v = __shfl_sync(0xffffffffu, v, jj);
                }
                x[r] = v;
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

// ---------------------------------------------------------------------------
// 3. generic trailing update (SIMT; every type).  64x64 tiles of the lower
//    trailing matrix, 16-wide k chunks through shared memory, 4x4 per thread.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tri_tile(long long b, int& I, int& J)
{
    long long i = (long long)((sqrt(8.0 * (double)b + 1.0) - 1.0) * 0.5);
    while ((i + 1) * (i + 2) / 2 <= b) ++i;
    while (i * (i + 1) / 2 > b) --i;
    I = (int)i;
    J = (int)(b - i * (i + 1) / 2);
}

template <class T, bool UP>
__global__ void __launch_bounds__(256) k_syrk_simt(T* __restrict__ A, long long lda, int k0, int nbk, int n,
                                                   const int* __restrict__ info)
{
    constexpr int BT = 64, BK = 16;
    __shared__ T As[BK][BT + 1];
    __shared__ T Bs[BK][BT + 1];
    if (*(volatile int*)info != 0) return;
    int I, J;
    tri_tile(blockIdx.x, I, J);
    const long long t0 = (long long)k0 + nbk;
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
            Bs[k][i] = (kin && rj + i < n) ? lview_ld<T, UP>(A, lda, rj + i, k0 + kc + k) : zero<T>();
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
            if (i < n && j < n && i >= j) {
                T c = lview_ld<T, UP>(A, lda, i, j);
                lview_st<T, UP>(A, lda, i, j, sub(c, acc[a][b]));
            }
        }
}

// ---------------------------------------------------------------------------
// host-side enqueue of the whole factorization
// ---------------------------------------------------------------------------
template <class T> constexpr int potrf_nb() { return sizeof(T) == 16 ? 64 : 128; }

template <class T, bool UP>
static cudaError_t potrf_enqueue(T* A, long long lda, int n, int* dinfo, cudaStream_t st)
{
    constexpr int NB = potrf_nb<T>();
    constexpr int NQ = NB / 32;
    constexpr int PR = sizeof(T) >= 16 ? 4 : 8;
    const size_t diag_smem = (size_t)NB * (NB + 1) * sizeof(T);
    const size_t panel_smem = (size_t)(NQ * 32) * (NQ * 32 + 1) * sizeof(T);
    static bool attr_done = false;
    if (!attr_done) {
        cudaFuncSetAttribute(k_potrf_diag<T, UP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)diag_smem);
        cudaFuncSetAttribute(k_trsm_panel<T, UP, NQ, PR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)panel_smem);
        attr_done = true;
    }
    const double cf = Traits<T>::cplx ? 4.0 : 1.0;  // real flops per multiply-add relative to a real one
    for (int k0 = 0; k0 < n; k0 += NB) {
        const int nbk = n - k0 < NB ? n - k0 : NB;
        const double b = nbk;
        {
            ProfScope ps(PK_POTRF_DIAG, st, cf * b * b * b / 3.0, sizeof(T) * b * (b + 1));
            k_potrf_diag<T, UP><<<1, 256, (size_t)nbk * (nbk + 1) * sizeof(T), st>>>(A, lda, k0, nbk, dinfo);
        }
        note_launches(1);
        const long long m = (long long)n - k0 - nbk;
        if (m <= 0) break;
        const int rows_per_cta = 8 * PR;
        const double md = (double)m;
        {
            ProfScope ps(PK_TRSM_PANEL, st, cf * md * b * b, sizeof(T) * (2.0 * md * b + b * (b + 1) / 2));
            k_trsm_panel<T, UP, NQ, PR><<<(unsigned)ceil_div(m, rows_per_cta), 256, panel_smem, st>>>(A, lda, k0,
                                                                                                       nbk, n, dinfo);
        }
        note_launches(1);
        {
            ProfScope ps(PK_SYRK_UPDATE, st, cf * md * (md + 1) * b, sizeof(T) * (md * (md + 1) + md * b));
            const cudaError_t e = trailing_update<T, UP>(A, lda, k0, nbk, n, dinfo, st);
            if (e != cudaSuccess) return e;
        }
        note_launches(1);
    }
    return cudaGetLastError();
}

template <class T, bool UP>
cudaError_t trailing_update_simt(T* A, long long lda, int k0, int nbk, int n, const int* dinfo, cudaStream_t st)
{
    const long long m = (long long)n - k0 - nbk;
    const long long t = ceil_div(m, 64);
    k_syrk_simt<T, UP><<<(unsigned)(t * (t + 1) / 2), 256, 0, st>>>(A, lda, k0, nbk, n, dinfo);
    return cudaSuccess;
}

template cudaError_t trailing_update_simt<float, false>(float*, long long, int, int, int, const int*, cudaStream_t);
template cudaError_t trailing_update_simt<float, true>(float*, long long, int, int, int, const int*, cudaStream_t);
template cudaError_t trailing_update_simt<double, false>(double*, long long, int, int, int, const int*, cudaStream_t);
template cudaError_t trailing_update_simt<double, true>(double*, long long, int, int, int, const int*, cudaStream_t);
template cudaError_t trailing_update_simt<cf32, false>(cf32*, long long, int, int, int, const int*, cudaStream_t);
template cudaError_t trailing_update_simt<cf32, true>(cf32*, long long, int, int, int, const int*, cudaStream_t);
template cudaError_t trailing_update_simt<cf64, false>(cf64*, long long, int, int, int, const int*, cudaStream_t);
template cudaError_t trailing_update_simt<cf64, true>(cf64*, long long, int, int, int, const int*, cudaStream_t);

template <class T>
static cudaError_t potrf_typed(char uplo, int n, void* A, long long lda, int* dinfo, cudaStream_t st)
{
    if (uplo == 'U') return potrf_enqueue<T, true>(static_cast<T*>(A), lda, n, dinfo, st);
    return potrf_enqueue<T, false>(static_cast<T*>(A), lda, n, dinfo, st);
}

}  // namespace ddlak

extern "C" int ddlak_potrf(char type, char uplo, int n, void* A, long long lda, int* dinfo, void* stream)
{
    using namespace ddlak;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(dinfo, 0, sizeof(int), st);
    if (e != cudaSuccess) return (int)e;
    if (n <= 0) return 0;
    switch (type) {
    case 's': e = potrf_typed<float>(uplo, n, A, lda, dinfo, st); break;
    case 'd': e = potrf_typed<double>(uplo, n, A, lda, dinfo, st); break;
    case 'c': e = potrf_typed<cf32>(uplo, n, A, lda, dinfo, st); break;
    case 'z': e = potrf_typed<cf64>(uplo, n, A, lda, dinfo, st); break;
    default: return (int)cudaErrorInvalidValue;
    }
    return (int)e;
}
