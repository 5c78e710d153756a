// Fused forward + backward substitution with a Cholesky factor (ddla::ppotrs on
// a 1x1 grid).
//
// The reference applies two vendor triangular solves, L then L^H
// (src/Cholesky/ppotrs.cpp:44-61 -> src/PBLAS/ptrtrs.cpp:150-155 ->
// src/BLAS/trsm.cpp:154-159, cublas?trsm).  Here both solves are ONE launch:
// the solution is split into block rows of RB rows and every CTA takes a
// ticket from a global counter.  Tickets 0..N-1 solve the forward block rows
// 0..N-1 (L Y = B), tickets N..2N-1 the backward block rows N-1..0
// (L^H X = Y).  A CTA only ever waits for a block row published under a
// smaller ticket, and every smaller ticket belongs to a CTA that has already
// started, so the waits always end; each wait is additionally bounded by a
// clock budget and reports DDLAK_WAIT_TIMEOUT instead of spinning forever.
//
// The right-hand sides are a view X(i, r): B[i + r*ldb] for side 'L' and
// conj(B[r + i*ldb]) for side 'R' (X * A = B  <=>  A * X^H = B^H, since A is
// Hermitian).  They are processed in chunks of RC columns; chunk c uses its own
// flag row and tickets interleave chunks so the ordering argument holds per
// chunk.
#include "common.cuh"
#include "ddla_kernels_internal.h"
#include "profile.h"

namespace ddlak {

namespace {

constexpr int RB = 64;   // rows per block row
constexpr int RC = 16;   // right-hand sides per chunk
constexpr int NT = 256;  // threads per CTA

template <class T, bool BT>
__device__ __forceinline__ T x_ld(const T* B, long long ldb, long long i, long long r)
{
    if (BT) return cj(B[r + i * ldb]);
    return B[i + r * ldb];
}
template <class T, bool BT>
__device__ __forceinline__ T x_ld_cg(const T* B, long long ldb, long long i, long long r)
{
    const T* p = BT ? B + r + i * ldb : B + i + r * ldb;
    T v;
    if constexpr (sizeof(T) == 4) { float t = __ldcg(reinterpret_cast<const float*>(p)); v = *reinterpret_cast<T*>(&t); }
    else if constexpr (sizeof(T) == 8) { double t = __ldcg(reinterpret_cast<const double*>(p)); v = *reinterpret_cast<T*>(&t); }
    else { double2 t = __ldcg(reinterpret_cast<const double2*>(p)); v = *reinterpret_cast<T*>(&t); }
    return BT ? cj(v) : v;
}
template <class T, bool BT>
__device__ __forceinline__ void x_st(T* B, long long ldb, long long i, long long r, T v)
{
    if (BT) B[r + i * ldb] = cj(v);
    else B[i + r * ldb] = v;
}

template <class T, bool UP, bool BT>
__global__ void __launch_bounds__(NT) k_potrs_fused(const T* __restrict__ A, long long lda, T* B, long long ldb, int n,
                                                    int nrhs, int nchunks, int* flags, int* ticket, int* status)
{
    using R = real_t<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T (*Ls)[RB + 1] = reinterpret_cast<T (*)[RB + 1]>(smem_raw);                 // off-diagonal tile, Ls[k][i]
    T (*Xs)[RC + 1] = reinterpret_cast<T (*)[RC + 1]>(smem_raw + sizeof(T) * RB * (RB + 1));  // other row's block
    T (*acc_s)[RC + 1] = Xs + RB;
    __shared__ int s_t;
    __shared__ int s_abort;
    if (threadIdx.x == 0) { s_t = atomicAdd(ticket, 1); s_abort = 0; }
    __syncthreads();
    const int N = (int)ceil_div(n, RB);
    const int t = s_t;
    const int chunk = t % nchunks;
    const int step = t / nchunks;
    const bool fwd = step < N;
    const int blk = fwd ? step : 2 * N - 1 - step;
    int* cflags = flags + (size_t)chunk * 2 * N;  // [0,N) forward, [N,2N) backward
    const long long r0 = (long long)chunk * RC;
    const int nr = (int)((nrhs - r0) < RC ? (nrhs - r0) : RC);
    const long long i0 = (long long)blk * RB;
    const int nrows = (int)((n - i0) < RB ? (n - i0) : RB);

    // thread -> (row, rhs group): rows tid%64, rhs (tid/64) + 4*q
    const int tr = threadIdx.x & (RB - 1);
    const int tg = threadIdx.x >> 6;
    T acc[RC / 4];

    if (!fwd) {
        // the block row's own forward result must be published first
        if (threadIdx.x == 0) {
            if (!bounded_wait_geq(&cflags[blk], 1, status)) s_abort = 1;
            __threadfence();
        }
        __syncthreads();
        if (s_abort) return;
    }
#pragma unroll
    for (int q = 0; q < RC / 4; ++q) {
        const int r = tg + 4 * q;
        acc[q] = (tr < nrows && r < nr) ? x_ld_cg<T, BT>(B, ldb, i0 + tr, r0 + r) : zero<T>();
    }

    const int jbeg = fwd ? 0 : blk + 1;
    const int jend = fwd ? blk : N;
    for (int j = jbeg; j < jend; ++j) {
        const long long j0 = (long long)j * RB;
        const int ncols = (int)((n - j0) < RB ? (n - j0) : RB);
        // tile: forward L(i0+i, j0+k); backward L^H(i0+i, j0+k) = conj(L(j0+k, i0+i))
        for (int idx = threadIdx.x; idx < RB * RB; idx += NT) {
            int i, k;
            if (fwd != UP) { i = idx % RB; k = idx / RB; } else { k = idx % RB; i = idx / RB; }
            T v = zero<T>();
            if (i < nrows && k < ncols)
                v = fwd ? lview_ld<T, UP>(A, lda, i0 + i, j0 + k) : cj(lview_ld<T, UP>(A, lda, j0 + k, i0 + i));
            Ls[k][i] = v;
        }
        if (threadIdx.x == 0) {
            if (!bounded_wait_geq(&cflags[fwd ? j : N + j], 1, status)) s_abort = 1;
            __threadfence();
        }
        __syncthreads();
        if (s_abort) return;
        for (int idx = threadIdx.x; idx < RB * RC; idx += NT) {
            const int k = idx % RB, r = idx / RB;
            Xs[k][r] = (k < ncols && r < nr) ? x_ld_cg<T, BT>(B, ldb, j0 + k, r0 + r) : zero<T>();
        }
        __syncthreads();
#pragma unroll 8
        for (int k = 0; k < RB; ++k) {
            const T l = Ls[k][tr];
#pragma unroll
            for (int q = 0; q < RC / 4; ++q) acc[q] = fms(acc[q], l, Xs[k][tg + 4 * q]);
        }
        __syncthreads();
    }

    // diagonal block: forward solves L_bb y = acc, backward L_bb^H x = acc
    for (int idx = threadIdx.x; idx < RB * RB; idx += NT) {
        const int i = idx % RB, k = idx / RB;
        // Ls[k][i] = L_bb(i, k) for i >= k
        Ls[k][i] = (i < nrows && k < nrows && i >= k) ? lview_ld<T, UP>(A, lda, i0 + i, i0 + k) : zero<T>();
    }
#pragma unroll
    for (int q = 0; q < RC / 4; ++q) acc_s[tr][tg + 4 * q] = acc[q];
    __syncthreads();
    {
        // 8 warps x 2 rhs columns; lanes own rows lane and lane+32
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        for (int rr = 0; rr < RC / 8; ++rr) {
            const int r = warp * (RC / 8) + rr;
            T v0 = acc_s[lane][r], v1 = acc_s[lane + 32][r];
            if (fwd) {
                for (int k = 0; k < nrows; ++k) {
                    const R dkk = re(Ls[k][k]);
                    T xk;
                    if (k < 32) {
                        if (lane == k) v0 = divr(v0, dkk);
                        xk = v0;
                        if constexpr (Traits<T>::cplx) {
                            xk.x = __shfl_sync(0xffffffffu, xk.x, k);
                            xk.y = __shfl_sync(0xffffffffu, xk.y, k);
                        } else xk = __shfl_sync(0xffffffffu, xk, k);
                        if (lane > k) v0 = fms(v0, Ls[k][lane], xk);
                        v1 = fms(v1, Ls[k][lane + 32], xk);
                    } else {
                        if (lane == k - 32) v1 = divr(v1, dkk);
                        xk = v1;
                        if constexpr (Traits<T>::cplx) {
                            xk.x = __shfl_sync(0xffffffffu, xk.x, k - 32);
                            xk.y = __shfl_sync(0xffffffffu, xk.y, k - 32);
                        } else xk = __shfl_sync(0xffffffffu, xk, k - 32);
                        if (lane + 32 > k) v1 = fms(v1, Ls[k][lane + 32], xk);
                    }
                }
            } else {
                for (int k = nrows - 1; k >= 0; --k) {
                    const R dkk = re(Ls[k][k]);
                    T xk;
                    // x_k = v_k / d_kk;  v_i -= conj(L(k, i)) x_k for i < k
                    if (k < 32) {
                        if (lane == k) v0 = divr(v0, dkk);
                        xk = v0;
                        if constexpr (Traits<T>::cplx) {
                            xk.x = __shfl_sync(0xffffffffu, xk.x, k);
                            xk.y = __shfl_sync(0xffffffffu, xk.y, k);
                        } else xk = __shfl_sync(0xffffffffu, xk, k);
                        if (lane < k) v0 = fms(v0, cj(Ls[lane][k]), xk);
                    } else {
                        if (lane == k - 32) v1 = divr(v1, dkk);
                        xk = v1;
                        if constexpr (Traits<T>::cplx) {
                            xk.x = __shfl_sync(0xffffffffu, xk.x, k - 32);
                            xk.y = __shfl_sync(0xffffffffu, xk.y, k - 32);
                        } else xk = __shfl_sync(0xffffffffu, xk, k - 32);
                        if (lane + 32 < k) v1 = fms(v1, cj(Ls[lane + 32][k]), xk);
                        v0 = fms(v0, cj(Ls[lane][k]), xk);
                    }
                }
            }
            acc_s[lane][r] = v0;
            acc_s[lane + 32][r] = v1;
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < RB * RC; idx += NT) {
        const int i = idx % RB, r = idx / RB;
        if (i < nrows && r < nr) x_st<T, BT>(B, ldb, i0 + i, r0 + r, acc_s[i][r]);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) st_release(&cflags[fwd ? blk : N + blk], 1);
}

template <class T, bool UP, bool BT>
cudaError_t potrs_launch(const T* A, long long lda, T* B, long long ldb, int n, int nrhs, int* flags, int* ticket,
                         int* status, cudaStream_t st)
{
    const int N = (int)ceil_div(n, RB);
    const int nchunks = (int)ceil_div(nrhs, RC);
    const long long grid = 2LL * N * nchunks;
    const size_t smem = sizeof(T) * ((size_t)RB * (RB + 1) + 2 * (size_t)RB * (RC + 1));
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_potrs_fused<T, UP, BT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    const double cf = Traits<T>::cplx ? 4.0 : 1.0;
    const double nd = n, rd = nrhs;
    ProfScope ps(PK_POTRS_FUSED, st, cf * 2.0 * nd * nd * rd, sizeof(T) * (nd * (nd + 1) + 4.0 * nd * rd));
    k_potrs_fused<T, UP, BT><<<(unsigned)grid, NT, smem, st>>>(A, lda, B, ldb, n, nrhs, nchunks, flags, ticket,
                                                                status);
    note_launches(1);
    return cudaGetLastError();
}

template <class T>
cudaError_t potrs_typed(char uplo, char side, int n, int nrhs, const void* A, long long lda, void* B, long long ldb,
                        int* flags, int* ticket, int* status, cudaStream_t st)
{
    const T* a = static_cast<const T*>(A);
    T* b = static_cast<T*>(B);
    const bool up = uplo == 'U', bt = side == 'R';
    if (up && bt) return potrs_launch<T, true, true>(a, lda, b, ldb, n, nrhs, flags, ticket, status, st);
    if (up) return potrs_launch<T, true, false>(a, lda, b, ldb, n, nrhs, flags, ticket, status, st);
    if (bt) return potrs_launch<T, false, true>(a, lda, b, ldb, n, nrhs, flags, ticket, status, st);
    return potrs_launch<T, false, false>(a, lda, b, ldb, n, nrhs, flags, ticket, status, st);
}

}  // namespace
}  // namespace ddlak

// Scratch: [status int][ticket int] padded to 256 B, then nchunks * 2N flags.
extern "C" unsigned long long ddlak_potrs_workspace(int n, int nrhs)
{
    if (n <= 0 || nrhs <= 0) return 0;
    const unsigned long long N = (unsigned long long)ddlak::ceil_div(n, ddlak::RB);
    const unsigned long long C = (unsigned long long)ddlak::ceil_div(nrhs, ddlak::RC);
    return 256 + ((C * 2 * N * sizeof(int) + 255) / 256) * 256;
}

extern "C" int ddlak_potrs(char type, char uplo, char side, int n, int nrhs, const void* A, long long lda, void* B,
                           long long ldb, void* work, unsigned long long work_bytes, void* stream)
{
    using namespace ddlak;
    if (n <= 0 || nrhs <= 0) return 0;
    if (work_bytes < ddlak_potrs_workspace(n, nrhs)) return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(work, 0, ddlak_potrs_workspace(n, nrhs), st);
    if (e != cudaSuccess) return (int)e;
    int* status = static_cast<int*>(work);
    int* ticket = status + 1;
    int* flags = reinterpret_cast<int*>(static_cast<char*>(work) + 256);
    switch (type) {
    case 's': e = potrs_typed<float>(uplo, side, n, nrhs, A, lda, B, ldb, flags, ticket, status, st); break;
    case 'd': e = potrs_typed<double>(uplo, side, n, nrhs, A, lda, B, ldb, flags, ticket, status, st); break;
    case 'c': e = potrs_typed<cf32>(uplo, side, n, nrhs, A, lda, B, ldb, flags, ticket, status, st); break;
    case 'z': e = potrs_typed<cf64>(uplo, side, n, nrhs, A, lda, B, ldb, flags, ticket, status, st); break;
    default: return (int)cudaErrorInvalidValue;
    }
    return (int)e;
}
