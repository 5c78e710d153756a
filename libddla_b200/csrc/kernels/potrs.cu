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
// Each CTA streams the off-diagonal tiles of its block row through a
// double-buffered cp.async ring (the tile loads do not depend on other CTAs,
// only the solved blocks do), visiting them in publication order, then solves
// its diagonal block with one warp per pair of right-hand sides using
// reciprocal pivots and warp shuffles.
//
// The right-hand sides are a view X(i, r): B[i + r*ldb] for side 'L' and
// conj(B[r + i*ldb]) for side 'R' (X * A = B  <=>  A * X^H = B^H, since A is
// Hermitian).  They are processed in chunks of RC columns; chunk c uses its own
// flag row and tickets interleave chunks so the ordering argument holds per
// chunk.
#include <mutex>

#include <ddla_kernels.h>

#include "common.cuh"
#include "ddla_kernels_internal.h"
#include "profile.h"

namespace ddlak {

namespace {

constexpr int RB = 64;   // rows per block row
constexpr int RC = 16;   // right-hand sides per chunk
constexpr int NT = 256;  // threads per CTA

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

__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <class T>
__device__ __forceinline__ T shfl_t(T v, int src)
{
    if constexpr (Traits<T>::cplx) {
        v.x = __shfl_sync(0xffffffffu, v.x, src);
        v.y = __shfl_sync(0xffffffffu, v.y, src);
        return v;
    } else {
        return __shfl_sync(0xffffffffu, v, src);
    }
}

// Shared-memory layout (elements of T unless noted):
//   Lbuf[2][RB][RB+1]  raw off-diagonal tiles, Lbuf[b][k][i]
//   Xs[RB][RC+1]       the solved block of the other block row
//   Acc[RB][RC+1]      this block row's right-hand sides
//   Rinv[RB]           reciprocal pivots (real type)
//   Ibuf[RB][RB+1]     (INV mode) the precomputed inverse of the diagonal block
// The factor is stored as TL and the right-hand sides as TX (TL == TX on the
// plain path; an FP32 factor with FP64 vectors for the mixed-precision solves).
template <class TL, class TX, bool INV = false>
__host__ __device__ constexpr size_t potrs_smem_bytes()
{
    return sizeof(TL) * 2 * (size_t)RB * (RB + 1) + sizeof(TX) * 2 * (size_t)RB * (RC + 1) + sizeof(real_t<TX>) * RB +
           (INV ? sizeof(TX) * (size_t)RB * (RB + 1) + 16 : 0);
}

template <class TX, class TL>
__device__ __forceinline__ TX widen(TL v)
{
    if constexpr (std::is_same<TX, TL>::value) return v;
    else return static_cast<TX>(v);
}

// INV: the diagonal step multiplies by Dinv (TX, one RB x RB column-major block per
// block row, entries (r, c) of inv(L_bb), zero outside the block) instead of
// substituting; for the repeated solves of the refinement with one factor.
// ID: forward substitution only, on the identity (generated in place of B's
// initial values): X = L^-1.  Chunk c's columns start at row c*RC, so block
// rows above that one are zero and are neither computed nor waited for.
// FO: forward substitution only, on B: X = L^-1 B (side 'L') or B L^-H (side
// 'R'); the forward half of the two-sided solve, every CTA a forward one.
template <class TL, class TX, bool UP, bool BT, bool INV = false, bool ID = false, bool FO = false>
__global__ void __launch_bounds__(NT) k_potrs_fused(const TL* __restrict__ A, long long lda, TX* B, long long ldb,
                                                    int n, int nrhs, int nchunks, int* flags, int* ticket,
                                                    int* status, const TX* __restrict__ Dinv)
{
    using T = TX;
    using R = real_t<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TL (*Lbuf)[RB][RB + 1] = reinterpret_cast<TL (*)[RB][RB + 1]>(smem_raw);
    T (*Ibuf)[RB + 1] = reinterpret_cast<T (*)[RB + 1]>(
        smem_raw + ((potrs_smem_bytes<TL, TX, false>() + 15) / 16) * 16);
    T (*Xs)[RC + 1] = reinterpret_cast<T (*)[RC + 1]>(smem_raw + sizeof(TL) * 2 * RB * (RB + 1));
    T (*Acc)[RC + 1] = Xs + RB;
    R* Rinv = reinterpret_cast<R*>(Acc + RB);
    __shared__ int s_t;
    __shared__ int s_abort;
    __shared__ int s_next;
    if (threadIdx.x == 0) { s_t = atomicAdd(ticket, 1); s_abort = 0; }
    __syncthreads();
    const int N = (int)ceil_div(n, RB);
    const int t = s_t;
    const int chunk = t % nchunks;
    const int step = t / nchunks;
    const bool fwd = ID || FO || step < N;
    const int blk = ID ? step : (fwd ? step : 2 * N - 1 - step);
    int* cflags = flags + (size_t)chunk * 2 * N;  // [0,N) forward, [N,2N) backward
    const long long r0 = (long long)chunk * RC;
    const int nr = (int)((nrhs - r0) < RC ? (nrhs - r0) : RC);
    const int jfirst = ID ? (int)(r0 / RB) : 0;  // first block row with a nonzero right-hand side
    if (ID && blk < jfirst) return;
    const long long i0 = (long long)blk * RB;
    const int nrows = (int)((n - i0) < RB ? (n - i0) : RB);
    // raw tile element (i, k): A[(i0+i) + (j0+k)*lda] when p1, A[(j0+k) + (i0+i)*lda] otherwise;
    // the operator entry is that value, conjugated when !p1 (see the four cases of the L view)
    const bool p1 = (fwd != UP);

    const int tr = threadIdx.x & (RB - 1);  // row of the block row
    const int tg = threadIdx.x >> 6;        // rhs group: columns tg, tg+4, tg+8, tg+12
    T acc[RC / 4];

    // Visit the other block rows in publication order (forward 0, 1, ..; backward N-1, N-2, ..):
    // every wait but the last one is already satisfied when reached.
    const int nvisit = ID ? blk - jfirst : (fwd ? blk : N - 1 - blk);
    auto visit = [&](int v) { return ID ? jfirst + v : (fwd ? v : N - 1 - v); };
    auto issue_tile = [&](int j, int buf) {
        const long long j0 = (long long)j * RB;
        const int ncols = (int)((n - j0) < RB ? (n - j0) : RB);
        for (int idx = threadIdx.x; idx < RB * RB; idx += NT) {
            int i, k;
            const TL* src;
            if (p1) { i = idx % RB; k = idx / RB; src = A + (i0 + i) + (j0 + k) * lda; }
            else { k = idx % RB; i = idx / RB; src = A + (j0 + k) + (i0 + i) * lda; }
            const bool valid = i < nrows && k < ncols;
            cp_async_elem<sizeof(TL)>(&Lbuf[buf][k][i], valid ? src : A, valid);
        }
    };
    // the diagonal block, raw: D[c][r] = A[(i0+r) + (i0+c)*lda] for 'L', A[(i0+c) + (i0+r)*lda] for 'U';
    // L(r, c) = D[c][r] ('L') or conj(D[c][r]) ('U') for r >= c.  Prefetched into the ring slot
    // the last off-diagonal tile leaves free, so it is resident when the solve reaches it.
    auto issue_diag = [&](int buf) {
        if constexpr (INV) {
            const T* src0 = Dinv + (long long)blk * RB * RB;
            for (int idx = threadIdx.x; idx < RB * RB; idx += NT) {
                const int r = idx % RB, c = idx / RB;
                cp_async_elem<sizeof(T)>(&Ibuf[c][r], src0 + idx, true);
            }
            return;
        }
        for (int idx = threadIdx.x; idx < RB * RB; idx += NT) {
            int r, c;
            const TL* src;
            if (!UP) { r = idx % RB; c = idx / RB; src = A + (i0 + r) + (i0 + c) * lda; }
            else { c = idx % RB; r = idx / RB; src = A + (i0 + c) + (i0 + r) * lda; }
            const bool valid = r < nrows && c < nrows;
            cp_async_elem<sizeof(TL)>(&Lbuf[buf][c][r], valid ? src : A, valid);
        }
    };
    if (nvisit > 0) issue_tile(visit(0), 0);
    else issue_diag(0);
    cp_commit();

    if (!fwd) {
        // the block row's own forward result must be published first
        if (threadIdx.x == 0) {
            if (!bounded_wait_geq(&cflags[blk], 1, status)) s_abort = 1;
            __threadfence();
        }
        __syncthreads();
        if (s_abort) { cp_wait<0>(); return; }
    }
#pragma unroll
    for (int q = 0; q < RC / 4; ++q) {
        const int r = tg + 4 * q;
        if constexpr (ID)
            acc[q] = (tr < nrows && r < nr && i0 + tr == r0 + r) ? from_real<T>(R(1)) : zero<T>();
        else
            acc[q] = (tr < nrows && r < nr) ? x_ld_cg<T, BT>(B, ldb, i0 + tr, r0 + r) : zero<T>();
    }

    // The solved block of the next visit is fetched into registers (L2 loads) while
    // the current tile is multiplied whenever its flag is already set, so only the
    // visits that really wait (the last ones) pay the load latency after the wait.
    constexpr int XE = RB * RC / NT;
    T xr[XE];
    bool pre = false;
    auto load_x = [&](int jj) {
        const long long jj0 = (long long)jj * RB;
        const int nc = (int)((n - jj0) < RB ? (n - jj0) : RB);
#pragma unroll
        for (int e = 0; e < XE; ++e) {
            const int idx = threadIdx.x + e * NT;
            const int k = idx % RB, r = idx / RB;
            xr[e] = (k < nc && r < nr) ? x_ld_cg<T, BT>(B, ldb, jj0 + k, r0 + r) : zero<T>();
        }
    };
    for (int v = 0; v < nvisit; ++v) {
        const int j = visit(v);
        if (v + 1 < nvisit) issue_tile(visit(v + 1), (v + 1) & 1);
        else issue_diag((v + 1) & 1);
        cp_commit();
        if (!pre) {
            if (threadIdx.x == 0) {
                if (!bounded_wait_geq(&cflags[fwd ? j : N + j], 1, status)) s_abort = 1;
                __threadfence();
            }
            __syncthreads();
            if (s_abort) { cp_wait<0>(); return; }
            load_x(j);
        }
#pragma unroll
        for (int e = 0; e < XE; ++e) {
            const int idx = threadIdx.x + e * NT;
            Xs[idx % RB][idx / RB] = xr[e];
        }
        if (threadIdx.x == 0) {
            bool ready = false;
            if (v + 1 < nvisit) {
                const int jn = visit(v + 1);
                ready = ld_acquire(&cflags[fwd ? jn : N + jn]) >= 1;
                if (ready) __threadfence();
            }
            s_next = ready ? 1 : 0;
        }
        cp_wait<1>();
        __syncthreads();
        pre = s_next != 0;
        if (pre) load_x(visit(v + 1));
        const TL (*Lt)[RB + 1] = Lbuf[v & 1];
        if (p1) {
#pragma unroll 8
            for (int k = 0; k < RB; ++k) {
                const T l = widen<T>(Lt[k][tr]);
#pragma unroll
                for (int q = 0; q < RC / 4; ++q) acc[q] = fms(acc[q], l, Xs[k][tg + 4 * q]);
            }
        } else {
#pragma unroll 8
            for (int k = 0; k < RB; ++k) {
                const T l = cj(widen<T>(Lt[k][tr]));
#pragma unroll
                for (int q = 0; q < RC / 4; ++q) acc[q] = fms(acc[q], l, Xs[k][tg + 4 * q]);
            }
        }
        __syncthreads();
    }
    cp_wait<0>();

    const TL (*D)[RB + 1] = Lbuf[nvisit & 1];
    // L(r, c) for r >= c, and conj(L(c, r)) for c > r, from the raw diagonal block
    auto lval = [&](int r, int c) { return UP ? cj(widen<T>(D[c][r])) : widen<T>(D[c][r]); };
    auto lcval = [&](int c, int r) { return UP ? widen<T>(D[r][c]) : cj(widen<T>(D[r][c])); };
#pragma unroll
    for (int q = 0; q < RC / 4; ++q) Acc[tr][tg + 4 * q] = acc[q];
    __syncthreads();
    if constexpr (!INV)
        for (int k = threadIdx.x; k < RB; k += NT) Rinv[k] = k < nrows ? R(1) / re(widen<T>(D[k][k])) : R(0);
    __syncthreads();
    if constexpr (INV) {
        // diagonal step as a product with the precomputed inverse block:
        // forward x = inv(L_bb) acc, backward x = inv(L_bb)^H acc
        T out[RC / 4];
#pragma unroll
        for (int q = 0; q < RC / 4; ++q) out[q] = zero<T>();
        if (fwd) {
#pragma unroll 8
            for (int k = 0; k < RB; ++k) {
                const T m = Ibuf[k][tr];
#pragma unroll
                for (int q = 0; q < RC / 4; ++q) out[q] = fma_(out[q], m, Acc[k][tg + 4 * q]);
            }
        } else {
#pragma unroll 8
            for (int k = 0; k < RB; ++k) {
                const T m = cj(Ibuf[tr][k]);
#pragma unroll
                for (int q = 0; q < RC / 4; ++q) out[q] = fma_(out[q], m, Acc[k][tg + 4 * q]);
            }
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < RC / 4; ++q) Acc[tr][tg + 4 * q] = out[q];
    } else {
        // warp w solves right-hand sides 2w and 2w+1 together; lanes own rows lane and lane+32
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int ra = 2 * warp, rb = 2 * warp + 1;
        T a0 = Acc[lane][ra], a1 = Acc[lane + 32][ra];
        T b0 = Acc[lane][rb], b1 = Acc[lane + 32][rb];
        if (fwd) {
            for (int k = 0; k < nrows; ++k) {
                const R rk = Rinv[k];
                if (k < 32) {
                    if (lane == k) { a0 = scal(a0, rk); b0 = scal(b0, rk); }
                    const T xa = shfl_t(a0, k), xb = shfl_t(b0, k);
                    const T l0 = lval(lane, k), l1 = lval(lane + 32, k);
                    if (lane > k) { a0 = fms(a0, l0, xa); b0 = fms(b0, l0, xb); }
                    a1 = fms(a1, l1, xa);
                    b1 = fms(b1, l1, xb);
                } else {
                    if (lane == k - 32) { a1 = scal(a1, rk); b1 = scal(b1, rk); }
                    const T xa = shfl_t(a1, k - 32), xb = shfl_t(b1, k - 32);
                    if (lane + 32 > k) {
                        const T l1 = lval(lane + 32, k);
                        a1 = fms(a1, l1, xa);
                        b1 = fms(b1, l1, xb);
                    }
                }
            }
        } else {
            // x_k = v_k / L_kk; v_i -= conj(L(k, i)) x_k for i < k
            for (int k = nrows - 1; k >= 0; --k) {
                const R rk = Rinv[k];
                if (k < 32) {
                    if (lane == k) { a0 = scal(a0, rk); b0 = scal(b0, rk); }
                    const T xa = shfl_t(a0, k), xb = shfl_t(b0, k);
                    if (lane < k) {
                        const T l0 = lcval(k, lane);
                        a0 = fms(a0, l0, xa);
                        b0 = fms(b0, l0, xb);
                    }
                } else {
                    if (lane == k - 32) { a1 = scal(a1, rk); b1 = scal(b1, rk); }
                    const T xa = shfl_t(a1, k - 32), xb = shfl_t(b1, k - 32);
                    const T l0 = lcval(k, lane);
                    a0 = fms(a0, l0, xa);
                    b0 = fms(b0, l0, xb);
                    if (lane + 32 < k) {
                        const T l1 = lcval(k, lane + 32);
                        a1 = fms(a1, l1, xa);
                        b1 = fms(b1, l1, xb);
                    }
                }
            }
        }
        Acc[lane][ra] = a0;
        Acc[lane + 32][ra] = a1;
        Acc[lane][rb] = b0;
        Acc[lane + 32][rb] = b1;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < RB * RC; idx += NT) {
        const int i = idx % RB, r = idx / RB;
        if (i < nrows && r < nr) x_st<T, BT>(B, ldb, i0 + i, r0 + r, Acc[i][r]);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) st_release(&cflags[fwd ? blk : N + blk], 1);
}

template <class T, bool UP, bool BT, class TL = T, bool INV = false, bool ID = false, bool FO = false>
cudaError_t potrs_launch(const TL* A, long long lda, T* B, long long ldb, int n, int nrhs, int* flags, int* ticket,
                         int* status, cudaStream_t st, const T* Dinv = nullptr)
{
    const int N = (int)ceil_div(n, RB);
    const int nchunks = (int)ceil_div(nrhs, RC);
    const long long grid = (ID || FO ? 1LL : 2LL) * N * nchunks;
    const size_t smem = potrs_smem_bytes<TL, T, INV>();
    if (cudaError_t e = smem_optin(k_potrs_fused<TL, T, UP, BT, INV, ID, FO>, smem); e != cudaSuccess) return e;
    const double cf = Traits<T>::cplx ? 4.0 : 1.0;
    const double nd = n, rd = nrhs;
    ProfScope ps(PK_POTRS_FUSED, st,
                 ID ? cf * nd * nd * nd / 3.0 : (FO ? cf * nd * nd * rd : cf * 2.0 * nd * nd * rd),
                 sizeof(TL) * nd * (nd + 1) + sizeof(T) * 4.0 * nd * rd);
    k_potrs_fused<TL, T, UP, BT, INV, ID, FO><<<(unsigned)grid, NT, smem, st>>>(A, lda, B, ldb, n, nrhs, nchunks,
                                                                                 flags, ticket, status, Dinv);
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

template <class T>
cudaError_t forward_typed(char uplo, char side, int n, int nrhs, const void* A, long long lda, void* B,
                          long long ldb, int* flags, int* ticket, int* status, cudaStream_t st)
{
    const T* a = static_cast<const T*>(A);
    T* b = static_cast<T*>(B);
    const bool up = uplo == 'U', bt = side == 'R';
    if (up && bt)
        return potrs_launch<T, true, true, T, false, false, true>(a, lda, b, ldb, n, nrhs, flags, ticket, status, st);
    if (up)
        return potrs_launch<T, true, false, T, false, false, true>(a, lda, b, ldb, n, nrhs, flags, ticket, status, st);
    if (bt)
        return potrs_launch<T, false, true, T, false, false, true>(a, lda, b, ldb, n, nrhs, flags, ticket, status, st);
    return potrs_launch<T, false, false, T, false, false, true>(a, lda, b, ldb, n, nrhs, flags, ticket, status, st);
}

cudaError_t potrs_dispatch(char type, char uplo, char side, int n, int nrhs, const void* A, long long lda, void* B,
                           long long ldb, int* flags, int* ticket, int* status, cudaStream_t st)
{
    switch (type) {
    case 's': return potrs_typed<float>(uplo, side, n, nrhs, A, lda, B, ldb, flags, ticket, status, st);
    case 'd': return potrs_typed<double>(uplo, side, n, nrhs, A, lda, B, ldb, flags, ticket, status, st);
    case 'c': return potrs_typed<cf32>(uplo, side, n, nrhs, A, lda, B, ldb, flags, ticket, status, st);
    case 'z': return potrs_typed<cf64>(uplo, side, n, nrhs, A, lda, B, ldb, flags, ticket, status, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace
}  // namespace ddlak

// ---------------------------------------------------------------------------
// inverses of the RB x RB diagonal blocks of an FP32 factor, in FP64: one CTA
// per block, the block widened into shared memory, one thread per column of
// the inverse (forward substitution against the identity).
// ---------------------------------------------------------------------------
namespace ddlak {
namespace {
__global__ void __launch_bounds__(128) k_inv_diag_blocks(const float* __restrict__ L, long long ldl, int n,
                                                         double* __restrict__ Dinv)
{
    __shared__ double Ls[RB][RB + 1];  // Ls[c][r] = L(r, c)
    const int blk = blockIdx.x;
    const long long i0 = (long long)blk * RB;
    const int nb = (int)((n - i0) < RB ? (n - i0) : RB);
    for (int idx = threadIdx.x; idx < RB * RB; idx += blockDim.x) {
        const int r = idx % RB, c = idx / RB;
        Ls[c][r] = (r < nb && c < nb && r >= c) ? (double)L[(i0 + r) + (i0 + c) * ldl] : 0.0;
    }
    __syncthreads();
    double* out = Dinv + (long long)blk * RB * RB;
    const int c = threadIdx.x;
    if (c < RB) {
        double y[RB];
#pragma unroll
        for (int r = 0; r < RB; ++r) y[r] = 0.0;
        if (c < nb) {
#pragma unroll
            for (int r = 0; r < RB; ++r) {
                if (r >= c && r < nb) {
                    double s = r == c ? 1.0 : 0.0;
#pragma unroll
                    for (int k = 0; k < RB; ++k)
                        if (k >= c && k < r) s = fma(-Ls[k][r], y[k], s);
                    y[r] = s / Ls[r][r];
                }
            }
        }
#pragma unroll
        for (int r = 0; r < RB; ++r) out[(long long)c * RB + r] = y[r];
    }
}
}  // namespace
}  // namespace ddlak

extern "C" unsigned long long ddlak_inv_diag_bytes(int n)
{
    return n > 0 ? (unsigned long long)ddlak::ceil_div(n, ddlak::RB) * ddlak::RB * ddlak::RB * sizeof(double) : 0;
}

extern "C" int ddlak_inv_diag_blocks(int n, const void* L32, long long ldl, void* Dinv, void* stream)
{
    using namespace ddlak;
    if (n <= 0) return 0;
    const int N = (int)ceil_div(n, RB);
    {
        ProfScope ps(PK_MIXED_OTHER, static_cast<cudaStream_t>(stream), (double)N * RB * RB * RB / 3.0,
                     (double)N * RB * RB * 12.0);
        k_inv_diag_blocks<<<N, 128, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const float*>(L32), ldl, n,
                                                                           static_cast<double*>(Dinv));
    }
    note_launches(1);
    return (int)cudaGetLastError();
}

// Solve with an FP32 factor (uplo 'L') and FP64 right-hand sides in place
// (the refinement solves of the mixed-precision path); same scratch as
// ddlak_potrs.  With Dinv (from ddlak_inv_diag_blocks) the diagonal steps are
// products with the precomputed inverse blocks instead of substitutions.
extern "C" int ddlak_potrs_mixed(int n, int nrhs, const void* L32, long long ldl, const void* Dinv, void* B,
                                 long long ldb, void* work, unsigned long long work_bytes, void* stream)
{
    using namespace ddlak;
    if (n <= 0 || nrhs <= 0) return 0;
    if (work_bytes < ddlak_potrs_workspace(n, nrhs)) return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(work, 0, ddlak_potrs_workspace(n, nrhs), st);
    if (e != cudaSuccess) return (int)e;
    int* status = static_cast<int*>(work);
    int* flags = reinterpret_cast<int*>(static_cast<char*>(work) + 256);
    if (Dinv)
        return (int)potrs_launch<double, false, false, float, true>(static_cast<const float*>(L32), ldl,
                                                                    static_cast<double*>(B), ldb, n, nrhs, flags,
                                                                    status + 1, status, st,
                                                                    static_cast<const double*>(Dinv));
    return (int)potrs_launch<double, false, false, float>(static_cast<const float*>(L32), ldl,
                                                          static_cast<double*>(B), ldb, n, nrhs, flags, status + 1,
                                                          status, st);
}

// Scratch: [status int][ticket int] padded to 256 B, then nchunks * 2N flags.
extern "C" unsigned long long ddlak_potrs_workspace(int n, int nrhs)
{
    if (n <= 0 || nrhs <= 0) return 0;
    const unsigned long long N = (unsigned long long)ddlak::ceil_div(n, ddlak::RB);
    const unsigned long long C = (unsigned long long)ddlak::ceil_div(nrhs, ddlak::RC);
    return 256 + ((C * 2 * N * sizeof(int) + 255) / 256) * 256;
}

// ---------------------------------------------------------------------------
// The same fused solve with its scratch in a fixed, library-owned device array
// instead of memory the caller or the allocator provides.  The array lives
// for the whole process on every device that loads the library (128 KB + 256 B),
// which bounds the problem: n <= 65536 (1024 block rows of 64) and nrhs <= 256
// (16 chunks of 16).  All calls share it, so calls that overlap on the GPU
// race on it; the words that must start at zero are cleared on the caller's
// stream before each launch.
// ---------------------------------------------------------------------------
namespace ddlak {
namespace {
constexpr int kFixedMaxN = 65536;
constexpr int kFixedMaxRhs = 256;
constexpr int kFixedHeaderInts = 64;  // status, ticket, padding to 256 bytes
constexpr int kFixedFlagInts = 2 * (kFixedMaxN / RB) * (kFixedMaxRhs / RC);
__device__ __align__(256) int g_potrs_fixed_scratch[kFixedHeaderInts + kFixedFlagInts];

// Device address of the array on the current device; looked up once per
// device (the first call on a device does the lookup, with that device current)
// and kept for the process's life, which assumes the device's primary context
// is never reset (cudaDeviceReset) while the library is in use.
int* fixed_scratch_ptr(int* err)
{
    static std::mutex mu;
    static int* ptrs[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) {
        *err = e != cudaSuccess ? (int)e : (int)cudaErrorInvalidDevice;
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(mu);
    if (ptrs[dev] == nullptr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_potrs_fixed_scratch);
        if (e != cudaSuccess) {
            *err = (int)e;
            return nullptr;
        }
        ptrs[dev] = static_cast<int*>(p);
    }
    *err = 0;
    return ptrs[dev];
}
}  // namespace
}  // namespace ddlak

extern "C" int ddlak_potrs_fixed_scratch_limits(int* max_n, int* max_nrhs)
{
    if (max_n) *max_n = ddlak::kFixedMaxN;
    if (max_nrhs) *max_nrhs = ddlak::kFixedMaxRhs;
    return 0;
}

extern "C" int ddlak_potrs_fixed_scratch(char type, char uplo, char side, int n, int nrhs, const void* A,
                                         long long lda, void* B, long long ldb, int** status_word, void* stream)
{
    using namespace ddlak;
    if (n <= 0 || nrhs <= 0) return 0;
    if (n > kFixedMaxN || nrhs > kFixedMaxRhs) return (int)cudaErrorInvalidValue;
    int err = 0;
    int* base = fixed_scratch_ptr(&err);
    if (base == nullptr) return err;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t flag_ints = (size_t)2 * ceil_div(n, RB) * ceil_div(nrhs, RC);
    cudaError_t e = cudaMemsetAsync(base, 0, (kFixedHeaderInts + flag_ints) * sizeof(int), st);
    if (e != cudaSuccess) return (int)e;
    if (status_word) *status_word = base;
    return (int)potrs_dispatch(type, uplo, side, n, nrhs, A, lda, B, ldb, base + kFixedHeaderInts, base + 1, base,
                               st);
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
    return (int)potrs_dispatch(type, uplo, side, n, nrhs, A, lda, B, ldb, flags, ticket, status, st);
}

// X = L^-1 B (side 'L', B n x nrhs) or X = B L^-H (side 'R', B nrhs x n), in place,
// with the factor read through its L view (uplo 'L': A's lower triangle; 'U': L = U^H):
// the forward half of ddlak_potrs.  Same scratch (ddlak_potrs_workspace(n, nrhs)) and
// status word.
extern "C" int ddlak_forward_solve(char type, char uplo, char side, int n, int nrhs, const void* A, long long lda,
                                   void* B, long long ldb, void* work, unsigned long long work_bytes, void* stream)
{
    using namespace ddlak;
    if (n <= 0 || nrhs <= 0) return 0;
    if (!A || !B || work_bytes < ddlak_potrs_workspace(n, nrhs)) return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(work, 0, ddlak_potrs_workspace(n, nrhs), st);
    if (e != cudaSuccess) return (int)e;
    int* status = static_cast<int*>(work);
    int* ticket = status + 1;
    int* flags = reinterpret_cast<int*>(static_cast<char*>(work) + 256);
    switch (type) {
    case 's': return (int)forward_typed<float>(uplo, side, n, nrhs, A, lda, B, ldb, flags, ticket, status, st);
    case 'd': return (int)forward_typed<double>(uplo, side, n, nrhs, A, lda, B, ldb, flags, ticket, status, st);
    case 'c': return (int)forward_typed<cf32>(uplo, side, n, nrhs, A, lda, B, ldb, flags, ticket, status, st);
    case 'z': return (int)forward_typed<cf64>(uplo, side, n, nrhs, A, lda, B, ldb, flags, ticket, status, st);
    default: return (int)cudaErrorInvalidValue;
    }
}

// W = L^-1 for a lower factor: the fused forward substitution on the identity.
extern "C" int ddlak_trtri_blocked(char type, int n, const void* L, long long ldl, void* W, long long ldw, void* work,
                                   unsigned long long work_bytes, void* stream)
{
    using namespace ddlak;
    if (n <= 0) return 0;
    if (!L || !W || ldl < n || ldw < n || work_bytes < ddlak_potrs_workspace(n, n)) return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(work, 0, ddlak_potrs_workspace(n, n), st);
    if (e != cudaSuccess) return (int)e;
    int* status = static_cast<int*>(work);
    int* ticket = status + 1;
    int* flags = reinterpret_cast<int*>(static_cast<char*>(work) + 256);
    if (type == 'd')
        return (int)potrs_launch<double, false, false, double, false, true>(
            static_cast<const double*>(L), ldl, static_cast<double*>(W), ldw, n, n, flags, ticket, status, st);
    if (type == 's')
        return (int)potrs_launch<float, false, false, float, false, true>(
            static_cast<const float*>(L), ldl, static_cast<float*>(W), ldw, n, n, flags, ticket, status, st);
    return (int)cudaErrorInvalidValue;
}
