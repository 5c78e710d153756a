// In-shared-memory Cholesky of one diagonal block (lower triangle of
// s[i + j*ld], i, j < nbk <= 128; nbk <= 64 for complex double), shared by the
// plain and mixed factorizations.
//
// Blocked by 32-column panels, so the CTA synchronises three times per panel
// instead of once per column.  Panel c0..c0+31:
//   (A) warp 0 factors the 32 x 32 diagonal block in registers (lane i holds
//       row i).  Step j publishes column j in a double-buffered shared vector
//       (one __syncwarp), every lane applies a_ik -= a_ij conj(a_kj) / d_j to
//       its row, and the owner of the next pivot computes 1/d_(j+1) inside the
//       step, so a step's critical path is one multiply, one multiply-add and
//       the shared round trip.  The square roots are deferred: column j is
//       scaled by 1/sqrt(d_j) once the panel is done.
//   (B) one thread per row below the panel solves x L11^H = a (forward
//       substitution with the final L11 and its reciprocal pivots from shared
//       memory).
//   (C) the trailing lower triangle is updated by the panel: 256 threads in a
//       16 x 16 grid, thread (tx, ty) owning rows tx + 16p and columns
//       ty + 16q (q <= p), so the shared reads are conflict-free or broadcast.
// Returns 0, or 1 + the index of the first column whose pivot is not positive
// (or NaN).  As in LAPACK ?potf2, the columns before it are final (in every
// row of the block) and the failed pivot keeps its value.
// Must be called by all 256 threads of the CTA.
#pragma once
#include <type_traits>
#include "common.cuh"

namespace ddlak {

template <class T>
__device__ __forceinline__ T shfl(T v, int src)
{
    if constexpr (Traits<T>::cplx) {
        v.x = __shfl_sync(0xffffffffu, v.x, src);
        v.y = __shfl_sync(0xffffffffu, v.y, src);
        return v;
    } else {
        return __shfl_sync(0xffffffffu, v, src);
    }
}

namespace diagf {

// 1/d for the pivots on the column chain: the hardware's approximate reciprocal
// (rcp.approx.ftz.f64, about single precision) refined by two Newton-Raphson
// steps r <- r + r (1 - d r), each of which squares the relative error, so the
// result is within an ulp or two of 1/d for the positive normal pivots this is
// used on (a non-positive pivot stops the factorization before its reciprocal
// is used).  Cheaper on the chain than the correctly rounded division.
__device__ __forceinline__ double recip_pivot(double d)
{
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
    double e = fma(-d, r, 1.0);
    r = fma(r, e, r);
    e = fma(-d, r, 1.0);
    return fma(r, e, r);
}
__device__ __forceinline__ float recip_pivot(float d) { return 1.0f / d; }

constexpr int PW = 32;    // panel width
constexpr int MAXN = 128;  // largest block
constexpr int UP = (MAXN - PW) / 16;  // row groups of the trailing update (6)

// (A) warp 0: the w x w diagonal block at (c0, c0).  On exit the block's
// columns before the first failed one hold L, s_rs[c0 + j] = 1 / l_jj for
// them, and a failure is recorded as *s_fail = c0 + j + 1.
template <class T, int WC = 0>  // WC: the width when known at compile time (a full panel), else 0
__device__ __forceinline__ void panel_diag(T* s, int ld, int c0, int w_rt, int lane, T (*colbuf)[PW],
                                           real_t<T>* s_inv, real_t<T>* s_rs, int* s_fail)
{
    using R = real_t<T>;
    const int w = WC ? WC : w_rt;
    const int i = lane;
    T a[PW];
#pragma unroll
    for (int k = 0; k < PW; ++k) a[k] = (i < w && k <= i) ? s[(c0 + i) + (c0 + k) * ld] : zero<T>();
    // column 0 and its pivot's reciprocal
    colbuf[0][i] = a[0];
    if (i == 0) s_inv[0] = recip_pivot(re(a[0]));
    __syncwarp();
    int fail = 0;
    R dpiv = R(0);
#pragma unroll
    for (int j = 0; j < PW; ++j) {
        if (j < w && !fail) {
            const T* cv = colbuf[j & 1];
            const R d = re(cv[j]);
            if (!(d > R(0))) {
                fail = j + 1;
            } else {
                if (i == j) dpiv = d;
                const R invd = s_inv[j & 1];
                const T tj = scal(a[j], invd);  // a_ij / d_j (upper-triangle garbage for i < j, never stored)
                if (j + 1 < PW) {
                    // the next column first, so its publication overlaps the rest of the step
                    a[j + 1] = fms(a[j + 1], tj, cj(cv[j + 1]));
                    colbuf[(j + 1) & 1][i] = a[j + 1];
                    // every lane takes its own reciprocal (no divergent branch on the chain);
                    // lane j + 1's is the next pivot's
                    const R rn = recip_pivot(re(a[j + 1]));
                    if (i == j + 1) s_inv[(j + 1) & 1] = rn;
#pragma unroll
                    for (int k = j + 2; k < PW; ++k) a[k] = fms(a[k], tj, cj(cv[k]));
                }
            }
            __syncwarp();
        }
    }
    // deferred scaling: l_kk = sqrt(d_k), l_ik = a_ik / sqrt(d_k)
    const int done = fail ? fail - 1 : w;
    R rs = R(0), sk = R(0);
    if (i < done) {
        sk = sqrt(dpiv);
        rs = R(1) / sk;
        s_rs[c0 + i] = rs;
    }
#pragma unroll
    for (int k = 0; k < PW; ++k) {
        const R rk = shfl(rs, k);
        if (k < done) {
            if (i == k) a[k] = from_real<T>(sk);
            else if (i > k) a[k] = scal(a[k], rk);
        }
    }
#pragma unroll
    for (int k = 0; k < PW; ++k)
        if (i < w && k <= i) s[(c0 + i) + (c0 + k) * ld] = a[k];
    if (fail && lane == 0) *s_fail = c0 + fail;
}

// (B) row r below the panel: x L11^H = a over the panel's first jd columns.
template <class T>
__device__ __forceinline__ void panel_row(T* s, int ld, int c0, int r, int jd, const real_t<T>* s_rs)
{
    T x[PW];
#pragma unroll
    for (int k = 0; k < PW; ++k) x[k] = k < jd ? s[r + (c0 + k) * ld] : zero<T>();
#pragma unroll
    for (int j = 0; j < PW; ++j) {
        if (j < jd) {
            x[j] = scal(x[j], s_rs[c0 + j]);
#pragma unroll
            for (int k = j + 1; k < PW; ++k) x[k] = fms(x[k], x[j], cj(s[(c0 + k) + (c0 + j) * ld]));
        }
    }
#pragma unroll
    for (int k = 0; k < PW; ++k)
        if (k < jd) s[r + (c0 + k) * ld] = x[k];
}

// (C) s[i, k] -= sum_j L[i, c0 + j] conj(L[k, c0 + j]) for c1 <= k <= i < nbk.
template <class T>
__device__ __forceinline__ void trailing(T* s, int ld, int c0, int c1, int nbk, int t)
{
    const int tx = t & 15, ty = t >> 4;
    const int m2 = nbk - c1;
    T acc[UP][UP];
#pragma unroll
    for (int p = 0; p < UP; ++p)
#pragma unroll
        for (int q = 0; q <= p; ++q) acc[p][q] = zero<T>();
#pragma unroll 4
    for (int j = 0; j < PW; ++j) {
        const T* col = s + (c0 + j) * ld + c1;
        T li[UP], lk[UP];
#pragma unroll
        for (int p = 0; p < UP; ++p) {
            li[p] = (16 * p < m2 && tx + 16 * p < m2) ? col[tx + 16 * p] : zero<T>();
            lk[p] = (16 * p < m2 && ty + 16 * p < m2) ? cj(col[ty + 16 * p]) : zero<T>();
        }
#pragma unroll
        for (int p = 0; p < UP; ++p)
            if (16 * p < m2)
#pragma unroll
                for (int q = 0; q <= p; ++q) acc[p][q] = fma_(acc[p][q], li[p], lk[q]);
    }
#pragma unroll
    for (int p = 0; p < UP; ++p)
#pragma unroll
        for (int q = 0; q <= p; ++q) {
            const int i = tx + 16 * p, k = ty + 16 * q;
            if (i < m2 && k <= i) {
                T* e = s + (c1 + i) + (long long)(c1 + k) * ld;
                *e = sub(*e, acc[p][q]);
            }
        }
}

// (C) for double on the FP64 tensor cores: the trailing lower triangle in 16 x 8
// tiles (mma.sync m16n8k4 f64), tile (I, K) covering rows c1 + 16 I .. + 15 and
// columns c1 + 8 K .. + 7.  The tiles of row blocks I0 <= I < I1, counted row by
// row, go to the workers (warps) round-robin.  Lane (g, q) feeds L(row g / g + 8,
// c0 + kk + q) and L(col g, c0 + kk + q) and receives the products for rows g
// and g + 8, columns 2q and 2q + 1.  Only k <= i is written.  With ld = 4 mod 16
// (doubles) the 16 lanes of a half-warp read 16 distinct banks.
__device__ __forceinline__ void mma16x8x4(double (&u)[2], double (&v)[2], double a_up, double a_lo, double b)
{
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
                 : "+d"(u[0]), "+d"(u[1]), "+d"(v[0]), "+d"(v[1])
                 : "d"(a_up), "d"(a_lo), "d"(b));
}

__device__ __forceinline__ void trailing_dmma(double* s, int ld, int c0, int c1, int nbk, int I0, int I1, int worker,
                                              int nworkers, int lane)
{
    const int g = lane >> 2, q = lane & 3;
    const int m2 = nbk - c1;
    const int ti = min((m2 + 15) / 16, I1);
    const int tk_all = (m2 + 7) / 8;
    int idx = 0;
    for (int I = I0; I < ti; ++I) {
        const int nk = min(2 * I + 2, tk_all);  // row block I holds column tiles 0 .. nk - 1
        for (int K = 0; K < nk; ++K, ++idx) {
            if (idx % nworkers != worker) continue;
            const int r_up = 16 * I + g, r_lo = r_up + 8, col = 8 * K + g;
            double u[2] = {0.0, 0.0}, v[2] = {0.0, 0.0};
#pragma unroll
            for (int kk = 0; kk < PW; kk += 4) {
                const double* cj0 = s + (c0 + kk + q) * ld + c1;
                const double a_up = r_up < m2 ? cj0[r_up] : 0.0;
                const double a_lo = r_lo < m2 ? cj0[r_lo] : 0.0;
                const double b = col < m2 ? cj0[col] : 0.0;
                mma16x8x4(u, v, a_up, a_lo, b);
            }
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int k = 8 * K + 2 * q + e;
                if (r_up < m2 && k <= r_up) s[(c1 + r_up) + (c1 + k) * ld] -= u[e];
                if (r_lo < m2 && k <= r_lo) s[(c1 + r_lo) + (c1 + k) * ld] -= v[e];
            }
        }
    }
}

// (B) for double: as panel_row, with the columns of L11 read two at a time
// (16-byte shared loads; ld and c0 even).  Same operations in the same order.
template <int JC = 0>  // JC: the number of final columns when known at compile time, else 0
__device__ __forceinline__ void panel_row_f64(double* s, int ld, int c0, int r, int jd_rt, const double* s_rs)
{
    const int jd = JC ? JC : jd_rt;
    double x[PW];
#pragma unroll
    for (int k = 0; k < PW; ++k) x[k] = k < jd ? s[r + (c0 + k) * ld] : 0.0;
#pragma unroll
    for (int j = 0; j < PW; ++j) {
        if (j < jd) {
            x[j] = x[j] * s_rs[c0 + j];
            const double* lj = s + c0 + (c0 + j) * ld;
#pragma unroll
            for (int m = (j + 1) >> 1; m < PW / 2; ++m) {
                const double2 v = *reinterpret_cast<const double2*>(lj + 2 * m);
                if (2 * m > j) x[2 * m] = fma(-x[j], v.x, x[2 * m]);
                x[2 * m + 1] = fma(-x[j], v.y, x[2 * m + 1]);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < PW; ++k)
        if (k < jd) s[r + (c0 + k) * ld] = x[k];
}

}  // namespace diagf

// Leading dimension of the shared block: for double 4 mod 16 (and even), which
// makes the DMMA fragment loads conflict-free and allows the 16-byte loads of
// panel_row_f64; nbk + 1 for the other types.
template <class T>
__host__ __device__ constexpr int diag_block_ld(int nbk)
{
    return std::is_same<T, double>::value ? ((nbk + 15) / 16) * 16 + 4 : nbk + 1;
}

// double: the next panel's column chain overlaps the current trailing update.
// After the rows of panel c0 are solved, warps 0 and 1 update the next 32 x 32
// diagonal block (the two row blocks of tiles at the top of the trailing
// triangle) and warp 0 goes straight on to its chain (A), while warps 1..7
// update the rows below it.  One CTA barrier per panel fewer, and the chain no
// longer waits for the whole trailing update.  Every entry receives the same
// operations as in the unpipelined order, so the factor is unchanged.  Full
// panels take the compile-time-width forms of the chain and the row solve.
// The partial-panel forms (a block whose order is not a multiple of 32: only the last
// block of a factorization) out of line, so that the full-panel code the kernel runs
// for every other block stays compact in the instruction cache.
static __device__ __noinline__ void panel_diag_f64_partial(double* s, int ld, int c0, int w, int lane,
                                                    double (*colbuf)[diagf::PW], double* s_inv, double* s_rs,
                                                    int* s_fail)
{
    diagf::panel_diag<double>(s, ld, c0, w, lane, colbuf, s_inv, s_rs, s_fail);
}
static __device__ __noinline__ void panel_row_f64_partial(double* s, int ld, int c0, int r, int jd, const double* s_rs)
{
    diagf::panel_row_f64(s, ld, c0, r, jd, s_rs);
}

__device__ __forceinline__ int factor_block_smem_f64(double* s, int ld, int nbk)
{
    using namespace diagf;
    __shared__ __align__(16) double colbuf[2][PW];
    __shared__ double s_inv[2];
    __shared__ double s_rs[MAXN];
    __shared__ int s_fail;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    if (t == 0) s_fail = 0;
    __syncthreads();
    auto chain = [&](int c, int w) {  // warp 0
        if (w == PW) panel_diag<double, PW>(s, ld, c, PW, lane, colbuf, s_inv, s_rs, &s_fail);
        else panel_diag_f64_partial(s, ld, c, w, lane, colbuf, s_inv, s_rs, &s_fail);
    };
    if (warp == 0) chain(0, nbk < PW ? nbk : PW);
    __syncthreads();
    for (int c0 = 0; c0 < nbk; c0 += PW) {
        const int w = nbk - c0 < PW ? nbk - c0 : PW;
        const int c1 = c0 + w;
        const int fail = s_fail;
        const int jd = fail ? fail - 1 - c0 : w;  // final columns of this panel
        if (jd == PW) {
            for (int r = c1 + t; r < nbk; r += blockDim.x) panel_row_f64<PW>(s, ld, c0, r, PW, s_rs);
        } else {
            for (int r = c1 + t; r < nbk; r += blockDim.x) panel_row_f64_partial(s, ld, c0, r, jd, s_rs);
        }
        __syncthreads();
        if (fail || c1 >= nbk) break;
        // warps 0 and 1 update the next diagonal block (the two top row blocks of
        // tiles); warp 1 then joins warps 2..7 on the rows below while warp 0,
        // once warp 1's tiles are in (named barrier 1), runs the next chain
        if (warp < 2) trailing_dmma(s, ld, c0, c1, nbk, 0, 2, warp, 2, lane);
        if (warp == 0) {
            asm volatile("bar.sync 1, 64;" ::: "memory");
            chain(c1, nbk - c1 < PW ? nbk - c1 : PW);
        } else {
            if (warp == 1) asm volatile("bar.arrive 1, 64;" ::: "memory");
            trailing_dmma(s, ld, c0, c1, nbk, 2, MAXN / 16, warp - 1, 7, lane);
        }
        __syncthreads();
    }
    return s_fail;
}

template <class T>
__device__ int factor_block_smem(T* s, int ld, int nbk)
{
    if constexpr (std::is_same<T, double>::value) {
        return factor_block_smem_f64(s, ld, nbk);
    } else {
        using R = real_t<T>;
        using namespace diagf;
        __shared__ T colbuf[2][PW];
        __shared__ R s_inv[2];
        __shared__ R s_rs[MAXN];
        __shared__ int s_fail;
        const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
        if (t == 0) s_fail = 0;
        __syncthreads();
        for (int c0 = 0; c0 < nbk; c0 += PW) {
            const int w = nbk - c0 < PW ? nbk - c0 : PW;
            const int c1 = c0 + w;
            if (warp == 0) panel_diag<T>(s, ld, c0, w, lane, colbuf, s_inv, s_rs, &s_fail);
            __syncthreads();
            const int fail = s_fail;
            const int jd = fail ? fail - 1 - c0 : w;  // final columns of this panel
            for (int r = c1 + t; r < nbk; r += blockDim.x) panel_row<T>(s, ld, c0, r, jd, s_rs);
            __syncthreads();
            if (fail) break;
            if (c1 < nbk) {
                trailing<T>(s, ld, c0, c1, nbk, t);
                __syncthreads();
            }
        }
        return s_fail;
    }
}

}  // namespace ddlak
