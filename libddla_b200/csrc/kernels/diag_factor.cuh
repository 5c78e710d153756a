// In-shared-memory Cholesky of one diagonal block (lower triangle of
// s[i + j*ld], i, j < nbk <= 128), shared by the plain and mixed factorizations.
//
// The block is factored in 32-wide steps: warp 0 factors each 32 x 32
// diagonal sub-block with the rows held in registers (pivot and column values
// broadcast with warp shuffles, no CTA barrier per column), one thread per row
// then solves the rows below against it with reciprocal pivots, and the whole
// CTA applies the rank-32 update to the rest of the block in 4x4 micro-tiles.
// Returns 0, or 1 + the index of the first column whose pivot is not positive
// (or NaN); that pivot keeps its failed value, as LAPACK ?potf2 leaves it.
// Must be called by all threads of the CTA (blockDim.x a multiple of 32).
#pragma once
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

template <class T>
__device__ int factor_block_smem(T* s, int ld, int nbk)
{
    using R = real_t<T>;
    __shared__ int s_fail;
    __shared__ R s_rinv[32];
    if (threadIdx.x == 0) s_fail = 0;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int jb = 0; jb < nbk; jb += 32) {
        const int w = nbk - jb < 32 ? nbk - jb : 32;
        // (a) 32 x 32 diagonal sub-block: lane r holds row r in registers
        if (warp == 0) {
            T a[32];
#pragma unroll
            for (int c = 0; c < 32; ++c) a[c] = (lane < w && c <= lane) ? s[(jb + lane) + (jb + c) * ld] : zero<T>();
            int fail = 0;
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                if (j < w && !fail) {
                    const R d = re(shfl(a[j], j));
                    if (!(d > R(0))) {
                        fail = j + 1;  // lane j keeps the failed value in a[j]
                    } else {
                        const R l = sqrt(d);
                        const R inv = R(1) / l;
                        if (lane == j) a[j] = from_real<T>(l);
                        if (lane > j) a[j] = scal(a[j], inv);
                        if (lane == 0) s_rinv[j] = inv;
#pragma unroll
                        for (int c = j + 1; c < 32; ++c) {
                            const T lcj = shfl(a[j], c);
                            if (lane >= c) a[c] = fmsc(a[c], a[j], lcj);
                        }
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < 32; ++c)
                if (lane < w && c <= lane) s[(jb + lane) + (jb + c) * ld] = a[c];
            if (fail && lane == 0) s_fail = jb + fail;
        }
        __syncthreads();
        if (s_fail) break;
        const int r0 = jb + w;
        const int m2 = nbk - r0;
        if (m2 <= 0) break;
        // (b) rows below: x * Ldd^H = a, a thread per row
        for (int row = r0 + threadIdx.x; row < nbk; row += blockDim.x) {
            T x[32];
#pragma unroll
            for (int c = 0; c < 32; ++c) x[c] = c < w ? s[row + (jb + c) * ld] : zero<T>();
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                if (j < w) {
                    x[j] = scal(x[j], s_rinv[j]);
#pragma unroll
                    for (int c = j + 1; c < 32; ++c)
                        if (c < w) x[c] = fmsc(x[c], x[j], s[(jb + c) + (jb + j) * ld]);
                }
            }
#pragma unroll
            for (int c = 0; c < 32; ++c)
                if (c < w) s[row + (jb + c) * ld] = x[c];
        }
        __syncthreads();
        // (c) trailing update of the block: 4x4 micro-tiles over the lower triangle
        const int t2 = (m2 + 3) >> 2;
        const int ntiles = t2 * (t2 + 1) / 2;
        for (int mt = threadIdx.x; mt < ntiles; mt += blockDim.x) {
            int I = (int)((sqrtf(8.f * mt + 1.f) - 1.f) * 0.5f);
            while ((I + 1) * (I + 2) / 2 <= mt) ++I;
            while (I * (I + 1) / 2 > mt) --I;
            const int J = mt - I * (I + 1) / 2;
            const int i0 = r0 + 4 * I, k0l = r0 + 4 * J;
            T acc[4][4];
#pragma unroll
            for (int p = 0; p < 4; ++p)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[p][q] = zero<T>();
            for (int c = 0; c < w; ++c) {
                T u[4], v[4];
#pragma unroll
                for (int p = 0; p < 4; ++p) u[p] = i0 + p < nbk ? s[(i0 + p) + (jb + c) * ld] : zero<T>();
#pragma unroll
                for (int q = 0; q < 4; ++q) v[q] = k0l + q < nbk ? cj(s[(k0l + q) + (jb + c) * ld]) : zero<T>();
#pragma unroll
                for (int p = 0; p < 4; ++p)
#pragma unroll
                    for (int q = 0; q < 4; ++q) acc[p][q] = fma_(acc[p][q], u[p], v[q]);
            }
#pragma unroll
            for (int p = 0; p < 4; ++p)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int i = i0 + p, k = k0l + q;
                    if (i < nbk && k <= i) s[i + k * ld] = sub(s[i + k * ld], acc[p][q]);
                }
        }
        __syncthreads();
    }
    __syncthreads();
    return s_fail;
}

}  // namespace ddlak
