// In-shared-memory Cholesky of one diagonal block (lower triangle of
// s[i + j*ld], i, j < nbk <= 128), shared by the plain and mixed factorizations.
//
// Right-looking, one column per step, with the block held in REGISTERS: the
// lower triangle is cut into BxB tiles and each thread owns one tile (136
// threads for a 128 x 128 block with B = 8).  Step j reads column j (current,
// unscaled values) and its pivot d = a_jj from a double-buffered shared
// vector, applies a_ik -= a_ij conj(a_kj) / d to the owned tile, the owners of
// column j+1 publish it, and the CTA synchronises once.  The square roots are
// deferred: the pivots are kept and every column is scaled by 1/sqrt(d_j) after
// the last step, so a step's critical path is one division and one
// multiply-add per element.  The column loop is unrolled by B so that the
// column's position inside a tile is a compile-time constant: the update has
// no per-element conditions (an upper-triangle element of a diagonal tile is
// updated too, never read for a lower one and never stored).
// Returns 0, or 1 + the index of the first column whose pivot is not positive
// (or NaN).  As in LAPACK ?potf2, the columns before it are final and the
// failed pivot keeps its value.
// Must be called by all threads of the CTA (blockDim.x >= number of tiles).
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

// tile edge: 8 for 4- and 8-byte types, 4 for complex double (register budget;
// complex double blocks are 64 wide, so 136 tiles either way)
template <class T> constexpr int diag_tile() { return sizeof(T) >= 16 ? 4 : 8; }

template <class T>
__device__ int factor_block_smem(T* s, int ld, int nbk)
{
    using R = real_t<T>;
    constexpr int B = diag_tile<T>();
    constexpr int MAXN = 128;
    static_assert(B % 2 == 0, "the column buffer parity must follow the column index within a tile");
    __shared__ T col[2][MAXN];
    __shared__ R piv[MAXN];
    __shared__ int s_fail;
    const int nt = (nbk + B - 1) / B;  // tiles per dimension
    const int ntiles = nt * (nt + 1) / 2;
    const int t = threadIdx.x;
    const bool owner = t < ntiles;
    int bi = 0, bk = 0;
    if (owner) {
        int i = (int)((sqrtf(8.f * t + 1.f) - 1.f) * 0.5f);
        while ((i + 1) * (i + 2) / 2 <= t) ++i;
        while (i * (i + 1) / 2 > t) --i;
        bi = i;
        bk = t - i * (i + 1) / 2;
    }
    const int r0 = bi * B, c0 = bk * B;
    T a[B][B];
#pragma unroll
    for (int p = 0; p < B; ++p)
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const int i = r0 + p, k = c0 + q;
            a[p][q] = (owner && i < nbk && k < nbk && i >= k) ? s[i + k * ld] : zero<T>();
        }
    // entries past nbk stay zero, so the update needs no range checks
    for (int i = t; i < 2 * MAXN; i += blockDim.x) col[i / MAXN][i % MAXN] = zero<T>();
    if (t == 0) s_fail = 0;
    __syncthreads();
    if (owner && bk == 0)
#pragma unroll
        for (int p = 0; p < B; ++p)
            if (r0 + p < nbk) col[0][r0 + p] = a[p][0];
    __syncthreads();

    int fail = 0;
    for (int jt = 0; jt < nt && !fail; ++jt) {
#pragma unroll
        for (int jq = 0; jq < B; ++jq) {
            const int j = jt * B + jq;
            if (j < nbk && !fail) {
                const T* cv = col[jq & 1];
                const R d = re(cv[j]);
                if (!(d > R(0))) {
                    fail = j + 1;
                } else {
                    const R invd = R(1) / d;
                    if (t == 0) piv[j] = d;
                    if (owner && bk >= jt) {
                        T lk[B];
#pragma unroll
                        for (int q = 0; q < B; ++q) lk[q] = scal(cj(cv[c0 + q]), invd);
                        if (bk > jt) {
#pragma unroll
                            for (int p = 0; p < B; ++p) {
                                const T li = cv[r0 + p];
#pragma unroll
                                for (int q = 0; q < B; ++q) a[p][q] = fms(a[p][q], li, lk[q]);
                            }
                        } else {
#pragma unroll
                            for (int p = 0; p < B; ++p) {
                                const T li = cv[r0 + p];
#pragma unroll
                                for (int q = jq + 1; q < B; ++q) a[p][q] = fms(a[p][q], li, lk[q]);
                            }
                        }
                        // publish column j+1 (its step-j update is complete)
                        if (jq + 1 < B) {
                            if (bk == jt)
#pragma unroll
                                for (int p = 0; p < B; ++p)
                                    if (r0 + p < nbk) col[(jq + 1) & 1][r0 + p] = a[p][jq + 1];
                        } else if (bk == jt + 1) {
#pragma unroll
                            for (int p = 0; p < B; ++p)
                                if (r0 + p < nbk) col[0][r0 + p] = a[p][0];
                        }
                    }
                }
                __syncthreads();
            }
        }
    }
    // deferred scaling of the final columns: l_kk = sqrt(d_k), l_ik = a_ik / sqrt(d_k)
    const int done = fail ? fail - 1 : nbk;
    if (owner) {
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const int k = c0 + q;
            if (k < done) {
                const R dk = piv[k];
                const R sk = sqrt(dk);
                const R rs = R(1) / sk;
#pragma unroll
                for (int p = 0; p < B; ++p) {
                    const int i = r0 + p;
                    if (i == k) a[p][q] = from_real<T>(sk);
                    else if (i > k) a[p][q] = scal(a[p][q], rs);
                }
            }
        }
    }
    if (t == 0) s_fail = fail;
#pragma unroll
    for (int p = 0; p < B; ++p)
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const int i = r0 + p, k = c0 + q;
            if (owner && i < nbk && k < nbk && i >= k) s[i + k * ld] = a[p][q];
        }
    __syncthreads();
    return s_fail;
}

}  // namespace ddlak
