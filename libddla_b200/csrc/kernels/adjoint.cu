// Cholesky / solve / log-determinant adjoint for loss = 1/2 (y^T A^-1 y + log det A)
// (no reference counterpart).  With A = L L^T and alpha = A^-1 y,
//   dloss/dA = Abar = 1/2 (A^-1 - alpha alpha^T),   dloss/dy = alpha,
// and A^-1 = W^T W with W = L^-1.  Kernels, over a batch of equal-order
// matrices laid out with fixed strides:
//   k_gp_build        A = K(theta) + sigma^2 I (squared-exponential kernel on
//                     points in R^d), lower triangle only (all the factorization reads);
//   k_trtri_batched   W = L^-1 (lower), one CTA per matrix and block-column range (order <= 1024):
//                     block columns of width B; for each 32-row block the rows'
//                     partial results are staged in shared memory, all warps solve
//                     them against the 32 x 32 diagonal block of L (a few columns
//                     each, shuffles), and every thread updates the rows it owns
//                     below from registers.  For FP64 it inverts only the 64 x 64
//                     diagonal blocks, which k_trtri_level joins pairwise on the
//                     FP64 tensor cores (recursive inversion, bottom-up);
//   k_adjoint_contract  (W^T W) tile by tile (128 x 128 lower tiles, k from the tile's
//                     first row: W is lower triangular) with a fused epilogue that
//                     either contracts Abar with dA/dtheta (recomputed from the
//                     points, never stored) into per-tile partial sums, or writes
//                     the dense symmetric Abar;
//   k_adjoint_reduce  per-matrix sums of the partials in a fixed order (deterministic);
//   k_batched_dot     y^T alpha per problem (FP64 accumulation).
#include <cuda_runtime.h>

#include <type_traits>

#include <ddla_kernels.h>

#include "common.cuh"
#include "profile.h"
#include "tc_common.cuh"

namespace ddlak {
namespace {

constexpr int TR_NT = 512;
constexpr int TR_NMAX = 1024;
constexpr int CT_TILE = 128;
// k-chunk of the contraction: 32 KB of static shared memory for both types
template <class T> constexpr int ct_kc() { return 64 / (int)sizeof(T); }
constexpr int CT_NT = 256;

// ---------------------------------------------------------------------------
// A = sigma_f^2 exp(-|x_i - x_j|^2 / (2 l^2)) + sigma^2 delta_ij, lower triangle.
// theta = {l, sigma_f^2, sigma^2} per matrix (tstride 3) or shared (tstride 0).
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_gp_build(int n, int d, const T* __restrict__ X, long long xstride, const double* __restrict__ theta,
                           int tstride, T* __restrict__ A, long long lda, long long astride)
{
    const int m = blockIdx.z;
    const int i = blockIdx.y * 32 + threadIdx.y, j0 = blockIdx.x * 32;
    if (j0 > blockIdx.y * 32 + 31) return;  // tile above the diagonal
    const T* x = X + m * xstride;
    const double* th = theta + (long long)m * tstride;
    const double l = th[0], sf2 = th[1], s2 = th[2];
    const double inv2l2 = 0.5 / (l * l);
    T* a = A + m * astride;
    const int j = j0 + threadIdx.x;
    if (i >= n || j >= n || j > i) return;
    double r2 = 0.0;
    for (int c = 0; c < d; ++c) {
        const double dx = (double)x[(long long)i * d + c] - (double)x[(long long)j * d + c];
        r2 += dx * dx;
    }
    double v = sf2 * exp(-r2 * inv2l2);
    if (i == j) v += s2;
    a[i + (long long)j * lda] = (T)v;
}

// ---------------------------------------------------------------------------
// W = L^-1 for every matrix of the batch (order n <= 1024), lower triangle of W.
// ---------------------------------------------------------------------------
template <class T> struct TrWidth { static constexpr int B = 16; };
template <> struct TrWidth<float> { static constexpr int B = 32; };

template <class T>
__global__ void __launch_bounds__(TR_NT, 1)
    k_trtri_batched(int n, const T* __restrict__ Lg, long long ldl, long long lstride, T* __restrict__ Wg,
                    long long ldw, long long wstride, int nsub, long long lsub, long long wsub)
{
    constexpr int B = TrWidth<T>::B;
    constexpr int RPT = TR_NMAX / TR_NT;
    constexpr int CPW = B / (TR_NT / 32);  // columns each warp solves
    __shared__ T Xs[2][32][B + 1];                  // staged rows, then the solved block (padded)
    __shared__ __align__(16) T Xr[2][32][B];        // the solved block, row-major for 128-bit broadcast reads
    __shared__ T Ls[2][32][33];
    __shared__ T Ri[2][32];  // reciprocal pivots of the staged diagonal block
    // blockIdx.x = matrix * nsub + sub-block (the diagonal blocks of a recursive inversion)
    const long long mm = blockIdx.x / nsub, sub = blockIdx.x % nsub;
    const T* L = Lg + mm * lstride + sub * lsub;
    T* W = Wg + mm * wstride + sub * wsub;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    // block columns of W are independent: part p of gridDim.y takes the range
    // [jb, je) holding about 1/P of the work ((n - J)^3 / 3 beyond column J)
    const int P = gridDim.y, p = blockIdx.y;
    auto jstart = [&](int q) -> int {
        if (q <= 0) return 0;
        if (q >= P) return n;
        const double f = 1.0 - cbrt((double)(P - q) / (double)P);
        return min(n, (int)(f * n) / B * B);
    };
    const int jb = jstart(p), je = jstart(p + 1);
    int step = 0;
    for (int J = jb; J < je; J += B) {
        const int nb = min(B, n - J);
        T acc[RPT][B];
#pragma unroll
        for (int r = 0; r < RPT; ++r)
#pragma unroll
            for (int q = 0; q < B; ++q) acc[r][q] = (t + r * TR_NT == J + q && q < nb) ? T(1) : T(0);
        const int I0 = J & ~31;
#pragma unroll
        for (int rb = 0; rb < RPT; ++rb) {
            for (int wb = 0; wb < TR_NT / 32; ++wb) {
                const int I = rb * TR_NT + wb * 32;
                if (I < I0 || I >= n) continue;  // uniform
                const int buf = step & 1;
                ++step;
                // 1. stage this row block's partial results and the diagonal block of L
                if (warp == wb)
#pragma unroll
                    for (int q = 0; q < B; ++q) Xs[buf][lane][q] = acc[rb][q];
                for (int e = t; e < 32 * 32; e += TR_NT) {
                    const int r = e & 31, c = e >> 5;
                    Ls[buf][r][c] = (c <= r && I + r < n) ? L[(I + r) + (long long)(I + c) * ldl] : T(0);
                }
                if (t < 32) Ri[buf][t] = I + t < n ? T(1) / L[(I + t) + (long long)(I + t) * ldl] : T(0);
                __syncthreads();
                // 2. X_I = L_II^-1 Xs: warp w solves columns w*CPW .. w*CPW+CPW-1, lane = row
                {
                    T x[CPW];
#pragma unroll
                    for (int c = 0; c < CPW; ++c) x[c] = Xs[buf][lane][warp * CPW + c];
                    const bool live = I + lane < n;
#pragma unroll 4
                    for (int k = 0; k < 32; ++k) {
                        const T rk = Ri[buf][k];
                        const T lk = Ls[buf][lane][k];
#pragma unroll
                        for (int c = 0; c < CPW; ++c) {
                            if (lane == k) x[c] = live ? x[c] * rk : T(0);
                            const T xk = __shfl_sync(0xffffffffu, x[c], k);
                            if (lane > k) x[c] = fms(x[c], lk, xk);
                        }
                    }
#pragma unroll
                    for (int c = 0; c < CPW; ++c) {
                        const int q = warp * CPW + c;
                        Xr[buf][lane][q] = x[c];
                        if (live && q < nb && I + lane >= J + q) W[(I + lane) + (long long)(J + q) * ldw] = x[c];
                    }
                }
                __syncthreads();
                // 3. rows below the block: acc -= L(i, I:I+32) X_I, four columns of L
                // at a time (loads in flight together), rows of X_I as 128-bit broadcasts
                bool act[RPT];
#pragma unroll
                for (int r = 0; r < RPT; ++r) {
                    const int i = t + r * TR_NT;
                    act[r] = r >= rb && i >= I + 32 && i < n;
                }
                constexpr int VW = 16 / sizeof(T);
                using V = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
                constexpr int KL = 4;  // columns of L loaded together
                for (int k0 = 0; k0 < 32; k0 += KL) {
                    T lv[RPT][KL];
#pragma unroll
                    for (int r = 0; r < RPT; ++r) {
                        const T* li = L + (t + r * TR_NT) + (long long)(I + k0) * ldl;
#pragma unroll
                        for (int kk = 0; kk < KL; ++kk) lv[r][kk] = act[r] ? li[(long long)kk * ldl] : T(0);
                    }
#pragma unroll
                    for (int kk = 0; kk < KL; ++kk) {
                        T xr[B];
                        const V* src = reinterpret_cast<const V*>(&Xr[buf][k0 + kk][0]);
#pragma unroll
                        for (int v = 0; v < B / VW; ++v) {
                            const V w = src[v];
                            if constexpr (VW == 2) {
                                xr[2 * v] = w.x;
                                xr[2 * v + 1] = w.y;
                            } else {
                                xr[4 * v] = w.x;
                                xr[4 * v + 1] = w.y;
                                xr[4 * v + 2] = w.z;
                                xr[4 * v + 3] = w.w;
                            }
                        }
#pragma unroll
                        for (int r = 0; r < RPT; ++r)
                            if (act[r])
#pragma unroll
                                for (int q = 0; q < B; ++q) acc[r][q] = fms(acc[r][q], lv[r][kk], xr[q]);
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// (W^T W) on 128 x 128 lower tiles with the adjoint epilogue.
//   mode 0: partial[m][tile][0..2] = sum over the tile's i >= j of
//           w_ij Abar_ij dA_ij/d{l, sigma_f^2, sigma^2}, w = 2 off the diagonal;
//   mode 1: G[i + j ldg] = G[j + i ldg] = Abar_ij (dense symmetric gradient).
// DIRECT: the operand already is A^-1 (orders above the batched inversion's
// limit, where A^-1 comes from the fused solve on the identity): the tile is
// read instead of multiplied.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tile_of_lower(int t, int& ti, int& tj)
{
    int i = (int)((sqrtf(8.f * t + 1.f) - 1.f) * 0.5f);
    while ((i + 1) * (i + 2) / 2 <= t) ++i;
    while (i * (i + 1) / 2 > t) --i;
    ti = i;
    tj = t - i * (i + 1) / 2;
}

template <class T, int MODE, bool DIRECT>
__global__ void __launch_bounds__(CT_NT, 1)
    k_adjoint_contract(int n, const T* __restrict__ Wg, long long ldw, long long wstride,
                       const T* __restrict__ alpha_g, long long astride, const T* __restrict__ X, int d,
                       long long xstride, const double* __restrict__ theta, int tstride, double* __restrict__ partial,
                       T* __restrict__ G, long long ldg, long long gstride)
{
    // thread (ty, tx) of 16 x 16 owns rows i0 + {ty*4 .. +3, 64 + ty*4 .. +3} and the
    // same pattern of columns: the k-loop reads them as 4-element runs (conflict free)
    constexpr int CT_KC = ct_kc<T>();
    // rows padded by 4 elements: the staging stores (consecutive k in consecutive
    // threads) then fall in different banks
    __shared__ __align__(16) T Wi[2][CT_KC][CT_TILE + 4];
    __shared__ __align__(16) T Wj[2][CT_KC][CT_TILE + 4];
    __shared__ double red[3][CT_NT / 32];
    const int m = blockIdx.y;
    const int tile = blockIdx.x;
    int ti, tj;
    tile_of_lower(tile, ti, tj);
    const int i0 = ti * CT_TILE, j0 = tj * CT_TILE;
    const T* W = Wg + m * wstride;
    const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
    auto row_of = [&](int u) { return (u < 4 ? ty * 4 + u : 64 + ty * 4 + (u - 4)); };
    auto col_of = [&](int v) { return (v < 4 ? tx * 4 + v : 64 + tx * 4 + (v - 4)); };
    T acc[8][8];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[a][b] = T(0);
    // k runs over [i0, n): W(k, i) = 0 for k < i.  DIRECT: Wg holds A^-1 itself.
    const int kbeg = i0, nk = n - kbeg;
    const int nch = DIRECT ? 0 : (nk + CT_KC - 1) / CT_KC;
    if constexpr (DIRECT) {
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
            for (int v = 0; v < 8; ++v) {
                const int i = i0 + row_of(u), j = j0 + col_of(v);
                if (i < n && j <= i) acc[u][v] = W[i + (long long)j * ldw];
            }
    }
    auto stage = [&](int ch, int buf) {
        const int k0 = kbeg + ch * CT_KC;
        for (int e = t; e < CT_KC * CT_TILE; e += CT_NT) {
            const int kk = e % CT_KC, c = e / CT_KC;
            const int k = k0 + kk;
            const int ci = i0 + c, cj = j0 + c;
            const bool vi = k < n && ci < n && k >= ci, vj = k < n && cj < n && k >= cj;
            cp_async_elem<sizeof(T)>(&Wi[buf][kk][c], vi ? W + k + (long long)ci * ldw : W, vi);
            cp_async_elem<sizeof(T)>(&Wj[buf][kk][c], vj ? W + k + (long long)cj * ldw : W, vj);
        }
    };
    if (nch > 0) stage(0, 0);
    cp_group_commit();
    constexpr int VW = 16 / sizeof(T);
    using V = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
    auto ld4 = [&](const T* p, T* out) {
#pragma unroll
        for (int h = 0; h < 4 / VW; ++h) {
            const V w = reinterpret_cast<const V*>(p)[h];
            if constexpr (VW == 2) {
                out[2 * h] = w.x;
                out[2 * h + 1] = w.y;
            } else {
                out[0] = w.x;
                out[1] = w.y;
                out[2] = w.z;
                out[3] = w.w;
            }
        }
    };
    for (int ch = 0; ch < nch; ++ch) {
        if (ch + 1 < nch) stage(ch + 1, (ch + 1) & 1);
        cp_group_commit();
        cp_group_wait<1>();
        __syncthreads();
        const int buf = ch & 1;
#pragma unroll
        for (int kk = 0; kk < CT_KC; ++kk) {
            T a[8], b[8];
            ld4(&Wi[buf][kk][ty * 4], a);
            ld4(&Wi[buf][kk][64 + ty * 4], a + 4);
            ld4(&Wj[buf][kk][tx * 4], b);
            ld4(&Wj[buf][kk][64 + tx * 4], b + 4);
#pragma unroll
            for (int u = 0; u < 8; ++u)
#pragma unroll
                for (int v = 0; v < 8; ++v) acc[u][v] = fma_(acc[u][v], a[u], b[v]);
        }
        __syncthreads();
    }
    cp_group_wait<0>();

    const T* al = alpha_g + m * astride;
    if constexpr (MODE == 1) {
        T* g = G + m * gstride;
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
            for (int v = 0; v < 8; ++v) {
                const int i = i0 + row_of(u), j = j0 + col_of(v);
                if (i < n && j <= i) {
                    const T ab = T(0.5) * (acc[u][v] - al[i] * al[j]);
                    g[i + (long long)j * ldg] = ab;
                    g[j + (long long)i * ldg] = ab;
                }
            }
    } else {
        const double* th = theta + (long long)m * tstride;
        const double l = th[0], sf2 = th[1];
        const double inv2l2 = 0.5 / (l * l), invl3 = 1.0 / (l * l * l);
        const T* x = X + m * xstride;
        double g0 = 0.0, g1 = 0.0, g2 = 0.0;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int i = i0 + row_of(u);
            if (i >= n) continue;
            const double ai = (double)al[i];
#pragma unroll
            for (int v = 0; v < 8; ++v) {
                const int j = j0 + col_of(v);
                if (j <= i) {
                    const double ab = 0.5 * ((double)acc[u][v] - ai * (double)al[j]);
                    const double w = i == j ? 1.0 : 2.0;
                    double r2 = 0.0;
                    for (int c = 0; c < d; ++c) {
                        const double dx = (double)x[(long long)i * d + c] - (double)x[(long long)j * d + c];
                        r2 += dx * dx;
                    }
                    const double e = exp(-r2 * inv2l2);
                    g0 += w * ab * sf2 * e * r2 * invl3;  // dA/dl
                    g1 += w * ab * e;                     // dA/dsigma_f^2
                    if (i == j) g2 += ab;                 // dA/dsigma^2
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            g0 += __shfl_xor_sync(0xffffffffu, g0, o);
            g1 += __shfl_xor_sync(0xffffffffu, g1, o);
            g2 += __shfl_xor_sync(0xffffffffu, g2, o);
        }
        if ((t & 31) == 0) {
            red[0][t >> 5] = g0;
            red[1][t >> 5] = g1;
            red[2][t >> 5] = g2;
        }
        __syncthreads();
        if (t < 3) {
            double sum = 0.0;
            for (int w = 0; w < CT_NT / 32; ++w) sum += red[t][w];
            partial[((long long)m * gridDim.x + tile) * 3 + t] = sum;
        }
    }
}

// out[m] = sum_i x_m[i] y_m[i] in FP64, one CTA per vector
template <class T>
__global__ void k_batched_dot(int n, const T* __restrict__ x, long long xs, const T* __restrict__ y, long long ys,
                              double* __restrict__ out)
{
    __shared__ double red[8];
    const int m = blockIdx.x;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += (double)x[m * xs + i] * (double)y[m * ys + i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += red[w];
        out[m] = r;
    }
}

// out[m] = 2 sum_i log L_m(i, i) in FP64 (log det of L L^T), one CTA per matrix
template <class T>
__global__ void k_batched_logdiag(int n, const T* __restrict__ L, long long ldl, long long ls, double* __restrict__ out)
{
    __shared__ double red[8];
    const int m = blockIdx.x;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += log((double)L[m * ls + i + (long long)i * ldl]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += red[w];
        out[m] = 2.0 * r;
    }
}

// grad[m][c] = sum over tiles of partial[m][tile][c], in tile order
__global__ void k_adjoint_reduce(int ntiles, const double* __restrict__ partial, double* __restrict__ grad)
{
    const int m = blockIdx.x, c = threadIdx.x;
    if (c >= 3) return;
    double s = 0.0;
    for (int k = 0; k < ntiles; ++k) s += partial[((long long)m * ntiles + k) * 3 + c];
    grad[(long long)m * 3 + c] = s;
}

template <class T>
int gp_build_t(int batch, int n, int d, const void* X, long long xstride, const double* theta, int tstride, void* A,
               long long lda, long long astride, cudaStream_t st)
{
    const int nt = (n + 31) / 32;
    dim3 grid(nt, nt, batch), block(32, 32);
    k_gp_build<T><<<grid, block, 0, st>>>(n, d, static_cast<const T*>(X), xstride, theta, tstride, static_cast<T*>(A),
                                         lda, astride);
    note_launches(1);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Recursive FP64 inversion, bottom-up: the 64 x 64 diagonal blocks by
// k_trtri_leaf64, then for h = 64, 128, ... each pair of inverted h-blocks
// (o = 2 p h) is joined by
//   W21 = -W22 (L21 W11),  L21 = L(o+h.., o..), W11 = W(o.., o..), W22 = W(o+h.., o+h..),
// two batched products on the FP64 tensor cores (mma.sync m16n8k4):
//   step 1: T = L21 W11 (W11 lower: k >= j), kept transposed in W's strictly
//           upper block W(o.., o+h..), which the result does not use;
//   step 2: W21 = -W22 T (W22 lower: k <= i), written to W(o+h.., o..).
// 64 x 64 tiles, 4 warps of 32 x 32, k in chunks of 32 staged by cp.async
// (double-buffered, three CTAs per SM); shared rows padded to 68 / 36 doubles so that the fragment reads
// are conflict free.  The strictly upper triangles of W are read nowhere
// (masked) and are overwritten as scratch.
// ---------------------------------------------------------------------------
constexpr int TL_BK = 32, TL_NS = 2, TL_LDK = 68, TL_LDJ = 36;  // 2 stages: 72 KB, 3 CTAs per SM
constexpr int TL_ASZ = TL_BK * TL_LDK;  // A slice [k][i]
constexpr int TL_BSZ = 64 * TL_LDJ;     // B slice [j][k] (step 1) or [k][j] (step 2, 32 x 68 fits)
constexpr size_t TL_SMEM = (size_t)TL_NS * (TL_ASZ + TL_BSZ) * sizeof(double);

__device__ __forceinline__ void tl_mma(double (&u)[2], double (&v)[2], double a_up, double a_lo, double b)
{
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
                 : "+d"(u[0]), "+d"(u[1]), "+d"(v[0]), "+d"(v[1])
                 : "d"(a_up), "d"(a_lo), "d"(b));
}

template <int STEP>
__global__ void __launch_bounds__(128) k_trtri_level(int n, int h, const double* __restrict__ Lg, long long ldl,
                                                     long long lstride, double* __restrict__ Wg, long long ldw,
                                                     long long wstride)
{
    extern __shared__ __align__(16) double tl_smem[];
    const int p = blockIdx.y;
    const long long m = blockIdx.z;
    const int o = 2 * p * h, r2 = min(h, n - o - h);  // rows of the lower block (> 0 by the grid)
    const int ntn = h / 64;
    const int i0 = (blockIdx.x / ntn) * 64, j0 = (blockIdx.x % ntn) * 64;
    if (i0 >= r2) return;
    const double* L = Lg + m * lstride;
    double* W = Wg + m * wstride;
    const int kbeg = STEP == 1 ? j0 : 0;
    const int kend = STEP == 1 ? h : min(i0 + 64, r2);
    const int nch = (kend - kbeg + TL_BK - 1) / TL_BK;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int wm = warp >> 1, wn = warp & 1, g = lane >> 2, q = lane & 3;

    auto stage = [&](int c, int sidx) {
        double* As = tl_smem + (size_t)sidx * (TL_ASZ + TL_BSZ);
        double* Bs = As + TL_ASZ;
        const int k0 = kbeg + c * TL_BK;
        for (int e = t; e < TL_BK * 64; e += 128) {
            const int i = e & 63, kk = e >> 6, k = k0 + kk, gi = i0 + i;
            bool v;
            const double* src;
            if (STEP == 1) {
                v = gi < r2 && k < kend;
                src = L + (o + h + gi) + (long long)(o + k) * ldl;
            } else {
                v = gi < r2 && k < kend && k <= gi;
                src = W + (o + h + gi) + (long long)(o + h + k) * ldw;
            }
            cp_async_elem<8>(&As[kk * TL_LDK + i], v ? src : W, v);
        }
        for (int e = t; e < TL_BK * 64; e += 128) {
            if (STEP == 1) {
                const int kk = e & 31, j = e >> 5, k = k0 + kk, gj = j0 + j;
                const bool v = k < kend && k >= gj;
                cp_async_elem<8>(&Bs[j * TL_LDJ + kk], v ? W + (o + k) + (long long)(o + gj) * ldw : W, v);
            } else {
                const int j = e & 63, kk = e >> 6, k = k0 + kk, gj = j0 + j;
                const bool v = k < kend;
                cp_async_elem<8>(&Bs[kk * TL_LDK + j], v ? W + (o + gj) + (long long)(o + h + k) * ldw : W, v);
            }
        }
    };

    double u[2][4][2], v[2][4][2];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) u[a][b][0] = u[a][b][1] = v[a][b][0] = v[a][b][1] = 0.0;
#pragma unroll
    for (int c = 0; c < TL_NS - 1; ++c) {
        if (c < nch) stage(c, c);
        cp_group_commit();
    }
    for (int c = 0; c < nch; ++c) {
        cp_group_wait<TL_NS - 2>();
        __syncthreads();
        if (c + TL_NS - 1 < nch) stage(c + TL_NS - 1, (c + TL_NS - 1) % TL_NS);
        cp_group_commit();
        const double* As = tl_smem + (size_t)(c % TL_NS) * (TL_ASZ + TL_BSZ);
        const double* Bs = As + TL_ASZ;
#pragma unroll
        for (int kk = 0; kk < TL_BK; kk += 4) {
            double a[2][2], b[4];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                a[mt][0] = As[(kk + q) * TL_LDK + wm * 32 + mt * 16 + g];
                a[mt][1] = As[(kk + q) * TL_LDK + wm * 32 + mt * 16 + 8 + g];
            }
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                const int jb = wn * 32 + nt * 8 + g;
                b[nt] = STEP == 1 ? Bs[jb * TL_LDJ + kk + q] : Bs[(kk + q) * TL_LDK + jb];
            }
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                for (int nt = 0; nt < 4; ++nt) tl_mma(u[mt][nt], v[mt][nt], a[mt][0], a[mt][1], b[nt]);
        }
    }
    cp_group_wait<0>();
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int j = j0 + wn * 32 + nt * 8 + 2 * q + e;
#pragma unroll
                for (int hh = 0; hh < 2; ++hh) {
                    const int i = i0 + wm * 32 + mt * 16 + g + 8 * hh;
                    if (i >= r2) continue;
                    const double val = hh ? v[mt][nt][e] : u[mt][nt][e];
                    if (STEP == 1) W[(o + j) + (long long)(o + h + i) * ldw] = val;
                    else W[(o + h + i) + (long long)(o + j) * ldw] = -val;
                }
            }
}

// The recursion's 64 x 64 leaves, four per CTA: thread j of a leaf's 64 computes
// column j of its inverse by substitution, w_j = 1 / l_jj and
// w_i = -(sum_{j <= k < i} l_ik w_k) / l_ii, with the column in registers and L
// read through the L1 cache (the 64 threads of a leaf read the same entry at each
// step).  Leaf g = blockIdx.x * 4 + threadIdx.x / 64 is block sub = g % nsub of
// matrix g / nsub; its order is 64, or `last` for the final block of a matrix
// whose order is not a multiple of 64.
constexpr int TLF = 64;
__global__ void __launch_bounds__(256) k_trtri_leaf64(long long nleaf, int nsub, int n, const double* __restrict__ Lg,
                                                      long long ldl, long long lstride, double* __restrict__ Wg,
                                                      long long ldw, long long wstride)
{
    const long long g = (long long)blockIdx.x * 4 + (threadIdx.x >> 6);
    if (g >= nleaf) return;
    const long long m = g / nsub;
    const int sub = (int)(g % nsub);
    const int o = sub * TLF, nb = n - o < TLF ? n - o : TLF;
    const int j = threadIdx.x & 63;
    const double* L = Lg + m * lstride + o + (long long)o * ldl;
    double* W = Wg + m * wstride + o + (long long)o * ldw;
    double w[TLF];
#pragma unroll
    for (int i = 0; i < TLF; ++i) {
        double acc = 0.0;
        const bool row = i < nb;
#pragma unroll
        for (int k = 0; k < i; ++k)
            if (row && k >= j) acc = fma(__ldg(&L[i + (long long)k * ldl]), w[k], acc);
        const double lii = row ? __ldg(&L[i + (long long)i * ldl]) : 1.0;
        w[i] = (i < j || !row) ? 0.0 : (i == j ? 1.0 / lii : -acc / lii);
    }
    if (j < nb)
#pragma unroll
        for (int i = 0; i < TLF; ++i)
            if (i >= j && i < nb) W[i + (long long)j * ldw] = w[i];
}

int trtri_recursive_f64(int batch, int n, const double* L, long long ldl, long long lstride, double* W, long long ldw,
                        long long wstride, cudaStream_t st)
{
    constexpr int LEAF = TLF;
    {
        const int nsub = (n + LEAF - 1) / LEAF;
        const long long nleaf = (long long)batch * nsub;
        k_trtri_leaf64<<<(unsigned)((nleaf + 3) / 4), 256, 0, st>>>(nleaf, nsub, n, L, ldl, lstride, W, ldw, wstride);
        note_launches(1);
    }
    if (cudaError_t e = cudaGetLastError(); e != cudaSuccess) return (int)e;
    if (cudaError_t e = smem_optin(k_trtri_level<1>, TL_SMEM); e != cudaSuccess) return (int)e;
    if (cudaError_t e = smem_optin(k_trtri_level<2>, TL_SMEM); e != cudaSuccess) return (int)e;
    for (int h = LEAF; h < n; h *= 2) {
        const int npairs = (n - h + 2 * h - 1) / (2 * h);  // pairs whose lower block exists
        const dim3 grid((unsigned)((h / 64) * (h / 64)), (unsigned)npairs, (unsigned)batch);
        k_trtri_level<1><<<grid, 128, TL_SMEM, st>>>(n, h, L, ldl, lstride, W, ldw, wstride);
        k_trtri_level<2><<<grid, 128, TL_SMEM, st>>>(n, h, L, ldl, lstride, W, ldw, wstride);
        note_launches(2);
    }
    return (int)cudaGetLastError();
}

template <class T>
int trtri_t(int batch, int n, const void* L, long long ldl, long long lstride, void* W, long long ldw,
            long long wstride, cudaStream_t st)
{
    // FP64 above one leaf, W apart from L: the recursive inversion on the tensor cores
    if constexpr (std::is_same<T, double>::value)
        if (n > 64 && L != W && batch <= 65535)
            return trtri_recursive_f64(batch, n, static_cast<const double*>(L), ldl, lstride, static_cast<double*>(W),
                                       ldw, wstride, st);
    // split each matrix over block-column ranges until the launch covers the SMs twice
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int parts = 1;
    while (parts < 8 && (long long)batch * parts < 2LL * sms && n / TrWidth<T>::B >= 4 * parts) parts *= 2;
    k_trtri_batched<T><<<dim3(batch, parts), TR_NT, 0, st>>>(n, static_cast<const T*>(L), ldl, lstride,
                                                             static_cast<T*>(W), ldw, wstride, 1, 0, 0);
    note_launches(1);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// The FP64 contraction (not DIRECT) on the FP64 tensor cores: the same tiles
// and epilogues, C(i, j) = sum_k W(k, i) W(k, j) by DMMA (mma.sync m16n8k4 f64,
// 8 warps of 64 x 32).  Operand slices arrive by TMA from the batch of W seen as
// a 3-D tensor: per stage the columns i0 .. i0+127 and j0 .. j0+127 over 32 k,
// as boxes of 36 k (the 4 extra pad the shared rows to 36 doubles, which keeps
// the fragment reads conflict free) x 128 columns, 3 stages; each warp releases
// a stage on its `empty` mbarrier, with no CTA barrier per chunk.  W's strictly
// upper triangle is unspecified after the inversion (the recursive one keeps
// scratch there), so in the chunks that reach it (k < i0 + 128) the fragments
// are masked as they are read.  Every wait is bounded: if one gives up the
// tile's result is NaN (the gradient comes back NaN) after a bounded wait for
// the copies still in flight.
// ---------------------------------------------------------------------------
constexpr int AD_BK = 32, AD_LDK = 36;
constexpr int AD_BOX = CT_TILE * AD_LDK;
constexpr unsigned AD_BOX_BYTES = AD_BOX * 8u;  // 36864
// TNC: the tile's column count.  128: 128 x 128 tiles, 8 warps, 3 stages, one CTA per SM
// (registers); 64: 128 x 64 tiles, 4 warps, 2 stages, two CTAs per SM, so that one CTA's
// prologue and epilogue run under the other's MMAs.  The warp tile is 64 x 32 in both.
#ifndef AD_CONTRACT_TNC
#define AD_CONTRACT_TNC 64
#endif
template <int TNC> struct AdShape {
    static constexpr int NT = 2 * TNC, NS = TNC == 128 ? 3 : 2, WN = TNC / 32;
    static constexpr int BOXJ = TNC * AD_LDK;
    static constexpr unsigned STAGE_BYTES = (unsigned)(AD_BOX + BOXJ) * 8u;
    static constexpr size_t SMEM = (size_t)NS * STAGE_BYTES + 128;
};

// tile t of the lower part, 128 x TNC tiles: (ti, tj) with tj <= ti (TNC = 128) or
// tj <= 2 ti + 1 (TNC = 64, row ti holding 2 ti + 2 tiles)
template <int TNC>
__device__ __forceinline__ void ad_tile(int t, int& ti, int& tj)
{
    if constexpr (TNC == 128) {
        tile_of_lower(t, ti, tj);
    } else {
        int i = (int)((sqrtf(4.f * t + 1.f) - 1.f) * 0.5f);
        while ((i + 1) * (i + 2) <= t) ++i;
        while (i > 0 && i * (i + 1) > t) --i;
        ti = i;
        tj = t - i * (i + 1);
    }
}

__device__ int g_adjoint_status;

template <int MODE, int TNC>
__global__ void __launch_bounds__(AdShape<TNC>::NT, TNC == 128 ? 1 : 2)
    k_adjoint_contract_dmma(const __grid_constant__ CUtensorMap wmap, const __grid_constant__ CUtensorMap wmapj,
                            int n, const double* __restrict__ alpha_g,
                            long long astride, const double* __restrict__ X, int d, long long xstride,
                            const double* __restrict__ theta, int tstride, double* __restrict__ partial,
                            double* __restrict__ G, long long ldg, long long gstride)
{
    using SH = AdShape<TNC>;
    constexpr int AD_NS = SH::NS, NW = SH::NT / 32;
    extern __shared__ __align__(128) unsigned char ad_raw[];
    __shared__ __align__(8) uint64_t full[AD_NS], empty[AD_NS];
    __shared__ double red[3][NW];
    // blockIdx.x = matrix, blockIdx.y = tile: the grid runs every matrix's longest tiles
    // (smallest i0, the most k) first
    const int m = blockIdx.x, tile = blockIdx.y;
    int ti, tj;
    ad_tile<TNC>(tile, ti, tj);
    const int i0 = ti * CT_TILE, j0 = tj * TNC;
    double* sm = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(ad_raw) + 127) & ~uintptr_t(127));
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int wm = warp / SH::WN, wn = warp % SH::WN;
    const int g = lane >> 2, q = lane & 3;
    const int kbeg = i0, nch = (n - kbeg + AD_BK - 1) / AD_BK;
    auto issue = [&](int c) {
        const int s = c % AD_NS;
        double* st = sm + (size_t)s * (AD_BOX + SH::BOXJ);
        tc::mbar_expect_tx(&full[s], SH::STAGE_BYTES);
        tc::tma_load_3d(st, &wmap, &full[s], kbeg + c * AD_BK, i0, m);
        tc::tma_load_3d(st + AD_BOX, &wmapj, &full[s], kbeg + c * AD_BK, j0, m);
    };
    if (t == 0) {
        for (int s = 0; s < AD_NS; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], NW);  // one arrival per warp
        }
        tc::mbar_fence_init();
        tc::prefetch_tmap(&wmap);
        tc::prefetch_tmap(&wmapj);
        for (int c = 0; c < AD_NS && c < nch; ++c) issue(c);
    }
    __syncthreads();
    double acc[8][4][2];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    bool ok = true;
    int consumed = 0, issued = nch < AD_NS ? nch : AD_NS;  // issued: thread 0's count
    for (int c = 0; c < nch; ++c) {
        const int s = c % AD_NS;
        if (!tc::mbar_wait(&full[s], (uint32_t)((c / AD_NS) & 1), &g_adjoint_status, 0x61)) {
            ok = false;
            break;
        }
        consumed = c + 1;
        const double* Wi = sm + (size_t)s * (AD_BOX + SH::BOXJ);
        const double* Wj = Wi + AD_BOX;
        const int k0 = kbeg + c * AD_BK;
        // W(k, col) = 0 for k < col (the strictly upper triangle, which the inversion
        // leaves unspecified): applied to the fragments of the chunks that reach it
        const bool mask_i = k0 < i0 + CT_TILE, mask_j = k0 < j0 + TNC;
        if (mask_i || mask_j) {
#pragma unroll
            for (int kk = 0; kk < AD_BK; kk += 4) {
                const int k = k0 + kk + q;
                double af[8], bf[4];
#pragma unroll
                for (int a = 0; a < 8; ++a) {
                    const int cl = wm * 64 + a * 8 + g;
                    const double v = Wi[cl * AD_LDK + kk + q];
                    af[a] = (mask_i && k < i0 + cl) ? 0.0 : v;
                }
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const int cl = wn * 32 + b * 8 + g;
                    const double v = Wj[cl * AD_LDK + kk + q];
                    bf[b] = (mask_j && k < j0 + cl) ? 0.0 : v;
                }
                // rows a*8+g and (a+1)*8+g as one m16n8k4 product: the same accumulators as two m8n8k4
#pragma unroll
                for (int a = 0; a < 8; a += 2)
#pragma unroll
                    for (int b = 0; b < 4; ++b) tl_mma(acc[a][b], acc[a + 1][b], af[a], af[a + 1], bf[b]);
            }
        } else {
            // the chunks clear of the triangle (all but the first few of a tile): the fragments
            // go from shared memory straight into the MMAs
#pragma unroll
            for (int kk = 0; kk < AD_BK; kk += 4) {
                double af[8], bf[4];
#pragma unroll
                for (int a = 0; a < 8; ++a) af[a] = Wi[(wm * 64 + a * 8 + g) * AD_LDK + kk + q];
#pragma unroll
                for (int b = 0; b < 4; ++b) bf[b] = Wj[(wn * 32 + b * 8 + g) * AD_LDK + kk + q];
#pragma unroll
                for (int a = 0; a < 8; a += 2)
#pragma unroll
                    for (int b = 0; b < 4; ++b) tl_mma(acc[a][b], acc[a + 1][b], af[a], af[a + 1], bf[b]);
            }
        }
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&empty[s]);  // this warp is done with stage s
        if (t == 0 && c >= 1 && c - 1 + AD_NS < nch) {
            const int cp = c - 1;  // refill chunk cp's stage with chunk cp + NS
            if (!tc::mbar_wait(&empty[cp % AD_NS], (uint32_t)((cp / AD_NS) & 1), &g_adjoint_status, 0x63)) {
                ok = false;
                break;
            }
            issue(cp + AD_NS);
            issued = cp + AD_NS + 1;
        }
    }
    ok = __syncthreads_and(ok);
    if (!ok) {
        // copies issued for chunks consumed .. issued - 1 may still be in flight
        if (t == 0)
            for (int c = consumed; c < issued; ++c)
                (void)tc::mbar_wait(&full[c % AD_NS], (uint32_t)((c / AD_NS) & 1), &g_adjoint_status, 0x62);
        __syncthreads();
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = nan;
    }
    const double* al = alpha_g + m * astride;
    auto row_of = [&](int a) { return i0 + wm * 64 + a * 8 + g; };
    auto col_of = [&](int b, int e) { return j0 + wn * 32 + b * 8 + 2 * q + e; };
    if constexpr (MODE == 1) {
        double* gm = G + m * gstride;
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int i = row_of(a), j = col_of(b, e);
                    if (i < n && j <= i) {
                        const double ab = 0.5 * (acc[a][b][e] - al[i] * al[j]);
                        gm[i + (long long)j * ldg] = ab;
                        gm[j + (long long)i * ldg] = ab;
                    }
                }
    } else {
        // the tile into shared memory (the operand stages are free: every chunk was consumed and
        // the barrier above passed), then one rolled loop over its entries, so that the
        // exponential's code is not replicated for every fragment entry
        constexpr int CLD = TNC + 1;
        double* cs = sm;
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b)
#pragma unroll
                for (int e = 0; e < 2; ++e)
                    cs[(wm * 64 + a * 8 + g) * CLD + wn * 32 + b * 8 + 2 * q + e] = acc[a][b][e];
        __syncthreads();
        const double* th = theta + (long long)m * tstride;
        const double l = th[0], sf2 = th[1];
        const double inv2l2 = 0.5 / (l * l), invl3 = 1.0 / (l * l * l);
        const double* x = X + m * xstride;
        double g0 = 0.0, g1 = 0.0, g2 = 0.0;
#pragma unroll 1
        for (int e = t; e < CT_TILE * TNC; e += SH::NT) {
            const int il = e / TNC, jl = e % TNC;
            const int i = i0 + il, j = j0 + jl;
            if (i >= n || j > i) continue;
            const double ab = 0.5 * (cs[il * CLD + jl] - al[i] * al[j]);
            const double w = i == j ? 1.0 : 2.0;
            double r2 = 0.0;
            for (int cc = 0; cc < d; ++cc) {
                const double dx = x[(long long)i * d + cc] - x[(long long)j * d + cc];
                r2 += dx * dx;
            }
            const double ex = exp(-r2 * inv2l2);
            g0 += w * ab * sf2 * ex * r2 * invl3;  // dA/dl
            g1 += w * ab * ex;                     // dA/dsigma_f^2
            if (i == j) g2 += ab;                  // dA/dsigma^2
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            g0 += __shfl_xor_sync(0xffffffffu, g0, o);
            g1 += __shfl_xor_sync(0xffffffffu, g1, o);
            g2 += __shfl_xor_sync(0xffffffffu, g2, o);
        }
        if (lane == 0) {
            red[0][warp] = g0;
            red[1][warp] = g1;
            red[2][warp] = g2;
        }
        __syncthreads();
        if (t < 3) {
            double sum = 0.0;
            for (int w = 0; w < NW; ++w) sum += red[t][w];
            partial[((long long)m * gridDim.y + tile) * 3 + t] = sum;
        }
    }
}

// The DMMA contraction when W's layout suits TMA (16-byte aligned base, even
// ldw and matrix stride); false (nothing launched) otherwise.
bool contract_dmma(int mode, int batch, int n, const double* W, long long ldw, long long wstride, const double* alpha,
                   long long astride, const double* X, int d, long long xstride, const double* theta, int tstride,
                   double* partial, double* grad, double* G, long long ldg, long long gstride, cudaStream_t st,
                   cudaError_t* err)
{
    constexpr int TNC = AD_CONTRACT_TNC;
    using SH = AdShape<TNC>;
    CUtensorMap wmap, wmapj;
    if (!tc::encode_colmajor_3d(&wmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, W, n, n, ldw, batch, wstride, AD_LDK,
                                CT_TILE) ||
        !tc::encode_colmajor_3d(&wmapj, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, W, n, n, ldw, batch, wstride, AD_LDK,
                                TNC))
        return false;
    const int nt = (n + CT_TILE - 1) / CT_TILE;
    const int ntiles = TNC == 64 ? nt * (nt + 1) : nt * (nt + 1) / 2;  // 64 columns: row ti holds 2 ti + 2 tiles
    if (ntiles > 65535) return false;
    dim3 grid(batch, ntiles);
    if (mode == 0) {
        if ((*err = smem_optin(k_adjoint_contract_dmma<0, TNC>, SH::SMEM)) != cudaSuccess) return true;
        k_adjoint_contract_dmma<0, TNC><<<grid, SH::NT, SH::SMEM, st>>>(wmap, wmapj, n, alpha, astride, X, d, xstride,
                                                                        theta, tstride, partial, nullptr, 0, 0);
        k_adjoint_reduce<<<batch, 32, 0, st>>>(ntiles, partial, grad);
        note_launches(2);
    } else {
        if ((*err = smem_optin(k_adjoint_contract_dmma<1, TNC>, SH::SMEM)) != cudaSuccess) return true;
        k_adjoint_contract_dmma<1, TNC><<<grid, SH::NT, SH::SMEM, st>>>(wmap, wmapj, n, alpha, astride, nullptr, 0, 0,
                                                                        nullptr, 0, nullptr, G, ldg, gstride);
        note_launches(1);
    }
    *err = cudaGetLastError();
    return true;
}

template <class T, bool DIRECT>
int contract_t(int mode, int batch, int n, const void* W, long long ldw, long long wstride, const void* alpha,
               long long astride, const void* X, int d, long long xstride, const double* theta, int tstride,
               double* partial, double* grad, void* G, long long ldg, long long gstride, cudaStream_t st)
{
    if constexpr (std::is_same<T, double>::value && !DIRECT) {
        cudaError_t e = cudaSuccess;
        if (contract_dmma(mode, batch, n, static_cast<const double*>(W), ldw, wstride,
                          static_cast<const double*>(alpha), astride, static_cast<const double*>(X), d, xstride, theta,
                          tstride, partial, grad, static_cast<double*>(G), ldg, gstride, st, &e))
            return (int)e;
    }
    const int nt = (n + CT_TILE - 1) / CT_TILE;
    const int ntiles = nt * (nt + 1) / 2;
    dim3 grid(ntiles, batch);
    if (mode == 0) {
        k_adjoint_contract<T, 0, DIRECT><<<grid, CT_NT, 0, st>>>(n, static_cast<const T*>(W), ldw, wstride,
                                                         static_cast<const T*>(alpha), astride,
                                                         static_cast<const T*>(X), d, xstride, theta, tstride, partial,
                                                         nullptr, 0, 0);
        k_adjoint_reduce<<<batch, 32, 0, st>>>(ntiles, partial, grad);
        note_launches(2);
    } else {
        k_adjoint_contract<T, 1, DIRECT><<<grid, CT_NT, 0, st>>>(n, static_cast<const T*>(W), ldw, wstride,
                                                         static_cast<const T*>(alpha), astride, nullptr, 0, 0,
                                                         nullptr, 0, nullptr, static_cast<T*>(G), ldg, gstride);
        note_launches(1);
    }
    return (int)cudaGetLastError();
}

}  // namespace
}  // namespace ddlak

extern "C" int ddlak_gp_build(char type, int batch, int n, int d, const void* X, long long xstride,
                              const double* theta, int tstride, void* A, long long lda, long long astride,
                              void* stream)
{
    using namespace ddlak;
    if (batch <= 0 || n <= 0) return 0;
    if (d < 1 || d > 16 || !X || !theta || !A || lda < n) return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ProfScope ps(PK_ADJOINT, st, 0.0, 0.0);
    if (type == 'd') return gp_build_t<double>(batch, n, d, X, xstride, theta, tstride, A, lda, astride, st);
    if (type == 's') return gp_build_t<float>(batch, n, d, X, xstride, theta, tstride, A, lda, astride, st);
    return (int)cudaErrorInvalidValue;
}

extern "C" int ddlak_trtri_batched(char type, int batch, int n, const void* L, long long ldl, long long lstride,
                                   void* W, long long ldw, long long wstride, void* stream)
{
    using namespace ddlak;
    if (batch <= 0 || n <= 0) return 0;
    if (n > TR_NMAX || !L || !W || ldl < n || ldw < n) return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const double nn = n;
    ProfScope ps(PK_TRTRI, st, batch * nn * nn * nn / 3.0, batch * nn * nn * (type == 'd' ? 8.0 : 4.0));
    if (type == 'd') return trtri_t<double>(batch, n, L, ldl, lstride, W, ldw, wstride, st);
    if (type == 's') return trtri_t<float>(batch, n, L, ldl, lstride, W, ldw, wstride, st);
    return (int)cudaErrorInvalidValue;
}

extern "C" unsigned long long ddlak_adjoint_partial_bytes(int batch, int n)
{
    // three partial sums per tile: the FP64 contraction's 128 x 64 tiles, nt (nt + 1) per
    // matrix (the register-tiled form uses nt (nt + 1) / 2 of 128 x 128)
    const unsigned long long nt = (unsigned long long)(n + ddlak::CT_TILE - 1) / ddlak::CT_TILE;
    return sizeof(double) * 3ull * (unsigned long long)batch * (nt * (nt + 1));
}

extern "C" int ddlak_batched_dot(char type, int batch, int n, const void* x, long long xstride, const void* y,
                                 long long ystride, double* out, void* stream)
{
    using namespace ddlak;
    if (batch <= 0) return 0;
    if (n < 0 || !out || (n > 0 && (!x || !y))) return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (type == 'd')
        k_batched_dot<double><<<batch, 256, 0, st>>>(n, static_cast<const double*>(x), xstride,
                                                     static_cast<const double*>(y), ystride, out);
    else if (type == 's')
        k_batched_dot<float><<<batch, 256, 0, st>>>(n, static_cast<const float*>(x), xstride,
                                                    static_cast<const float*>(y), ystride, out);
    else
        return (int)cudaErrorInvalidValue;
    note_launches(1);
    return (int)cudaGetLastError();
}

extern "C" int ddlak_batched_logdiag(char type, int batch, int n, const void* L, long long ldl, long long lstride,
                                     double* out, void* stream)
{
    using namespace ddlak;
    if (batch <= 0) return 0;
    if (n < 0 || !out || (n > 0 && (!L || ldl < n))) return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (type == 'd')
        k_batched_logdiag<double><<<batch, 256, 0, st>>>(n, static_cast<const double*>(L), ldl, lstride, out);
    else if (type == 's')
        k_batched_logdiag<float><<<batch, 256, 0, st>>>(n, static_cast<const float*>(L), ldl, lstride, out);
    else
        return (int)cudaErrorInvalidValue;
    note_launches(1);
    return (int)cudaGetLastError();
}

extern "C" int ddlak_adjoint_contract(char type, int mode, int batch, int n, const void* W, long long ldw,
                                      long long wstride, const void* alpha, long long astride, const void* X, int d,
                                      long long xstride, const double* theta, int tstride, double* partial,
                                      double* grad, void* G, long long ldg, long long gstride, void* stream)
{
    using namespace ddlak;
    if (batch <= 0 || n <= 0) return 0;
    if (!W || !alpha || ldw < n || mode < 0 || mode > 3) return (int)cudaErrorInvalidValue;
    if ((mode & 1) == 0 && (!X || d < 1 || d > 16 || !theta || !partial || !grad)) return (int)cudaErrorInvalidValue;
    if ((mode & 1) == 1 && (!G || ldg < n)) return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const double nn = n;
    ProfScope ps(PK_ADJOINT, st, batch * nn * nn * nn / 3.0, 0.0);
    const bool direct = (mode & 2) != 0;
    mode &= 1;
    if (type == 'd')
        return direct ? contract_t<double, true>(mode, batch, n, W, ldw, wstride, alpha, astride, X, d, xstride, theta,
                                                 tstride, partial, grad, G, ldg, gstride, st)
                      : contract_t<double, false>(mode, batch, n, W, ldw, wstride, alpha, astride, X, d, xstride,
                                                  theta, tstride, partial, grad, G, ldg, gstride, st);
    if (type == 's')
        return direct ? contract_t<float, true>(mode, batch, n, W, ldw, wstride, alpha, astride, X, d, xstride, theta,
                                                tstride, partial, grad, G, ldg, gstride, st)
                      : contract_t<float, false>(mode, batch, n, W, ldw, wstride, alpha, astride, X, d, xstride,
                                                 theta, tstride, partial, grad, G, ldg, gstride, st);
    return (int)cudaErrorInvalidValue;
}
