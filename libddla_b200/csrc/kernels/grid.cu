// Local kernels of the distributed (P x Q grid) Cholesky factorization and
// triangular solve.  The reference runs these steps with vendor calls on its
// stored tiles (herk / gemm / gemmBatched in src/Cholesky/ppotrf.cpp:196-317,
// gemm in src/PBLAS/ptrtrs.cpp:209-224) after moving panels between ranks;
// here every rank first holds the whole solved panel in global row order (the
// "full panel" F, assembled by the host from the ranks' pieces), and one
// kernel applies it to the rank's local block-cyclic storage through index
// maps, so no per-tile pointer arrays and no per-tile launches are needed.
//
// Index map (ddlak_gmap): local index l of a block-cyclically distributed
// dimension (block nb, nprocs processes, this rank's coordinate coord, first
// process src), offset by `first`, goes to
//   g(l) = ((L / nb) * nprocs + (coord - src) mod nprocs) * nb + L mod nb - base,
// L = first + l (the ScaLAPACK local-to-global map, minus `base`); nprocs == 0
// is the identity l -> l.
#include <cuda_runtime.h>

#include <ddla_kernels.h>

#include "common.cuh"
#include "profile.h"

namespace ddlak {
namespace {

__device__ __forceinline__ long long gmap(const ddlak_gmap& m, long long l)
{
    if (m.nprocs == 0) return l;
    const long long L = m.first + l;
    const long long blk = L / m.nb;
    return (blk * m.nprocs + ((m.coord - m.src) % m.nprocs + m.nprocs) % m.nprocs) * m.nb + (L - blk * m.nb) -
           m.base;
}

template <class T> __device__ __forceinline__ T tmul(T a, T b) { return fma_(zero<T>(), a, b); }

constexpr int GT = 64;  // output tile
constexpr int GK = 16;  // contraction slab

// C(i, j) = beta C(i, j) + alpha sum_p opA(i, p) opB(p, j) on the elements the mask keeps:
//   opA(i, p) = A[ma(i) + p lda]          (AC false)   conj(A[ma(p) + i lda])  (AC true)
//   opB(p, j) = B[mb(p) + j ldb]          (BC false)   conj(B[mb(j) + p ldb])  (BC true)
//   MASK 0: every element; 1: mi(i) >= mj(j); 2: mi(i) <= mj(j).
// With beta_zero, C is written without being read.
template <class T, bool AC, bool BC, int MASK>
__global__ void __launch_bounds__(256) k_grid_gemm(int m, int n, int k, T alpha, const T* __restrict__ A,
                                                   long long lda, ddlak_gmap ma, const T* __restrict__ B,
                                                   long long ldb, ddlak_gmap mb, T beta, int beta_zero,
                                                   T* __restrict__ C, long long ldc, ddlak_gmap mi, ddlak_gmap mj)
{
    __shared__ T As[GK][GT + 1];
    __shared__ T Bs[GK][GT + 1];
    const int i0 = blockIdx.y * GT, j0 = blockIdx.x * GT;
    if (MASK != 0) {
        // the maps are increasing, so a tile entirely outside the kept triangle is skipped
        const long long gi_lo = gmap(mi, i0), gi_hi = gmap(mi, min(i0 + GT, m) - 1);
        const long long gj_lo = gmap(mj, j0), gj_hi = gmap(mj, min(j0 + GT, n) - 1);
        if (MASK == 1 && gi_hi < gj_lo) return;
        if (MASK == 2 && gi_lo > gj_hi) return;
    }
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    T acc[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = zero<T>();
    for (int p0 = 0; p0 < k; p0 += GK) {
        for (int e = threadIdx.x; e < GK * GT; e += blockDim.x) {
            // consecutive threads walk the stored dimension of each operand
            const int pp = AC ? (e % GK) : (e / GT), ii = AC ? (e / GK) : (e % GT);
            const int i = i0 + ii, p = p0 + pp;
            T v = zero<T>();
            if (i < m && p < k) v = AC ? cj(A[gmap(ma, p) + (long long)i * lda]) : A[gmap(ma, i) + (long long)p * lda];
            As[pp][ii] = v;
        }
        for (int e = threadIdx.x; e < GK * GT; e += blockDim.x) {
            const int pp = BC ? (e / GT) : (e % GK), jj = BC ? (e % GT) : (e / GK);
            const int j = j0 + jj, p = p0 + pp;
            T v = zero<T>();
            if (j < n && p < k) v = BC ? cj(B[gmap(mb, j) + (long long)p * ldb]) : B[gmap(mb, p) + (long long)j * ldb];
            Bs[pp][jj] = v;
        }
        __syncthreads();
#pragma unroll 4
        for (int pp = 0; pp < GK; ++pp) {
            T a[4], b[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) a[u] = As[pp][tx + 16 * u];
#pragma unroll
            for (int v = 0; v < 4; ++v) b[v] = Bs[pp][ty + 16 * v];
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[u][v] = fma_(acc[u][v], a[u], b[v]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int i = i0 + tx + 16 * u, j = j0 + ty + 16 * v;
            if (i >= m || j >= n) continue;
            if (MASK == 1 && gmap(mi, i) < gmap(mj, j)) continue;
            if (MASK == 2 && gmap(mi, i) > gmap(mj, j)) continue;
            T* c = C + i + (long long)j * ldc;
            const T t = tmul(alpha, acc[u][v]);
            *c = beta_zero ? t : add(tmul(beta, *c), t);
        }
}

// dst(i, j) = src(i, j), or conj(src(j, i)) with conj_trans; i < rows, j < cols
template <class T>
__global__ void k_grid_pack(int conj_trans, int rows, int cols, const T* __restrict__ src, long long lds,
                            T* __restrict__ dst, long long ldd)
{
    const long long total = (long long)rows * cols;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % rows), j = (int)(e / rows);
        dst[i + j * ldd] = conj_trans ? cj(src[j + i * lds]) : src[i + j * lds];
    }
}

// dst(g(l), c) = src(l, c), l < rows, c < cols
template <class T>
__global__ void k_grid_unscatter(int rows, int cols, const T* __restrict__ src, long long lds, T* __restrict__ dst,
                                 long long ldd, ddlak_gmap map)
{
    const long long total = (long long)rows * cols;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int l = (int)(e % rows), c = (int)(e / rows);
        dst[gmap(map, l) + c * ldd] = src[l + c * lds];
    }
}

template <class T>
__global__ void k_grid_identity(int n, T* __restrict__ W, long long ldw)
{
    const long long total = (long long)n * n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % n), j = (int)(e / n);
        W[i + j * ldw] = i == j ? from_real<T>(real_t<T>(1)) : zero<T>();
    }
}

template <class R>
__global__ void k_grid_accumulate(unsigned long long count, const R* __restrict__ src, R* __restrict__ dst)
{
    for (unsigned long long e = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; e < count;
         e += (unsigned long long)gridDim.x * blockDim.x)
        dst[e] += src[e];
}

unsigned elementwise_grid(long long total)
{
    const long long b = (total + 255) / 256;
    return (unsigned)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

template <class T> T scalar_of(double re, double im);
template <> float scalar_of<float>(double re, double) { return (float)re; }
template <> double scalar_of<double>(double re, double) { return re; }
template <> cf32 scalar_of<cf32>(double re, double im) { return {(float)re, (float)im}; }
template <> cf64 scalar_of<cf64>(double re, double im) { return {re, im}; }

template <class T, bool AC, bool BC>
cudaError_t gemm_masked(int mask, dim3 grid, cudaStream_t st, int m, int n, int k, T alpha, const T* A, long long lda,
                        const ddlak_gmap& ma, const T* B, long long ldb, const ddlak_gmap& mb, T beta, int bz, T* C,
                        long long ldc, const ddlak_gmap& mi, const ddlak_gmap& mj)
{
    if (mask == 1)
        k_grid_gemm<T, AC, BC, 1><<<grid, 256, 0, st>>>(m, n, k, alpha, A, lda, ma, B, ldb, mb, beta, bz, C, ldc, mi, mj);
    else if (mask == 2)
        k_grid_gemm<T, AC, BC, 2><<<grid, 256, 0, st>>>(m, n, k, alpha, A, lda, ma, B, ldb, mb, beta, bz, C, ldc, mi, mj);
    else
        k_grid_gemm<T, AC, BC, 0><<<grid, 256, 0, st>>>(m, n, k, alpha, A, lda, ma, B, ldb, mb, beta, bz, C, ldc, mi, mj);
    return cudaGetLastError();
}

template <class T>
cudaError_t gemm_typed(char opA, char opB, int mask, int m, int n, int k, const double* alpha, const void* A,
                       long long lda, const ddlak_gmap& ma, const void* B, long long ldb, const ddlak_gmap& mb,
                       const double* beta, void* C, long long ldc, const ddlak_gmap& mi, const ddlak_gmap& mj,
                       cudaStream_t st)
{
    const dim3 grid((unsigned)((n + GT - 1) / GT), (unsigned)((m + GT - 1) / GT));
    const T al = scalar_of<T>(alpha[0], alpha[1]);
    const int bz = beta == nullptr;
    const T be = bz ? zero<T>() : scalar_of<T>(beta[0], beta[1]);
    const T* a = static_cast<const T*>(A);
    const T* b = static_cast<const T*>(B);
    T* c = static_cast<T*>(C);
    note_launches(1);
    if (opA == 'C' && opB == 'C')
        return gemm_masked<T, true, true>(mask, grid, st, m, n, k, al, a, lda, ma, b, ldb, mb, be, bz, c, ldc, mi, mj);
    if (opA == 'C')
        return gemm_masked<T, true, false>(mask, grid, st, m, n, k, al, a, lda, ma, b, ldb, mb, be, bz, c, ldc, mi, mj);
    if (opB == 'C')
        return gemm_masked<T, false, true>(mask, grid, st, m, n, k, al, a, lda, ma, b, ldb, mb, be, bz, c, ldc, mi, mj);
    return gemm_masked<T, false, false>(mask, grid, st, m, n, k, al, a, lda, ma, b, ldb, mb, be, bz, c, ldc, mi, mj);
}

template <class T>
cudaError_t elementwise_typed(int what, int flag, int rows, int cols, const void* src, long long lds, void* dst,
                              long long ldd, const ddlak_gmap* map, cudaStream_t st)
{
    const unsigned g = elementwise_grid((long long)rows * cols);
    note_launches(1);
    if (what == 0)
        k_grid_pack<T><<<g, 256, 0, st>>>(flag, rows, cols, static_cast<const T*>(src), lds, static_cast<T*>(dst), ldd);
    else if (what == 1)
        k_grid_unscatter<T><<<g, 256, 0, st>>>(rows, cols, static_cast<const T*>(src), lds, static_cast<T*>(dst), ldd,
                                               *map);
    else
        k_grid_identity<T><<<g, 256, 0, st>>>(rows, static_cast<T*>(dst), ldd);
    return cudaGetLastError();
}

template <class F>
int by_type(char type, F&& f)
{
    switch (type) {
    case 's': return (int)f(float{});
    case 'd': return (int)f(double{});
    case 'c': return (int)f(cf32{});
    case 'z': return (int)f(cf64{});
    default: return (int)cudaErrorInvalidValue;
    }
}

bool valid_map(const ddlak_gmap* m) { return m == nullptr || m->nprocs == 0 || (m->nprocs > 0 && m->nb > 0); }

}  // namespace
}  // namespace ddlak

using namespace ddlak;

extern "C" int ddlak_grid_gemm(char type, char opA, char opB, int mask, int m, int n, int k, const double* alpha,
                               const void* A, long long lda, const ddlak_gmap* ma, const void* B, long long ldb,
                               const ddlak_gmap* mb, const double* beta, void* C, long long ldc, const ddlak_gmap* mi,
                               const ddlak_gmap* mj, void* stream)
{
    if (m < 0 || n < 0 || k < 0 || mask < 0 || mask > 2 || !alpha || (opA != 'N' && opA != 'C') ||
        (opB != 'N' && opB != 'C') || !valid_map(ma) || !valid_map(mb) || !valid_map(mi) || !valid_map(mj))
        return (int)cudaErrorInvalidValue;
    if (mask != 0 && (!mi || !mj)) return (int)cudaErrorInvalidValue;
    if (m == 0 || n == 0) return 0;
    const ddlak_gmap id{0, 0, 0, 0, 0, 0};
    const ddlak_gmap& a = ma ? *ma : id;
    const ddlak_gmap& b = mb ? *mb : id;
    const ddlak_gmap& i = mi ? *mi : id;
    const ddlak_gmap& j = mj ? *mj : id;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return by_type(type, [&](auto t) {
        using T = decltype(t);
        return gemm_typed<T>(opA, opB, mask, m, n, k, alpha, A, lda, a, B, ldb, b, beta, C, ldc, i, j, st);
    });
}

extern "C" int ddlak_grid_pack(char type, int conj_trans, int rows, int cols, const void* src, long long lds,
                               void* dst, long long ldd, void* stream)
{
    if (rows < 0 || cols < 0) return (int)cudaErrorInvalidValue;
    if (rows == 0 || cols == 0) return 0;
    return by_type(type, [&](auto t) {
        return elementwise_typed<decltype(t)>(0, conj_trans, rows, cols, src, lds, dst, ldd, nullptr,
                                              static_cast<cudaStream_t>(stream));
    });
}

extern "C" int ddlak_grid_unscatter(char type, int rows, int cols, const void* src, long long lds, void* dst,
                                    long long ldd, const ddlak_gmap* map, void* stream)
{
    if (rows < 0 || cols < 0 || !map || !valid_map(map)) return (int)cudaErrorInvalidValue;
    if (rows == 0 || cols == 0) return 0;
    return by_type(type, [&](auto t) {
        return elementwise_typed<decltype(t)>(1, 0, rows, cols, src, lds, dst, ldd, map,
                                              static_cast<cudaStream_t>(stream));
    });
}

extern "C" int ddlak_grid_identity(char type, int n, void* W, long long ldw, void* stream)
{
    if (n < 0 || ldw < n) return (int)cudaErrorInvalidValue;
    if (n == 0) return 0;
    return by_type(type, [&](auto t) {
        return elementwise_typed<decltype(t)>(2, 0, n, n, nullptr, 0, W, ldw, nullptr,
                                              static_cast<cudaStream_t>(stream));
    });
}

extern "C" int ddlak_grid_accumulate(char real_type, unsigned long long count, const void* src, void* dst,
                                     void* stream)
{
    if (count == 0) return 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const unsigned g = elementwise_grid((long long)count);
    note_launches(1);
    if (real_type == 's')
        k_grid_accumulate<float><<<g, 256, 0, st>>>(count, static_cast<const float*>(src), static_cast<float*>(dst));
    else if (real_type == 'd')
        k_grid_accumulate<double><<<g, 256, 0, st>>>(count, static_cast<const double*>(src), static_cast<double*>(dst));
    else
        return (int)cudaErrorInvalidValue;
    return (int)cudaGetLastError();
}
