// Triangular solves of the mixed refinement by inverted diagonal super-blocks.
//
// The refinement solves L L^T x = b many times with one FP32 factor L (FP64
// vectors).  A chain of 64-row block rows is bound by the latency of its n/64
// sequential links; here the diagonal blocks of order BS = 1024 are inverted
// once (in FP64, by the batched W = L^-1 kernel on widened copies) and each
// direction is n/BS phases of two wide kernels:
//   forward,  phase s:  y_s = inv(L_ss) b_s;          b_i -= L_is y_s   (i > s)
//   backward, phase s:  x_s = inv(L_ss)^T y_s;        y_j -= L_sj^T x_s (j < s)
// The panel kernels stream the FP32 factor once per direction with 16-byte loads
// (HBM-bound), split along the 1024-long inner dimension when a phase has few
// row (column) tiles, the partial sums folded in with FP64 atomics.  The
// inverse blocks are mirrored into their unused upper halves so that both
// diagonal-block products read contiguous columns.  y lives in a scratch
// vector Y; b is overwritten by x.  nrhs <= 16.
#include <cuda_runtime.h>

#include <cstdint>

#include <ddla_kernels.h>

#include "common.cuh"
#include "profile.h"

namespace ddlak {
namespace {

constexpr int BS = 1024;  // super-block order
constexpr int BIS_NT = 256;

// tmp[s] (BS x BS, ld BS) = FP64 copy of the lower triangle of the diagonal block s of L32
__global__ void k_bis_widen(int n, const float* __restrict__ L, long long ldl, double* __restrict__ tmp)
{
    const int s = blockIdx.z;
    const long long s0 = (long long)s * BS;
    const int bsz = (int)((n - s0) < BS ? (n - s0) : BS);
    const int i = blockIdx.y * 32 + threadIdx.y, k = blockIdx.x * 32 + threadIdx.x;
    double* t = tmp + (long long)s * BS * BS;
    if (i >= BS || k >= BS) return;
    t[i + (long long)k * BS] = (i < bsz && k < bsz && i >= k) ? (double)L[(s0 + i) + (s0 + k) * ldl] : 0.0;
}

// Mirror the strictly lower part of every inverse block into its upper half:
// D[k + i BS] = D[i + k BS] for k < i.  Column i then holds row i of the
// inverse in rows 0..i and column i in rows i..: both products read columns.
__global__ void k_bis_mirror(double* __restrict__ Dinv)
{
    __shared__ double t[32][33];
    const int bx = blockIdx.x, by = blockIdx.y;
    if (by < bx) return;
    double* D = Dinv + (long long)blockIdx.z * BS * BS;
    const int tx = threadIdx.x, ty = threadIdx.y;
    t[ty][tx] = D[(by * 32 + tx) + (long long)(bx * 32 + ty) * BS];  // source (i, k), i = by*32+tx
    __syncthreads();
    const int k = bx * 32 + tx, i = by * 32 + ty;
    if (i > k) D[k + (long long)i * BS] = t[tx][ty];
}

// y_s = inv(L_ss) b_s (FWD) or x_s = inv(L_ss)^T y_s: one warp per output row i,
// lanes over column i of the mirrored inverse (rows 0..i, or i..bsz-1)
template <int NQ, bool FWD>
__global__ void __launch_bounds__(BIS_NT) k_bis_diag(int n, int nrhs, int s, const double* __restrict__ Dinv,
                                                     const double* __restrict__ Vin, long long ldin,
                                                     double* __restrict__ Vout, long long ldout)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* vs = reinterpret_cast<double*>(smem_raw);  // [NQ][BS]
    const long long s0 = (long long)s * BS;
    const int bsz = (int)((n - s0) < BS ? (n - s0) : BS);
    const double* D = Dinv + (long long)s * BS * BS;
    for (int e = threadIdx.x; e < bsz * NQ; e += BIS_NT) {
        const int k = e % bsz, q = e / bsz;
        vs[q * BS + k] = q < nrhs ? Vin[(s0 + k) + q * ldin] : 0.0;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * (BIS_NT / 32) + warp;
    if (i >= bsz) return;
    double acc[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) acc[q] = 0.0;
    const double* col = D + (long long)i * BS;
    const int kb = FWD ? 0 : i, ke = FWD ? i + 1 : bsz;
#pragma unroll 4
    for (int k = kb + lane; k < ke; k += 32) {
        const double d = col[k];
#pragma unroll
        for (int q = 0; q < NQ; ++q) acc[q] = fma(d, vs[q * BS + k], acc[q]);
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NQ; ++q)
            if (q < nrhs) Vout[(s0 + i) + q * ldout] = acc[q];
}

// b_i -= L(i, s-block k-range) y_s for the rows below block s, in 64-row tiles
// (tile bx, bx + gridDim.x, ...: the staged y range is reused) and the k-range of
// blockIdx.y (the range split over gridDim.y, partial sums folded in with atomics).
// thread (g: rows 4g..4g+3 of the tile read as float4, ks: one of 16 k-slices)
template <int NQ>
__global__ void __launch_bounds__(BIS_NT) k_bis_panel(int n, int nrhs, int s, const float* __restrict__ L,
                                                      long long ldl, const double* __restrict__ Y,
                                                      double* __restrict__ B, long long ldb)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int kseg = BS / gridDim.y;
    double (*ys)[NQ + 1] = reinterpret_cast<double (*)[NQ + 1]>(smem_raw);  // [kseg][NQ+1]
    double (*red)[64][NQ] = reinterpret_cast<double (*)[64][NQ]>(smem_raw + sizeof(double) * BS * (NQ + 1));
    const long long s0 = (long long)s * BS;
    const long long r0 = s0 + BS;  // first row below a full block s
    const long long tiles = ceil_div(n - r0, 64);
    const int kb0 = blockIdx.y * kseg;
    for (int e = threadIdx.x; e < kseg * NQ; e += BIS_NT) {
        const int k = e % kseg, q = e / kseg;
        ys[k][q] = q < nrhs ? Y[(s0 + kb0 + k) + q * (long long)n] : 0.0;
    }
    const int g = threadIdx.x & 15, ks = threadIdx.x >> 4;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kper = kseg / 16;
    const int kb = ks * kper, ke = kb + kper;
    for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const long long i0 = r0 + tile * 64;
        const long long ir = i0 + 4 * g;
        __syncthreads();  // ys staged / red of the previous tile consumed
        double acc[4][NQ];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int q = 0; q < NQ; ++q) acc[u][q] = 0.0;
        if (ir + 3 < n) {
            const float* base = L + ir + (s0 + kb0 + kb) * ldl;
#pragma unroll 8
            for (int k = kb; k < ke; ++k, base += ldl) {
                const float4 l = *reinterpret_cast<const float4*>(base);
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    const double y = ys[k][q];
                    acc[0][q] = fma((double)l.x, y, acc[0][q]);
                    acc[1][q] = fma((double)l.y, y, acc[1][q]);
                    acc[2][q] = fma((double)l.z, y, acc[2][q]);
                    acc[3][q] = fma((double)l.w, y, acc[3][q]);
                }
            }
        } else {
            for (int k = kb; k < ke; ++k)
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (ir + u < n) {
                        const double l = L[(ir + u) + (s0 + kb0 + k) * ldl];
#pragma unroll
                        for (int q = 0; q < NQ; ++q) acc[u][q] = fma(l, ys[k][q], acc[u][q]);
                    }
        }
        // reduce the 16 k-slices: pairs in-warp (lane ^ 16), then 8 partials through shared memory
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int q = 0; q < NQ; ++q) acc[u][q] += __shfl_xor_sync(0xffffffffu, acc[u][q], 16);
        if (lane < 16)
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int q = 0; q < NQ; ++q) red[warp][4 * g + u][q] = acc[u][q];
        __syncthreads();
        for (int e = threadIdx.x; e < 64 * NQ; e += BIS_NT) {
            const int r = e & 63, q = e >> 6;
            if (q < nrhs && i0 + r < n) {
                double sum = 0.0;
#pragma unroll
                for (int w = 0; w < BIS_NT / 32; ++w) sum += red[w][r][q];
                atomicAdd(&B[(i0 + r) + q * ldb], -sum);
            }
        }
    }
}

// y_j -= sum_{i in block s, row range of blockIdx.y} L(i, j) x_i for columns j < s*BS:
// one thread per column j (tiles of 256 columns, bx, bx + gridDim.x, ...), the
// column's rows read as float4 and its dot products kept in registers; x of the
// row range staged row-major so that its values are 128-bit broadcast reads.
template <int NQ>
__global__ void __launch_bounds__(BIS_NT) k_bis_panel_t(int n, int nrhs, int s, const float* __restrict__ L,
                                                        long long ldl, const double* __restrict__ B, long long ldb,
                                                        double* __restrict__ Y)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const long long s0 = (long long)s * BS;
    const int bsz = (int)((n - s0) < BS ? (n - s0) : BS);
    const int iseg = BS / gridDim.y;
    const int ib0 = blockIdx.y * iseg;
    if (ib0 >= bsz) return;
    const int ie = (ib0 + iseg) < bsz ? (ib0 + iseg) : bsz;
    const int cnt = ie - ib0;
    double (*xs)[NQ] = reinterpret_cast<double (*)[NQ]>(smem_raw);  // [iseg][NQ]
    for (int e = threadIdx.x; e < iseg * NQ; e += BIS_NT) {
        const int k = e / NQ, q = e % NQ;
        xs[k][q] = (q < nrhs && k < cnt) ? B[(s0 + ib0 + k) + q * ldb] : 0.0;
    }
    __syncthreads();
    const long long tiles = ceil_div(s0, BIS_NT);
    const int c4 = cnt & ~3;
    for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const long long j = tile * BIS_NT + threadIdx.x;
        if (j >= s0) continue;
        const float* col = L + s0 + ib0 + j * ldl;
        double acc[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) acc[q] = 0.0;
#pragma unroll 4
        for (int i = 0; i < c4; i += 4) {
            const float4 l = __ldg(reinterpret_cast<const float4*>(col + i));
#pragma unroll
            for (int q = 0; q < NQ; ++q)
                acc[q] = fma((double)l.x, xs[i][q],
                             fma((double)l.y, xs[i + 1][q], fma((double)l.z, xs[i + 2][q], fma((double)l.w, xs[i + 3][q], acc[q]))));
        }
        for (int i = c4; i < cnt; ++i) {
            const double l = col[i];
#pragma unroll
            for (int q = 0; q < NQ; ++q) acc[q] = fma(l, xs[i][q], acc[q]);
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q)
            if (q < nrhs) atomicAdd(&Y[j + q * (long long)n], -acc[q]);
    }
}

// the smallest power-of-two split (<= cap) giving at least `want` CTAs
int split_for(long long tiles, int cap, long long want)
{
    int k = 1;
    while (k < cap && tiles * k < want) k *= 2;
    return k;
}

template <int NQ>
cudaError_t bis_solve_t(int n, int nrhs, const float* L, long long ldl, const double* Dinv, double* B, long long ldb,
                        double* Y, cudaStream_t st)
{
    const int S = (int)ceil_div(n, BS);
    const size_t sm_panel = sizeof(double) * (BS * (NQ + 1) + (BIS_NT / 32) * 64 * NQ);
    const size_t sm_vec = sizeof(double) * BS * (NQ + 1);
    static bool attr = [&] {
        cudaFuncSetAttribute(k_bis_panel<NQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_panel);
        cudaFuncSetAttribute(k_bis_panel_t<NQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_vec);
        cudaFuncSetAttribute(k_bis_diag<NQ, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_vec);
        cudaFuncSetAttribute(k_bis_diag<NQ, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_vec);
        return true;
    }();
    (void)attr;
    int sms = 148;
    {
        int dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    const long long want = 3LL * sms;  // CTAs of a phase: resident CTAs on every SM
    int launches = 0;
    // forward: L y = b (y into Y)
    for (int s = 0; s < S; ++s) {
        const long long s0 = (long long)s * BS;
        const int bsz = (int)((n - s0) < BS ? (n - s0) : BS);
        k_bis_diag<NQ, true><<<(unsigned)ceil_div(bsz, BIS_NT / 32), BIS_NT, sm_vec, st>>>(n, nrhs, s, Dinv, B, ldb,
                                                                                          Y, n);
        ++launches;
        const long long rest = n - s0 - bsz;
        if (rest > 0) {
            const long long tiles = ceil_div(rest, 64);
            const int ks = split_for(tiles, 16, want);
            const long long gx = tiles < ceil_div(want, ks) ? tiles : ceil_div(want, ks);
            k_bis_panel<NQ><<<dim3((unsigned)gx, (unsigned)ks), BIS_NT, sm_panel, st>>>(n, nrhs, s, L, ldl, Y, B,
                                                                                        ldb);
            ++launches;
        }
    }
    // backward: L^T x = y (x into B)
    for (int s = S - 1; s >= 0; --s) {
        const long long s0 = (long long)s * BS;
        const int bsz = (int)((n - s0) < BS ? (n - s0) : BS);
        k_bis_diag<NQ, false><<<(unsigned)ceil_div(bsz, BIS_NT / 32), BIS_NT, sm_vec, st>>>(n, nrhs, s, Dinv, Y, n,
                                                                                           B, ldb);
        ++launches;
        if (s0 > 0) {
            const long long tiles = ceil_div(s0, BIS_NT);
            const int is = split_for(tiles, 16, want);
            const long long gx = tiles < ceil_div(want, is) ? tiles : ceil_div(want, is);
            k_bis_panel_t<NQ><<<dim3((unsigned)gx, (unsigned)is), BIS_NT, sm_vec, st>>>(n, nrhs, s, L, ldl, B, ldb,
                                                                                        Y);
            ++launches;
        }
    }
    note_launches(launches);
    return cudaGetLastError();
}

}  // namespace
}  // namespace ddlak

extern "C" int ddlak_bis_block(void) { return ddlak::BS; }

extern "C" unsigned long long ddlak_bis_inverse_bytes(int n)
{
    const unsigned long long S = (unsigned long long)ddlak::ceil_div(n > 0 ? n : 0, ddlak::BS);
    return S * ddlak::BS * ddlak::BS * sizeof(double);
}

extern "C" int ddlak_bis_inverse(int n, const void* L32, long long ldl, void* Dinv, void* tmp, void* stream)
{
    using namespace ddlak;
    if (n <= 0) return 0;
    if (!L32 || !Dinv || !tmp || ldl < n) return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int S = (int)ceil_div(n, BS);
    {
        ProfScope ps(PK_MIXED_OTHER, st, (double)S * BS * BS * BS / 3.0, 16.0 * S * BS * BS);
        dim3 grid(BS / 32, BS / 32, S), block(32, 32);
        k_bis_widen<<<grid, block, 0, st>>>(n, static_cast<const float*>(L32), ldl, static_cast<double*>(tmp));
        note_launches(1);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    const long long bb = (long long)BS * BS;
    const int full = n / BS, last = n - full * BS;
    int r = 0;
    if (full > 0)
        r = ddlak_trtri_batched('d', full, BS, tmp, BS, bb, Dinv, BS, bb, stream);
    if (r == 0 && last > 0)
        r = ddlak_trtri_batched('d', 1, last, static_cast<double*>(tmp) + full * bb, BS, bb,
                                static_cast<double*>(Dinv) + full * bb, BS, bb, stream);
    if (r != 0) return r;
    dim3 grid(BS / 32, BS / 32, S), block(32, 32);
    k_bis_mirror<<<grid, block, 0, st>>>(static_cast<double*>(Dinv));
    note_launches(1);
    return (int)cudaGetLastError();
}

extern "C" unsigned long long ddlak_bis_solve_workspace(int n, int nrhs)
{
    return ((unsigned long long)(n > 0 ? n : 0) * (nrhs > 0 ? nrhs : 0) * sizeof(double) + 255) / 256 * 256;
}

extern "C" int ddlak_bis_solve(int n, int nrhs, const void* L32, long long ldl, const void* Dinv, void* B,
                               long long ldb, void* work, unsigned long long work_bytes, void* stream)
{
    using namespace ddlak;
    if (n <= 0 || nrhs <= 0) return 0;
    if (nrhs > 16 || !L32 || !Dinv || !B || ldb < n || ldl < n || (ldl & 3) ||
        (reinterpret_cast<uintptr_t>(L32) & 15) || work_bytes < ddlak_bis_solve_workspace(n, nrhs))
        return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const double nd = n, rd = nrhs;
    ProfScope ps(PK_POTRS_FUSED, st, 2.0 * nd * nd * rd, 4.0 * nd * (nd + 1));
    const float* L = static_cast<const float*>(L32);
    const double* D = static_cast<const double*>(Dinv);
    double* b = static_cast<double*>(B);
    double* Y = static_cast<double*>(work);
    if (nrhs <= 8) return (int)bis_solve_t<8>(n, nrhs, L, ldl, D, b, ldb, Y, st);
    return (int)bis_solve_t<16>(n, nrhs, L, ldl, D, b, ldb, Y, st);
}
