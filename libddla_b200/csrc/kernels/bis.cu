// Triangular solves of the mixed refinement by inverted diagonal super-blocks.
//
// The refinement solves L L^T x = b many times with one FP32 factor L.  The
// diagonal blocks of order BS = 1024 are inverted once (in FP64, by the batched
// W = L^-1 kernel on widened copies), and each solve is then
//   forward,  phase s = 0..S-1:   y_s = inv(L_ss) b_s;        b_i -= L_is y_s   (i > s)
//   backward, phase s = S-1..0:   x_s = inv(L_ss)^T y_s;      y_j -= L_sj^T x_s (j < s)
// run by ONE persistent kernel (k_bis_chain) over a queue of units in that
// order.  A unit on the chain from one diagonal block to the next is a 64-row
// (or 64-column) tile times one 256-wide slice of the inner dimension (KS):
// 64 KB of FP32 matrix, one TMA box streamed into shared memory while the unit
// waits for its inputs; the rest of each panel goes in whole-block bulk units
// (four boxes) that trail the chain (queue order below).  A CTA takes the next
// unit from an atomic counter, starts its matrix loads, waits (bounded) on the
// counters its inputs are published on, computes, folds its partial product
// into the target vector with atomics and counts itself done:
//   cnt_f[t]   forward panel units applied to tile t of b    (complete at 4 per earlier phase)
//   ydone[p]   forward diagonal units done for 64-row part p of y
//   fdone      forward units done (the backward pass starts when all are)
//   cnt_b[t]   backward panel units applied to tile t of y
//   xdone[p]   backward diagonal units done for part p of x
// Every wait is on units earlier in the queue, held by running CTAs, so the
// queue cannot deadlock.  Splitting the inner dimension puts four CTAs on each
// tile of the chain from one diagonal block to the next, and because the
// contributions to a tile commute, the bulk of each panel never waits for
// another phase.  The atomics make the last bits of the result depend on the
// order the units finish.
//
// Arithmetic type T: float for the classic refinement sweeps (the FP32 factor
// with FP32 solves, as LAPACK ?sposv: the solve's rounding is far below the
// factor's), double for the GMRES preconditioner.  Vectors are held row-major,
// 8 right-hand sides per row (32 or 64 bytes), the inverse blocks in T with
// their strictly lower part mirrored into the upper half so that both the
// product with inv(L_ss) and with its transpose read 4 contiguous rows per
// load.  nrhs <= 16 (two passes of 8 beyond 8).  If a wait gives up, the
// status word is set, every CTA leaves, and the solution is returned as NaN,
// which the refinement treats as a failed sweep.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include <ddla_kernels.h>

#include "common.cuh"
#include "profile.h"
#include "tc_common.cuh"

namespace ddlak {
namespace {

constexpr int BS = 1024;  // super-block order
constexpr int CT = 64;    // rows of a vector tile
constexpr int TPB = BS / CT;
constexpr int CQ = 8;     // right-hand sides per pass
constexpr int CH_NT = 512;

// tmp[s] (BS x BS, ld BS) = FP64 copy of the lower triangle of the diagonal block s of L32
template <class LT>
__global__ void k_bis_widen(int n, const LT* __restrict__ L, long long ldl, double* __restrict__ tmp)
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
// D[k + i BS] = D[i + k BS] for k < i.
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

__global__ void k_bis_narrow(long long count, const double* __restrict__ src, float* __restrict__ dst)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count; e += (long long)gridDim.x * blockDim.x)
        dst[e] = (float)src[e];
}

// ---------------------------------------------------------------------------
// the persistent chain
// ---------------------------------------------------------------------------
struct Chain {
    int n, S, Tt;
    long long nf, total;
    long long ldl;
    int* ctl;  // [0] status, [1] fdone, [2..3] queue head (64-bit)
    int* cnt_f;
    int* ydone;
    int* cnt_b;
    int* xdone;
};

constexpr int KS = 256;  // inner-dimension slice of a unit
constexpr int QPB = BS / KS;

__host__ __device__ __forceinline__ int blk_size(int n, int s)
{
    const long long r = (long long)n - (long long)s * BS;
    return r < BS ? (int)r : BS;
}
__host__ __device__ __forceinline__ int blk_parts(int n, int s) { return (blk_size(n, s) + CT - 1) / CT; }
__host__ __device__ __forceinline__ int blk_slices(int n, int s) { return (blk_size(n, s) + KS - 1) / KS; }
// slices of the forward diagonal part p (columns 0 .. min((p+1)*64, bsz)) and of the backward one (p*64 .. bsz)
__host__ __device__ __forceinline__ int fdiag_slices(int bsz, int p)
{
    const int ke = (p + 1) * CT < bsz ? (p + 1) * CT : bsz;
    return (ke + KS - 1) / KS;
}
__host__ __device__ __forceinline__ int bdiag_slices(int bsz, int p) { return (bsz + KS - 1) / KS - (p * CT) / KS; }
__host__ __device__ __forceinline__ int fdiag_units(int bsz)
{
    int u = 0;
    for (int p = 0; p < (bsz + CT - 1) / CT; ++p) u += fdiag_slices(bsz, p);
    return u;
}
__host__ __device__ __forceinline__ int bdiag_units(int bsz)
{
    int u = 0;
    for (int p = 0; p < (bsz + CT - 1) / CT; ++p) u += bdiag_slices(bsz, p);
    return u;
}

// Queue order.  Forward group g = 0..S-1: the diagonal slices of block g
// (kind 0), the sliced panel units of phase g on the tiles of blocks g+1..g+LA
// (kind 1: the next diagonal blocks' inputs), then the bulk of phase g-LAG: one
// unit per tile of blocks g-LAG+LA+1.. over the whole inner range (kind 4).
// Backward group g = S-1..0: the diagonal slices of block g (kind 2), the
// sliced panel units of phase g on the column tiles of blocks g-1..g-LA
// (kind 3), then the bulk of phase g+LAG on the column tiles of blocks
// < g+LAG-LA (kind 5).  A phase's bulk is taken LAG groups after its diagonal
// block, when its inputs are long complete, and its first tiles are needed
// LA-LAG+1 groups later, so the chain from one diagonal block to the next
// neither queues behind the bulk nor waits for it.
constexpr int LA = 3;
constexpr int LAG = 2;
static_assert(LAG <= LA, "a bulk unit must precede every diagonal block it feeds");

__host__ __device__ __forceinline__ long long group_units(int n, int S, int Tt, bool fwd, int g)
{
    const int nq = blk_slices(n, g);
    if (fwd) {
        long long u = fdiag_units(blk_size(n, g));
        const long long ce = (long long)(g + LA + 1) * TPB < Tt ? (long long)(g + LA + 1) * TPB : Tt;
        if (ce > (long long)(g + 1) * TPB) u += (ce - (long long)(g + 1) * TPB) * nq;
        if (g >= LAG) {
            const long long b0 = (long long)(g - LAG + LA + 1) * TPB;
            if (Tt > b0) u += Tt - b0;
        }
        return u;
    }
    long long u = bdiag_units(blk_size(n, g));
    u += (long long)(g - (g > LA ? g - LA : 0)) * TPB * nq;
    if (g + LAG <= S - 1 && g + LAG - LA > 0) u += (long long)(g + LAG - LA) * TPB;
    return u;
}

// unit v of group g -> (kind, phase, index, slice); index = diagonal part
// (kinds 0, 2), row tile (1, 4) or column tile (3, 5)
__host__ __device__ void decode_in_group(const Chain& c, bool fwd, int g, long long v, int& kind, int& s, int& idx,
                                         int& kq)
{
    const int bsz = blk_size(c.n, g), dp = blk_parts(c.n, g), nq = blk_slices(c.n, g);
    kq = 0;
    if (fwd) {
        for (int p = 0; p < dp; ++p) {
            const int k = fdiag_slices(bsz, p);
            if (v < k) { kind = 0; s = g; idx = p; kq = (int)v; return; }
            v -= k;
        }
        const long long ce = (long long)(g + LA + 1) * TPB < c.Tt ? (long long)(g + LA + 1) * TPB : c.Tt;
        const long long nc = ce > (long long)(g + 1) * TPB ? (ce - (long long)(g + 1) * TPB) * nq : 0;
        if (v < nc) { kind = 1; s = g; idx = (g + 1) * TPB + (int)(v / nq); kq = (int)(v % nq); return; }
        v -= nc;
        kind = 4;
        s = g - LAG;
        idx = (g - LAG + LA + 1) * TPB + (int)v;
        return;
    }
    for (int p = dp - 1; p >= 0; --p) {
        const int k = bdiag_slices(bsz, p);
        if (v < k) { kind = 2; s = g; idx = p; kq = (p * CT) / KS + (int)v; return; }
        v -= k;
    }
    const long long nc = (long long)(g - (g > LA ? g - LA : 0)) * TPB * nq;
    if (v < nc) { kind = 3; s = g; idx = g * TPB - 1 - (int)(v / nq); kq = (int)(v % nq); return; }
    v -= nc;
    kind = 5;
    s = g + LAG;
    idx = (g + LAG - LA) * TPB - 1 - (int)v;
}

// unit u -> group by a forward scan (the checker's reference; the kernel keeps a cursor)
__host__ __device__ void decode_unit(const Chain& c, long long u, int& kind, int& s, int& idx, int& kq)
{
    long long base = 0;
    for (int g = 0; g < c.S; ++g) {
        const long long gu = group_units(c.n, c.S, c.Tt, true, g);
        if (u < base + gu) { decode_in_group(c, true, g, u - base, kind, s, idx, kq); return; }
        base += gu;
    }
    for (int g = c.S - 1; g >= 0; --g) {
        const long long gu = group_units(c.n, c.S, c.Tt, false, g);
        if (u < base + gu) { decode_in_group(c, false, g, u - base, kind, s, idx, kq); return; }
        base += gu;
    }
    kind = -1;
    s = idx = kq = 0;
}

// A CTA takes increasing unit numbers, so its group is found by moving forward.
struct Cursor {
    bool fwd = true;
    int g = 0;
    long long base = 0;
    __host__ __device__ void decode(const Chain& c, long long u, int& kind, int& s, int& idx, int& kq)
    {
        while (true) {
            if (fwd ? g >= c.S : g < 0) { kind = -1; s = idx = kq = 0; return; }
            const long long gu = group_units(c.n, c.S, c.Tt, fwd, g);
            if (u < base + gu) { decode_in_group(c, fwd, g, u - base, kind, s, idx, kq); return; }
            base += gu;
            if (fwd && g == c.S - 1) { fwd = false; g = c.S - 1; }
            else g += fwd ? 1 : -1;
        }
    }
};

template <class T> struct VecIO;
template <> struct VecIO<float> {
    static __device__ __forceinline__ void ld8(const float* p, float (&v)[CQ])
    {
        const float4 a = *reinterpret_cast<const float4*>(p), b = *reinterpret_cast<const float4*>(p + 4);
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    }
    static __device__ __forceinline__ void ld4(const float* p, float (&a)[4])
    {
        const float4 v = *reinterpret_cast<const float4*>(p);
        a[0] = v.x; a[1] = v.y; a[2] = v.z; a[3] = v.w;
    }
};
template <> struct VecIO<double> {
    static __device__ __forceinline__ void ld8(const double* p, double (&v)[CQ])
    {
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const double2 a = *reinterpret_cast<const double2*>(p + 2 * h);
            v[2 * h] = a.x;
            v[2 * h + 1] = a.y;
        }
    }
    static __device__ __forceinline__ void ld4(const double* p, double (&a)[4])
    {
        const double2 v0 = *reinterpret_cast<const double2*>(p), v1 = *reinterpret_cast<const double2*>(p + 2);
        a[0] = v0.x; a[1] = v0.y; a[2] = v1.x; a[3] = v1.y;
    }
};

// Every unit streams its matrix through shared memory in 64 KB chunks, one
// TMA box each: a 64-row x KC-column box of L or of the inverse blocks for the
// row units (KC = 256 for FP32, 128 for FP64), a PR-row x 64-column box of L
// for the column units (PR = 256 for an FP32 factor, 128 for FP64).  A TMA box costs a CTA about half a microsecond however
// large it is, so the boxes are as large as two stages of shared memory allow;
// a sliced unit is one box, prefetched in full while the unit waits.
constexpr int CHUNK = 65536;
constexpr int NSTAGE = 2;
template <class MT> constexpr int chunk_cols() { return CHUNK / (CT * (int)sizeof(MT)); }
template <class LT> constexpr int pt_rows() { return CHUNK / (CT * (int)sizeof(LT)); }  // rows of a column-unit chunk

// Row unit, one chunk: acc(4g+u, q) += sum over this thread's columns of the
// chunk (k-slice ks of 32) of M(4g+u, k) V(k, q), M(r, k) at tile[k*64 + r]
// (column k of the chunk = block column kb + j*KC + k), V(k, q) at
// vs[(j*KC + k)*CQ + q].  Columns at or past ke, and (MASK 1) past the row or
// (MASK 2) before it, contribute 0.
template <class T, class MT, int MASK>
__device__ __forceinline__ void row_chunk(const MT* tile, const T* vs, int j, int kb, int ke, int rloc, int g, int ks,
                                          T (&acc)[4][CQ])
{
    constexpr int KC = chunk_cols<MT>(), KT = KC / 32;
    const int r4 = 4 * g;
#pragma unroll 2
    for (int kk = 0; kk < KT; ++kk) {
        const int kc = ks * KT + kk;
        const int kabs = kb + j * KC + kc;
        MT a[4];
        VecIO<MT>::ld4(tile + kc * CT + r4, a);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int row = rloc + r4 + u;
            const bool ok = kabs < ke && (MASK != 1 || kabs <= row) && (MASK != 2 || kabs >= row);
            if (!ok) a[u] = MT(0);
        }
        T v[CQ];
        VecIO<T>::ld8(vs + (j * KC + kc) * CQ, v);
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int q = 0; q < CQ; ++q) acc[u][q] = fma((T)a[u], v[q], acc[u][q]);
    }
}

// Column unit, one chunk (rows j*PR .. j*PR+PR-1 of the unit, 64 columns,
// tile[c*PR + r]): warp w owns columns 4w..4w+3, lane l the rows 4l..4l+3 of
// each 128-row step, so the 32 lanes read 512 (FP32) or 1024 (FP64) contiguous
// bytes of a column.  xq holds the vector q-major (xq[q*XQ + row]), read the
// same way.  The sum over the lanes is taken once per unit (col_reduce).
template <class LT> constexpr int xq_rows() { return BS + pt_rows<LT>(); }  // rows of the q-major vector
template <class T, class LT>
__device__ __forceinline__ void col_chunk(const LT* tile, const T* xq, int j, T (&acc)[4][CQ])
{
    constexpr int PR = pt_rows<LT>(), XQ = xq_rows<LT>();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int step = 0; step < PR / 128; ++step) {
        const int r = step * 128 + 4 * lane;
        T x[CQ][4];
#pragma unroll
        for (int q = 0; q < CQ; ++q) VecIO<T>::ld4(xq + q * XQ + j * PR + r, x[q]);
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
            LT l[4];
            VecIO<LT>::ld4(tile + (4 * w + cc) * PR + r, l);
#pragma unroll
            for (int q = 0; q < CQ; ++q)
                acc[cc][q] = fma((T)l[3], x[q][3], fma((T)l[2], x[q][2], fma((T)l[1], x[q][1], fma((T)l[0], x[q][0], acc[cc][q]))));
        }
    }
}

// Sum v[0..7] over the 32 lanes of a warp in 9 shuffles: halves of the values
// are exchanged at distances 16, 8, 4, then the last value at 2 and 1.  Lane l
// ends with the total of value ((l >> 4) & 1)*4 + ((l >> 3) & 1)*2 + ((l >> 2) & 1).
template <class T>
__device__ __forceinline__ T warp_sum8(T (&v)[CQ])
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int m = 16, len = CQ; m >= 4; m >>= 1, len >>= 1) {
        const bool up = (lane & m) != 0;
        const int half = len / 2;
#pragma unroll
        for (int i = 0; i < half; ++i) {
            const T send = up ? v[i] : v[i + half];
            const T keep = up ? v[i + half] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, m);
        }
    }
    T r = v[0];
    r += __shfl_xor_sync(0xffffffffu, r, 2);
    r += __shfl_xor_sync(0xffffffffu, r, 1);
    return r;
}

constexpr int VS_ROWS = BS + 256;  // staged row-major vector rows: a block plus the overhang of the last chunk

// the reduction of a unit's partial sums (16 warps x 64 x CQ) reuses the stages
template <class T>
constexpr size_t chain_smem()
{
    static_assert((size_t)NSTAGE * CHUNK >= sizeof(T) * (CH_NT / 32) * CT * CQ, "reduction does not fit the stages");
    static_assert(VS_ROWS >= xq_rows<float>() && VS_ROWS >= xq_rows<double>(), "vector staging");
    return 1024 + (size_t)NSTAGE * CHUNK + sizeof(T) * (size_t)VS_ROWS * CQ;
}

// Thread 0's wait list for a unit, polled by the lanes of warp 0 in parallel.
__device__ __forceinline__ bool wait_inputs(const Chain& c, int kind, int s, int kb, int ke, int bsz, int* status)
{
    const int lane = threadIdx.x & 31;
    bool ok = true;
    const int lo = kb / CT, hi = (ke - 1) / CT;  // tiles or 64-row parts of block s the unit reads
    for (int i = lo + lane; i <= hi && ok; i += 32) {
        if (kind == 0) ok = bounded_wait_geq(&c.cnt_f[s * TPB + i], QPB * s, status);
        else if (kind == 1) ok = bounded_wait_geq(&c.ydone[s * TPB + i], fdiag_slices(bsz, i), status);
        else if (kind == 2) {
            const int need = s == c.S - 1 ? 0 : QPB * (c.S - 2 - s) + blk_slices(c.n, c.S - 1);
            ok = bounded_wait_geq(&c.cnt_b[s * TPB + i], need, status);
        } else ok = bounded_wait_geq(&c.xdone[s * TPB + i], bdiag_slices(bsz, i), status);
    }
    if (kind == 2 && s == c.S - 1 && lane == 31 && ok) ok = bounded_wait_geq(c.ctl + 1, (int)c.nf, status);
    return __all_sync(0xffffffffu, ok);
}

template <class T, class LT>
__global__ void __launch_bounds__(CH_NT, 1) k_bis_chain(const __grid_constant__ CUtensorMap mapL,
                                                        const __grid_constant__ CUtensorMap mapLt,
                                                        const __grid_constant__ CUtensorMap mapD, Chain c,
                                                        T* Bv, T* Y, T* X)
{
    constexpr int NS = NSTAGE;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    T* vs = reinterpret_cast<T*>(base + NS * CHUNK);
    T* red = reinterpret_cast<T*>(base);  // after a unit's last chunk
    __shared__ __align__(8) uint64_t full[NS];
    __shared__ long long s_u;
    __shared__ int s_ok;
    int* status = c.ctl;
    int* fdone = c.ctl + 1;
    unsigned long long* head = reinterpret_cast<unsigned long long*>(c.ctl + 2);
    const int tid = threadIdx.x;
    constexpr int KCD = chunk_cols<T>();      // inverse-block columns per chunk
    constexpr int KCL = chunk_cols<LT>();  // factor columns per chunk (row units)
    constexpr int PR = pt_rows<LT>();      // factor rows per chunk (column units)
    constexpr int XQ = xq_rows<LT>();
    if (tid == 0) {
        for (int s = 0; s < NS; ++s) tc::mbar_init(&full[s], 1);
        tc::mbar_fence_init();
        tc::prefetch_tmap(&mapL);
        tc::prefetch_tmap(&mapLt);
        tc::prefetch_tmap(&mapD);
    }
    __syncthreads();
    unsigned long long seq = 0;  // chunks this CTA has consumed
    __shared__ int s_unit[4];
    Cursor cur;                  // thread 0's
    while (true) {
        if (tid == 0) {
            s_u = (long long)atomicAdd(head, 1ULL);
            if (s_u < c.total) cur.decode(c, s_u, s_unit[0], s_unit[1], s_unit[2], s_unit[3]);
        }
        __syncthreads();
        const long long u = s_u;
        if (u >= c.total) break;
        const int unit_kind = s_unit[0], s = s_unit[1], idx = s_unit[2], kq = s_unit[3];
        const bool bulk = unit_kind >= 4;  // a whole-block panel unit (kinds 4, 5 compute as 1, 3)
        const int kind = unit_kind == 4 ? 1 : (unit_kind == 5 ? 3 : unit_kind);
        const int bsz = blk_size(c.n, s);
        const long long s0 = (long long)s * BS;
        // rows (parts / tiles) and the inner range [kb, ke) of the block the unit covers
        int nch, kb = kq * KS, ke, rloc = 0;
        const T* vsrc;
        if (kind == 0) {
            rloc = idx * CT;
            ke = min(min(kb + KS, rloc + CT), bsz);
            nch = (ke - kb + KCD - 1) / KCD;
            vsrc = Bv + (s0 + kb) * CQ;
        } else if (kind == 1) {
            ke = bulk ? bsz : min(kb + KS, bsz);
            nch = (ke - kb + KCL - 1) / KCL;
            vsrc = Y + (s0 + kb) * CQ;
        } else if (kind == 2) {
            rloc = idx * CT;
            kb = max(kb, rloc);
            ke = min(kq * KS + KS, bsz);
            nch = (ke - kb + KCD - 1) / KCD;
            vsrc = Y + (s0 + kb) * CQ;
        } else {
            ke = bulk ? bsz : min(kb + KS, bsz);
            nch = (ke - kb + PR - 1) / PR;
            vsrc = X + (s0 + kb) * CQ;
        }
        auto issue = [&](int j) {
            const int st = (int)((seq + j) % NS);
            unsigned char* dst = base + st * CHUNK;
            tc::mbar_expect_tx(&full[st], CHUNK);
            if (kind == 0 || kind == 2)
                tc::tma_load_2d(dst, &mapD, &full[st], rloc, s * BS + kb + j * KCD);
            else if (kind == 1)
                tc::tma_load_2d(dst, &mapL, &full[st], idx * CT, (int)(s0 + kb + j * KCL));
            else
                tc::tma_load_2d(dst, &mapLt, &full[st], (int)(s0 + kb + j * PR), idx * CT);
        };
        auto prefetch = [&](int j) {
            if (kind == 0 || kind == 2)
                tc::tma_prefetch_l2_2d(&mapD, rloc, s * BS + kb + j * KCD);
            else if (kind == 1)
                tc::tma_prefetch_l2_2d(&mapL, idx * CT, (int)(s0 + kb + j * KCL));
            else
                tc::tma_prefetch_l2_2d(&mapLt, (int)(s0 + kb + j * PR), idx * CT);
        };
        const int npro = nch < NS ? nch : NS;
        if (tid == 0) {
            // the matrix is read-only: its chunks stream in while the unit waits for its inputs
            tc::fence_proxy_async_smem();  // the previous unit's reduction wrote the stages
            for (int j = 0; j < npro; ++j) issue(j);
            for (int j = npro; j < nch; ++j) prefetch(j);  // the rest of the unit heads for L2 now
        }
        if (tid < 32) {
            const bool ok = kind >= 0 && wait_inputs(c, kind, s, kb, ke, bsz, status);
            if (tid == 0) s_ok = ok;
        }
        __syncthreads();
        if (!s_ok) {
            // a wait gave up (status set): let the chunks in flight land (bounded), then leave
            for (int j = 0; j < npro; ++j)
                (void)tc::mbar_wait(&full[(seq + j) % NS], (uint32_t)(((seq + j) / NS) & 1), status, 0x52);
            break;
        }
        // stage the vector rows kb .. kb + nch*chunk of the block (zeros past the block): row-major
        // for the row units, q-major for the column units
        const int vavail = bsz - kb;
        if (kind != 3) {
            const int vlen = nch * (kind == 1 ? KCL : KCD);
            constexpr int PER = CQ * (int)sizeof(T) / 16;  // 16-byte pieces per row
            const float4* src = reinterpret_cast<const float4*>(vsrc);
            float4* dst = reinterpret_cast<float4*>(vs);
#pragma unroll 4
            for (int e = tid; e < vlen * PER; e += CH_NT)
                dst[e] = (e / PER) < vavail ? __ldcg(src + e) : make_float4(0.f, 0.f, 0.f, 0.f);
        } else {
            constexpr int QP = 16 / (int)sizeof(T);  // right-hand sides per 16-byte piece
            const int vlen = nch * PR;
            const float4* src = reinterpret_cast<const float4*>(vsrc);
            for (int e = tid; e < vlen * (CQ / QP); e += CH_NT) {
                const int row = e / (CQ / QP), q0 = (e % (CQ / QP)) * QP;
                const float4 v = row < vavail ? __ldcg(src + e) : make_float4(0.f, 0.f, 0.f, 0.f);
                const T* pv = reinterpret_cast<const T*>(&v);
#pragma unroll
                for (int i = 0; i < QP; ++i) vs[(q0 + i) * XQ + row] = pv[i];
            }
        }
        __syncthreads();
        T acc[4][CQ];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int q = 0; q < CQ; ++q) acc[a][q] = T(0);
        const int g = tid & 15, ks = tid >> 4;
        bool ok = true;
        int j = 0;
        for (; j < nch; ++j) {
            const int st = (int)((seq + j) % NS);
            const uint32_t par = (uint32_t)(((seq + j) / NS) & 1);
            ok = __syncthreads_and(tc::mbar_wait(&full[st], par, status, 0x51));
            if (!ok) break;
            const unsigned char* tile = base + st * CHUNK;
            if (kind == 0)
                row_chunk<T, T, 1>(reinterpret_cast<const T*>(tile), vs, j, kb, ke, rloc, g, ks, acc);
            else if (kind == 1)
                row_chunk<T, LT, 0>(reinterpret_cast<const LT*>(tile), vs, j, kb, ke, rloc, g, ks, acc);
            else if (kind == 2)
                row_chunk<T, T, 2>(reinterpret_cast<const T*>(tile), vs, j, kb, ke, rloc, g, ks, acc);
            else
                col_chunk<T, LT>(reinterpret_cast<const LT*>(tile), vs, j, acc);
            __syncthreads();  // stage consumed by every thread
            if (tid == 0 && j + NS < nch) issue(j + NS);
        }
        if (!ok) {
            // an arrival wait gave up: wait (bounded) for the chunks still in flight, then leave
            for (int jj = j; jj < nch && jj < j + NS; ++jj)
                (void)tc::mbar_wait(&full[(seq + jj) % NS], (uint32_t)(((seq + jj) / NS) & 1), status, 0x52);
            break;
        }
        seq += nch;
        // reduce to the unit's 512 outputs: (row or column e >> 3, right-hand side e & 7)
        const int w = tid >> 5, lane = tid & 31;
        T o = T(0);
        if (kind != 3) {
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int q = 0; q < CQ; ++q) acc[a][q] += __shfl_xor_sync(0xffffffffu, acc[a][q], 16);
            if (lane < 16)
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int q = 0; q < CQ; ++q) red[(w * CT + 4 * g + a) * CQ + q] = acc[a][q];
            __syncthreads();
#pragma unroll
            for (int ww = 0; ww < CH_NT / 32; ++ww) o += red[ww * CT * CQ + tid];
        } else {
            const int q = ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) {
                const T sum = warp_sum8<T>(acc[cc]);
                if ((lane & 3) == 0) red[(4 * w + cc) * CQ + q] = sum;
            }
            __syncthreads();
            o = red[tid];
        }
        const int r = tid >> 3;
        if (kind == 0) {
            if (rloc + r < bsz) atomicAdd(&Y[(s0 + rloc) * CQ + tid], o);
        } else if (kind == 1) {
            if ((long long)idx * CT + r < c.n) atomicAdd(&Bv[(long long)idx * CT * CQ + tid], -o);
        } else if (kind == 2) {
            if (rloc + r < bsz) atomicAdd(&X[(s0 + rloc) * CQ + tid], o);
        } else {
            atomicAdd(&Y[(long long)idx * CT * CQ + tid], -o);
        }
        __syncthreads();  // every update of the unit issued; vs / red free
        if (tid == 0) {
            // release: the unit's updates (ordered before by the barrier) precede the count
            const int applied = bulk ? blk_slices(c.n, s) : 1;  // a bulk unit counts as all slices of its phase
            if (kind == 0) red_release_add(&c.ydone[s * TPB + idx], 1);
            else if (kind == 1) red_release_add(&c.cnt_f[idx], applied);
            else if (kind == 2) red_release_add(&c.xdone[s * TPB + idx], 1);
            else red_release_add(&c.cnt_b[idx], applied);
            if (kind <= 1) red_release_add(fdone, 1);
        }
    }
}

// Bv(i, q) = B(i, q) for q < nr, 0 beyond (row-major, CQ per row)
template <class T>
__global__ void k_bis_pack(int n, int nr, const double* __restrict__ B, long long ldb, T* __restrict__ Bv)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)n * CQ;
         e += (long long)gridDim.x * blockDim.x) {
        const long long i = e / CQ;
        const int q = (int)(e % CQ);
        Bv[e] = q < nr ? (T)B[i + q * ldb] : T(0);
    }
}

// B(i, q) = Bv(i, q), or NaN when a wait of the chain gave up
template <class T>
__global__ void k_bis_unpack(int n, int nr, const T* __restrict__ Bv, double* __restrict__ B, long long ldb,
                             const int* __restrict__ status)
{
    const bool bad = *status != DDLAK_OK;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)n * nr;
         e += (long long)gridDim.x * blockDim.x) {
        const long long i = e % n;
        const int q = (int)(e / n);
        B[i + q * ldb] = bad ? __longlong_as_double(0x7ff8000000000000LL) : (double)__ldcg(Bv + i * CQ + q);
    }
}

struct ChainLayout {
    int S, Tt;
    long long nf, nb;
    size_t flag_bytes, vec_bytes;
};

ChainLayout chain_layout(int n, size_t elem)
{
    ChainLayout l{};
    l.S = (int)ceil_div(n, BS);
    l.Tt = (int)ceil_div(n, CT);
    for (int g = 0; g < l.S; ++g) {
        l.nf += group_units(n, l.S, l.Tt, true, g);
        l.nb += group_units(n, l.S, l.Tt, false, g);
    }
    l.flag_bytes = ((size_t)(64 + 2 * l.Tt + 2 * l.S * TPB) * sizeof(int) + 255) / 256 * 256;
    l.vec_bytes = ((size_t)n * CQ * elem + 255) / 256 * 256;
    return l;
}

// workspace: [flags][Y][X][Bv]; the flags, Y and X start at zero
template <class T, class LT>
cudaError_t bis_chain_solve(int n, int nrhs, const LT* L, long long ldl, const T* Dinv, double* B, long long ldb,
                            void* work, cudaStream_t st)
{
    if (n > (1 << 30) / 2) return cudaErrorInvalidValue;  // TMA coordinates are 32-bit
    const ChainLayout lay = chain_layout(n, sizeof(T));
    char* w = static_cast<char*>(work);
    int* ctl = reinterpret_cast<int*>(w);
    T* Yv = reinterpret_cast<T*>(w + lay.flag_bytes);
    T* Xv = reinterpret_cast<T*>(w + lay.flag_bytes + lay.vec_bytes);
    T* Bv = reinterpret_cast<T*>(w + lay.flag_bytes + 2 * lay.vec_bytes);
    Chain c{};
    c.n = n;
    c.S = lay.S;
    c.Tt = lay.Tt;
    c.nf = lay.nf;
    c.total = lay.nf + lay.nb;
    c.ldl = ldl;
    c.ctl = ctl;
    c.cnt_f = ctl + 64;
    c.ydone = c.cnt_f + lay.Tt;
    c.cnt_b = c.ydone + lay.S * TPB;
    c.xdone = c.cnt_b + lay.Tt;
    const size_t smem = chain_smem<T>();
    CUtensorMap mapL, mapLt, mapD;
    const CUtensorMapDataType dt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    const CUtensorMapDataType lt = sizeof(LT) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    if (!tc::encode_colmajor_2d(&mapL, lt, (int)sizeof(LT), L, n, n, ldl, CT, chunk_cols<LT>(),
                                CU_TENSOR_MAP_SWIZZLE_NONE) ||
        !tc::encode_colmajor_2d(&mapLt, lt, (int)sizeof(LT), L, n, n, ldl, pt_rows<LT>(), CT,
                                CU_TENSOR_MAP_SWIZZLE_NONE) ||
        !tc::encode_colmajor_2d(&mapD, dt, (int)sizeof(T), Dinv, BS, (long long)lay.S * BS, BS, CT, chunk_cols<T>(),
                                CU_TENSOR_MAP_SWIZZLE_NONE))
        return cudaErrorInvalidValue;
    if (cudaError_t e = smem_optin(k_bis_chain<T, LT>, smem); e != cudaSuccess) return e;
    // every CTA of the queue resident at once: SMs of this device x CTAs per SM
    int grid = 0;
    {
        int dev = 0, sms = 148, per = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_bis_chain<T, LT>, CH_NT, smem);
        grid = sms * (per > 0 ? per : 1);
    }
    const unsigned g = (unsigned)std::min<long long>(grid, c.total);
    const unsigned gv = (unsigned)std::min<long long>(ceil_div((long long)n * CQ, 256), 1184);
    int launches = 0;
    for (int r0 = 0; r0 < nrhs; r0 += CQ) {
        const int nr = std::min(CQ, nrhs - r0);
        cudaError_t e = cudaMemsetAsync(ctl, 0, lay.flag_bytes + 2 * lay.vec_bytes, st);
        if (e != cudaSuccess) return e;
        k_bis_pack<T><<<gv, 256, 0, st>>>(n, nr, B + r0 * ldb, ldb, Bv);
        k_bis_chain<T, LT><<<g, CH_NT, smem, st>>>(mapL, mapLt, mapD, c, Bv, Yv, Xv);
        k_bis_unpack<T><<<gv, 256, 0, st>>>(n, nr, Xv, B + r0 * ldb, ldb, ctl);
        launches += 3;
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
        k_bis_widen<float><<<grid, block, 0, st>>>(n, static_cast<const float*>(L32), ldl, static_cast<double*>(tmp));
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

extern "C" int ddlak_bis_inverse_f64(int n, const void* L, long long ldl, void* Dinv, void* stream)
{
    using namespace ddlak;
    if (n <= 0) return 0;
    if (!L || !Dinv || ldl < n) return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the inverses straight from the factor's diagonal blocks (the batched inversion reads only
    // their lower triangles): block s starts at L + s BS (ldl + 1)
    const double* Ld = static_cast<const double*>(L);
    double* D = static_cast<double*>(Dinv);
    const long long bb = (long long)BS * BS, lstride = (long long)BS * (ldl + 1);
    const int full = n / BS, last = n - full * BS;
    int r = 0;
    if (full > 0) r = ddlak_trtri_batched('d', full, BS, Ld, ldl, lstride, D, BS, bb, stream);
    if (r == 0 && last > 0)
        r = ddlak_trtri_batched('d', 1, last, Ld + (long long)full * lstride, ldl, lstride, D + full * bb, BS, bb,
                                stream);
    if (r != 0) return r;
    const int S = (int)ceil_div(n, BS);
    dim3 grid(BS / 32, BS / 32, S), block(32, 32);
    k_bis_mirror<<<grid, block, 0, st>>>(D);
    note_launches(1);
    return (int)cudaGetLastError();
}

extern "C" int ddlak_bis_inverse_narrow(int n, const void* Dinv, void* Dinv32, void* stream)
{
    using namespace ddlak;
    if (n <= 0) return 0;
    if (!Dinv || !Dinv32) return (int)cudaErrorInvalidValue;
    const long long count = (long long)ceil_div(n, BS) * BS * BS;
    k_bis_narrow<<<1184, 256, 0, static_cast<cudaStream_t>(stream)>>>(count, static_cast<const double*>(Dinv),
                                                                      static_cast<float*>(Dinv32));
    note_launches(1);
    return (int)cudaGetLastError();
}

// The solve's queue as the kernel walks it, for checking on the host: the unit
// counts of both directions and the decode of one unit.
extern "C" int ddlak_bis_queue_size(int n, long long* forward_units, long long* total_units)
{
    using namespace ddlak;
    if (n <= 0 || !forward_units || !total_units) return (int)cudaErrorInvalidValue;
    const ChainLayout l = chain_layout(n, sizeof(float));
    *forward_units = l.nf;
    *total_units = l.nf + l.nb;
    return 0;
}

extern "C" int ddlak_bis_queue_unit(int n, long long u, int* kind, int* phase, int* index, int* slice)
{
    using namespace ddlak;
    if (n <= 0 || !kind || !phase || !index || !slice) return (int)cudaErrorInvalidValue;
    const ChainLayout l = chain_layout(n, sizeof(float));
    if (u < 0 || u >= l.nf + l.nb) return (int)cudaErrorInvalidValue;
    Chain c{};
    c.n = n;
    c.S = l.S;
    c.Tt = l.Tt;
    c.nf = l.nf;
    c.total = l.nf + l.nb;
    decode_unit(c, u, *kind, *phase, *index, *slice);
    return 0;
}

extern "C" unsigned long long ddlak_bis_solve_workspace(int n, int nrhs)
{
    using namespace ddlak;
    (void)nrhs;
    if (n <= 0) return 256;
    const ChainLayout l = chain_layout(n, sizeof(double));
    return l.flag_bytes + 3 * l.vec_bytes;
}

namespace {
int bis_check(int n, int nrhs, const void* L32, long long ldl, const void* Dinv, const void* B, long long ldb,
              unsigned long long work_bytes)
{
    if (nrhs > 16 || !L32 || !Dinv || !B || ldb < n || ldl < n || (ldl & 3) ||
        (reinterpret_cast<uintptr_t>(L32) & 15) || (reinterpret_cast<uintptr_t>(Dinv) & 15) ||
        work_bytes < ddlak_bis_solve_workspace(n, nrhs))
        return (int)cudaErrorInvalidValue;
    return 0;
}
}  // namespace

extern "C" int ddlak_bis_solve(int n, int nrhs, const void* L32, long long ldl, const void* Dinv, void* B,
                               long long ldb, void* work, unsigned long long work_bytes, void* stream)
{
    using namespace ddlak;
    if (n <= 0 || nrhs <= 0) return 0;
    if (int r = bis_check(n, nrhs, L32, ldl, Dinv, B, ldb, work_bytes)) return r;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const double nd = n, rd = nrhs;
    ProfScope ps(PK_POTRS_FUSED, st, 2.0 * nd * nd * rd, 4.0 * nd * (nd + 1));
    return (int)bis_chain_solve<double, float>(n, nrhs, static_cast<const float*>(L32), ldl, static_cast<const double*>(Dinv),
                                        static_cast<double*>(B), ldb, work, st);
}

extern "C" int ddlak_bis_solve_f64(int n, int nrhs, const void* L, long long ldl, const void* Dinv, void* B,
                                   long long ldb, void* work, unsigned long long work_bytes, void* stream)
{
    using namespace ddlak;
    if (n <= 0 || nrhs <= 0) return 0;
    if (nrhs > 16 || !L || !Dinv || !B || ldb < n || ldl < n || (ldl & 1) || (reinterpret_cast<uintptr_t>(L) & 15) ||
        (reinterpret_cast<uintptr_t>(Dinv) & 15) || work_bytes < ddlak_bis_solve_workspace(n, nrhs))
        return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const double nd = n, rd = nrhs;
    ProfScope ps(PK_POTRS_FUSED, st, 2.0 * nd * nd * rd, 8.0 * nd * (nd + 1));
    return (int)bis_chain_solve<double, double>(n, nrhs, static_cast<const double*>(L), ldl,
                                                static_cast<const double*>(Dinv), static_cast<double*>(B), ldb, work,
                                                st);
}

extern "C" int ddlak_bis_solve_f32(int n, int nrhs, const void* L32, long long ldl, const void* Dinv32, void* B,
                                   long long ldb, void* work, unsigned long long work_bytes, void* stream)
{
    using namespace ddlak;
    if (n <= 0 || nrhs <= 0) return 0;
    if (int r = bis_check(n, nrhs, L32, ldl, Dinv32, B, ldb, work_bytes)) return r;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const double nd = n, rd = nrhs;
    ProfScope ps(PK_POTRS_FUSED, st, 2.0 * nd * nd * rd, 4.0 * nd * (nd + 1));
    return (int)bis_chain_solve<float, float>(n, nrhs, static_cast<const float*>(L32), ldl, static_cast<const float*>(Dinv32),
                                       static_cast<double*>(B), ldb, work, st);
}
