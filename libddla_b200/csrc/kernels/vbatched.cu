// Batched uneven Cholesky: factor, solve and log-determinant of thousands of
// independent Hermitian positive-definite matrices of different orders in ONE
// persistent launch (no reference counterpart; the per-matrix equivalent is
// ppotrf + ppotrs + diag_logdet, src/Cholesky/ppotrf.cpp:326-349,
// ppotrs.cpp:65-85, diag_logdet.cpp:42-55).
//
// Scheduling: grid = SMs x resident CTAs.  Each CTA takes the next matrix from
// a device work list (sorted by decreasing order, so the largest start first:
// longest-processing-time order) with one atomicAdd, processes it alone, and
// takes the next.  The last CTA to leave resets the two counters, so the same
// launch can be replayed (it is captured in a CUDA graph by the host).
//
// Per matrix (order n <= NMAX, lower storage, lda >= n), 256 threads:
//   left-looking blocked Cholesky with block columns of width W (a tuned
//   choice per matrix, see ddlak_vbatched_variants).  For block column J the
//   threads hold its rows in registers (thread t owns rows t, t+256, ...),
//   subtract L(J:n, 0:J) L(J:J+W, 0:J)^H streamed through shared memory in
//   chunks of KC columns with cp.async double buffering, then warp 0 factors
//   the W x W diagonal block with shuffles, every thread solves its own rows
//   against it (X L11^H = C), and the block column is stored.  The right-hand
//   side lives in shared memory: its forward substitution rides along with
//   the factorization (warp 0 solves the diagonal part, the other rows are
//   updated from the registers that already hold L), the backward one runs
//   after it in steps of 32 rows.  log det A = 2 sum log l_jj in FP64.
// info follows LAPACK ?potrf (order of the first non-positive leading minor);
// a failed matrix keeps its right-hand side and gets logdet NaN.
#include <cuda_runtime.h>

#include <ddla_kernels.h>

#include "common.cuh"
#include "profile.h"

namespace ddlak {
namespace {

constexpr int VB_NT = 256;  // threads per CTA
constexpr int VB_KC = 8;    // columns per streamed chunk
constexpr int VB_BW = 32;   // rows per backward-substitution step
constexpr int VB_MAXW = 32;

// the two block-column widths a launch can use per matrix (registers: rows per
// thread x width values of the block column)
template <class T, int NMAX> struct VbWidths { static constexpr int w0 = 8, w1 = 16; };
template <> struct VbWidths<float, 512> { static constexpr int w0 = 16, w1 = 32; };

template <class T>
__device__ __forceinline__ T wshfl(T v, int src)
{
    return __shfl_sync(0xffffffffu, v, src);
}

template <class T, int NMAX>
struct VbSmem {
    static constexpr int LDS = NMAX;
    static constexpr size_t chunk_elems = (size_t)2 * VB_KC * LDS;
    static constexpr size_t bytes = sizeof(T) * (chunk_elems + NMAX + VB_MAXW * (VB_MAXW + 1) + VB_BW) +
                                    sizeof(T) * NMAX /* 1/l_jj */;
};

template <class T, int NMAX, int W>
__device__ void vb_matrix(int n, T* __restrict__ A, long long lda, T* __restrict__ b, double* logdet_out,
                          int* info_out, unsigned char* smem, int* s_flag, double* s_red)
{
    constexpr int RPT = NMAX / VB_NT;
    constexpr int LDS = VbSmem<T, NMAX>::LDS;
    constexpr int LW = W + 1;
    static_assert(W % VB_KC == 0 && W <= VB_MAXW && NMAX % VB_NT == 0, "block shape");
    T* Ls = reinterpret_cast<T*>(smem);
    T* bs = Ls + VbSmem<T, NMAX>::chunk_elems;
    T* L11 = bs + NMAX;
    T* st = L11 + VB_MAXW * (VB_MAXW + 1);
    T* rinv = st + VB_BW;

    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const bool solve = b != nullptr;
    if (solve)
        for (int i = t; i < n; i += VB_NT) bs[i] = b[i];
    double lsum = 0.0;  // warp 0: sum of log l_jj over the pivots this lane produced
    int info = 0;

    for (int J = 0; J < n; J += W) {
        const int nw = min(W, n - J), mJ = n - J;
        T c[RPT][W];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = t + r * VB_NT;
#pragma unroll
            for (int q = 0; q < W; ++q)
                c[r][q] = (i < mJ && q < nw && q <= i) ? A[(J + i) + (long long)(J + q) * lda] : T(0);
        }
        // c -= L(J:n, 0:J) * L(J:J+W, 0:J)^H, streamed in chunks of VB_KC columns
        const int nch = J / VB_KC;
        auto stage = [&](int ch, int buf) {
            T* dst = Ls + (size_t)buf * VB_KC * LDS;
            const int k0 = ch * VB_KC;
#pragma unroll
            for (int kk = 0; kk < VB_KC; ++kk) {
                const T* src = A + J + (long long)(k0 + kk) * lda;
#pragma unroll
                for (int r = 0; r < RPT; ++r) {
                    const int i = t + r * VB_NT;
                    if (i < mJ) cp_async_elem<sizeof(T)>(dst + kk * LDS + i, src + i, true);
                }
            }
        };
        if (nch > 0) stage(0, 0);
        cp_group_commit();
        for (int ch = 0; ch < nch; ++ch) {
            if (ch + 1 < nch) stage(ch + 1, (ch + 1) & 1);
            cp_group_commit();
            cp_group_wait<1>();
            __syncthreads();
            const T* src = Ls + (size_t)(ch & 1) * VB_KC * LDS;
            // a warp whose rows of set r all lie past the block column's last row skips them
            bool live[RPT];
#pragma unroll
            for (int r = 0; r < RPT; ++r) live[r] = (t - lane) + r * VB_NT < mJ;
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                if (!live[r]) continue;
#pragma unroll
                for (int kk = 0; kk < VB_KC; ++kk) {
                    const T li = src[kk * LDS + t + r * VB_NT];
#pragma unroll
                    for (int q = 0; q < W; ++q) c[r][q] = fms(c[r][q], li, src[kk * LDS + q]);
                }
            }
            __syncthreads();
        }
        cp_group_wait<0>();

        // Warp 0 holds rows 0..31 of the block column in c[0]: the diagonal block
        // (lanes < nw) and, for W < 32, the first rows below it.  Right-looking
        // elimination across the lanes factors the former and solves the latter.
        if (warp == 0) {
            int fail = 0;
            T rv = T(0);
#pragma unroll
            for (int j = 0; j < W; ++j) {
                if (j < nw && !fail) {
                    const T d = wshfl(c[0][j], j);
                    if (!(d > T(0))) {
                        fail = j + 1;
                    } else {
                        const T l = sqrt(d), inv = T(1) / l;
                        if (lane == j) {
                            c[0][j] = l;
                            rv = inv;
                            lsum += log((double)l);
                        } else if (lane > j) {
                            c[0][j] *= inv;
                        }
#pragma unroll
                        for (int q = j + 1; q < W; ++q) {
                            const T lqj = wshfl(c[0][j], q);
                            if (lane >= q) c[0][q] = fms(c[0][q], c[0][j], lqj);
                        }
                    }
                }
            }
            if (!fail && solve) {
                T v = lane < nw ? bs[J + lane] : T(0);
#pragma unroll
                for (int j = 0; j < W; ++j) {
                    if (j < nw) {
                        if (lane == j) v *= rv;
                        const T y = wshfl(v, j);
                        if (lane > j && lane < nw) v = fms(v, c[0][j], y);
                    }
                }
                if (lane < nw) bs[J + lane] = v;
            }
            // the columns before a failed pivot are final (LAPACK ?potf2 leaves them)
            const int good = fail ? fail - 1 : nw;
            if (lane < good) {
#pragma unroll
                for (int q = 0; q < W; ++q)
                    if (q <= lane) L11[lane * LW + q] = c[0][q];
                rinv[J + lane] = rv;
            }
            if (lane == 0) s_flag[0] = fail ? J + fail : 0;
        }
        __syncthreads();
        info = s_flag[0];
        // columns of this block column to finish and store: all, or those before the failure
        const int good = info ? info - 1 - J : nw;

        // rows below the diagonal block: X L11^H = C (rows of warp 0's c[0] are
        // already solved), then the forward-solve update of b
        bool act[RPT];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = t + r * VB_NT;
            act[r] = i >= good && i < mJ && !(r == 0 && warp == 0);
        }
#pragma unroll
        for (int q = 0; q < W; ++q) {
            if (q < good) {
                T s[RPT];
#pragma unroll
                for (int r = 0; r < RPT; ++r) s[r] = c[r][q];
#pragma unroll
                for (int p = 0; p < q; ++p) {
                    const T l = L11[q * LW + p];
#pragma unroll
                    for (int r = 0; r < RPT; ++r) s[r] = fms(s[r], c[r][p], l);
                }
                const T ri = rinv[J + q];
#pragma unroll
                for (int r = 0; r < RPT; ++r)
                    if (act[r]) c[r][q] = s[r] * ri;
            }
        }
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = t + r * VB_NT;
            if (i >= good && i < mJ) {
                T* dst = A + (J + i);
#pragma unroll
                for (int q = 0; q < W; ++q)
                    if (q < good) dst[(long long)(J + q) * lda] = c[r][q];
                if (solve && !info) {
                    T s = bs[J + i];
#pragma unroll
                    for (int q = 0; q < W; ++q)
                        if (q < nw) s = fms(s, c[r][q], bs[J + q]);
                    bs[J + i] = s;
                }
            } else if (r == 0 && i < good) {
                T* dst = A + (J + i);
#pragma unroll
                for (int q = 0; q < W; ++q)
                    if (q <= i) dst[(long long)(J + q) * lda] = L11[i * LW + q];
            }
        }
        __syncthreads();
        if (info) break;
    }

    if (warp == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
        if (lane == 0) s_red[0] = lsum;
    }
    if (solve && info == 0) {
        // backward substitution L^H x = y, VB_BW rows per step from the bottom
        for (int J = ((n - 1) / VB_BW) * VB_BW; J >= 0; J -= VB_BW) {
            const int nw = min(VB_BW, n - J);
            for (int q = warp; q < nw; q += VB_NT / 32) {
                const T* col = A + (long long)(J + q) * lda;
                T acc = T(0);
                for (int i = J + nw + lane; i < n; i += 32) acc = fma_(acc, col[i], bs[i]);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
                if (lane == 0) st[q] = acc;
            }
            __syncthreads();
            if (warp == 0) {
                T v = lane < nw ? bs[J + lane] - st[lane] : T(0);
                const T* col = A + (long long)(J + lane) * lda;  // column J+lane of L
                T lc[VB_BW];
#pragma unroll
                for (int j = 0; j < VB_BW; ++j) lc[j] = (lane < nw && j > lane && j < nw) ? col[J + j] : T(0);
#pragma unroll
                for (int j = VB_BW - 1; j >= 0; --j) {
                    if (j < nw) {
                        if (lane == j) v *= rinv[J + j];
                        const T xj = wshfl(v, j);
                        if (lane < j) v = fms(v, lc[j], xj);
                    }
                }
                if (lane < nw) bs[J + lane] = v;
            }
            __syncthreads();
        }
        for (int i = t; i < n; i += VB_NT) b[i] = bs[i];
    }
    __syncthreads();
    if (t == 0) {
        *info_out = info;
        *logdet_out = info ? __longlong_as_double(0x7ff8000000000000LL) : 2.0 * s_red[0];
    }
    __syncthreads();
}

template <class T, int NMAX>
__global__ void __launch_bounds__(VB_NT, NMAX <= 512 ? 2 : 1)
    k_posv_vbatched(int batch, const int* __restrict__ d_n, T* const* __restrict__ d_A, const int* __restrict__ d_lda,
                    T* const* __restrict__ d_B, double* __restrict__ d_logdet, int* __restrict__ d_info,
                    const int* __restrict__ order, const unsigned char* __restrict__ wsel, int* counters)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_m;
    __shared__ int s_flag[2];
    __shared__ double s_red[2];
    for (;;) {
        if (threadIdx.x == 0) s_m = atomicAdd(&counters[0], 1);
        __syncthreads();
        const int m = s_m;
        __syncthreads();
        if (m >= batch) break;
        const int id = order ? order[m] : m;
        const int n = d_n[id];
        if (n <= 0 || n > NMAX || d_lda[id] < n) {
            if (threadIdx.x == 0) {
                d_info[id] = n == 0 ? 0 : -1;
                d_logdet[id] = n == 0 ? 0.0 : __longlong_as_double(0x7ff8000000000000LL);
            }
            continue;
        }
        T* A = d_A[id];
        T* B = d_B ? d_B[id] : nullptr;
        const long long lda = d_lda[id];
        if (wsel && wsel[id])
            vb_matrix<T, NMAX, VbWidths<T, NMAX>::w1>(n, A, lda, B, d_logdet + id, d_info + id, smem_raw, s_flag, s_red);
        else
            vb_matrix<T, NMAX, VbWidths<T, NMAX>::w0>(n, A, lda, B, d_logdet + id, d_info + id, smem_raw, s_flag, s_red);
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&counters[1], 1) == (int)gridDim.x - 1) {
            atomicExch(&counters[0], 0);
            atomicExch(&counters[1], 0);
            __threadfence();
        }
    }
}

// A well-conditioned SPD stand-in for the autotuner: n on the diagonal,
// 1/(1+|i-j|) off it (diagonally dominant for n >= 16).
template <class T>
__global__ void k_fill_spd(int batch, const int* __restrict__ d_n, T* const* __restrict__ d_A,
                           const int* __restrict__ d_lda, T* const* __restrict__ d_B)
{
    const int id = blockIdx.x;
    if (id >= batch) return;
    const int n = d_n[id];
    const long long lda = d_lda[id];
    T* A = d_A[id];
    for (long long e = threadIdx.x; e < (long long)n * n; e += blockDim.x) {
        const int i = (int)(e % n), j = (int)(e / n);
        A[i + j * lda] = i == j ? T(n) : T(1) / T(1 + abs(i - j));
    }
    if (d_B && d_B[id])
        for (int i = threadIdx.x; i < n; i += blockDim.x) d_B[id][i] = T(1);
}

template <class T, int NMAX>
cudaError_t vb_launch(int batch, const int* d_n, void* const* d_A, const int* d_lda, void* const* d_B,
                      double* d_logdet, int* d_info, const int* order, const unsigned char* wsel, int* counters,
                      int grid, cudaStream_t st)
{
    constexpr size_t smem = VbSmem<T, NMAX>::bytes;
    if (cudaError_t e = smem_optin(k_posv_vbatched<T, NMAX>, smem); e != cudaSuccess) return e;
    k_posv_vbatched<T, NMAX><<<grid, VB_NT, smem, st>>>(batch, d_n, reinterpret_cast<T* const*>(d_A), d_lda,
                                                        reinterpret_cast<T* const*>(d_B), d_logdet, d_info, order,
                                                        wsel, counters);
    note_launches(1);
    return cudaGetLastError();
}

template <class T, int NMAX>
int vb_max_grid()
{
    constexpr size_t smem = VbSmem<T, NMAX>::bytes;
    if (smem_optin(k_posv_vbatched<T, NMAX>, smem) != cudaSuccess) return 0;
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_posv_vbatched<T, NMAX>, VB_NT, smem) != cudaSuccess)
        return 0;
    return sms * per;
}

}  // namespace
}  // namespace ddlak

extern "C" int ddlak_vbatched_variants(char type, int nmax, int* widths)
{
    if (nmax != 512 && nmax != 1024) return (int)cudaErrorInvalidValue;
    using namespace ddlak;
    if (type == 'd' && nmax == 512) { widths[0] = VbWidths<double, 512>::w0; widths[1] = VbWidths<double, 512>::w1; }
    else if (type == 'd') { widths[0] = VbWidths<double, 1024>::w0; widths[1] = VbWidths<double, 1024>::w1; }
    else if (type == 's' && nmax == 512) { widths[0] = VbWidths<float, 512>::w0; widths[1] = VbWidths<float, 512>::w1; }
    else if (type == 's') { widths[0] = VbWidths<float, 1024>::w0; widths[1] = VbWidths<float, 1024>::w1; }
    else return (int)cudaErrorInvalidValue;
    return 0;
}

extern "C" int ddlak_vbatched_max_grid(char type, int nmax)
{
    using namespace ddlak;
    if (type == 'd') return nmax == 512 ? vb_max_grid<double, 512>() : nmax == 1024 ? vb_max_grid<double, 1024>() : 0;
    if (type == 's') return nmax == 512 ? vb_max_grid<float, 512>() : nmax == 1024 ? vb_max_grid<float, 1024>() : 0;
    return 0;
}

extern "C" int ddlak_posv_vbatched(char type, int nmax, int batch, const int* d_n, void* const* d_A,
                                   const int* d_lda, void* const* d_B, double* d_logdet, int* d_info,
                                   const int* d_order, const unsigned char* d_wsel, int* d_counters, int grid,
                                   void* stream)
{
    using namespace ddlak;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (batch <= 0) return 0;
    if (grid <= 0 || !d_n || !d_A || !d_lda || !d_logdet || !d_info || !d_counters) return (int)cudaErrorInvalidValue;
    ProfScope ps(PK_BATCHED, st, 0.0, 0.0);
    if (type == 'd') {
        if (nmax == 512)
            return (int)vb_launch<double, 512>(batch, d_n, d_A, d_lda, d_B, d_logdet, d_info, d_order, d_wsel,
                                               d_counters, grid, st);
        if (nmax == 1024)
            return (int)vb_launch<double, 1024>(batch, d_n, d_A, d_lda, d_B, d_logdet, d_info, d_order, d_wsel,
                                                d_counters, grid, st);
    } else if (type == 's') {
        if (nmax == 512)
            return (int)vb_launch<float, 512>(batch, d_n, d_A, d_lda, d_B, d_logdet, d_info, d_order, d_wsel,
                                              d_counters, grid, st);
        if (nmax == 1024)
            return (int)vb_launch<float, 1024>(batch, d_n, d_A, d_lda, d_B, d_logdet, d_info, d_order, d_wsel,
                                               d_counters, grid, st);
    }
    return (int)cudaErrorInvalidValue;
}

extern "C" int ddlak_fill_spd_vbatched(char type, int batch, const int* d_n, void* const* d_A, const int* d_lda,
                                       void* const* d_B, void* stream)
{
    using namespace ddlak;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (batch <= 0) return 0;
    if (type == 'd')
        k_fill_spd<double><<<batch, 256, 0, st>>>(batch, d_n, reinterpret_cast<double* const*>(d_A), d_lda,
                                                  reinterpret_cast<double* const*>(d_B));
    else if (type == 's')
        k_fill_spd<float><<<batch, 256, 0, st>>>(batch, d_n, reinterpret_cast<float* const*>(d_A), d_lda,
                                                 reinterpret_cast<float* const*>(d_B));
    else
        return (int)cudaErrorInvalidValue;
    note_launches(1);
    return (int)cudaGetLastError();
}
