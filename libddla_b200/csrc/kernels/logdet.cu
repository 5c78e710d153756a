// Log of the diagonal product, ddla::diag_logdet on a 1x1 grid.
//
// Per-entry term and join follow the reference's DiagLogTerm / DiagLogJoin
// (src/diag_logdet_impl.h:42-94): for an entry x + iy, widened to double,
//   nonfinite             -> flag 1
//   |x| = |y| = 0         -> flag 2 (zero)
//   otherwise magnitude = log(hi) + 0.5*log1p((lo/hi)^2), hi/lo = max/min(|x|,|y|)
//             phase     = atan2(y, x) if y != 0, else 0 with flag 4 when x < 0
// joined by summing magnitude and phase, OR-ing flags 1|2 and XOR-ing the
// negative-real parity 4.  The reference reduces with thrust::transform_reduce
// on the handle stream (src/diag_logdet_kernels.cpp:13-25); here a grid-stride
// pass writes one partial per CTA and a single CTA folds the partials in a
// fixed order, so the result is deterministic run to run.
#include "common.cuh"
#include "profile.h"

namespace ddlak {

struct LogState {
    double mag;
    double phase;
    int flags;
    int pad;
};

__device__ __forceinline__ LogState join(LogState a, LogState b)
{
    LogState r;
    r.mag = a.mag + b.mag;
    r.phase = a.phase + b.phase;
    r.flags = ((a.flags | b.flags) & 3) | ((a.flags ^ b.flags) & 4);
    r.pad = 0;
    return r;
}

// Which local entry holds global diagonal entry g of a block-cyclic matrix, as
// the reference's DiagLogTerm maps it (src/diag_logdet_impl.h:55-74): items
// walk this rank's local rows (pr >= pc) or local columns, item -> global
// index g -> (local row, local column); entries whose row or column this rank
// does not own contribute nothing.  A 1x1 grid maps item i to (i, i).
struct GridLayout {
    int n, mb, nb, pr, pc, row, col, rsrc, csrc;
    bool along_rows;
};

template <class T>
__device__ __forceinline__ LogState term_at(const T* A, long long index);

template <class T>
__device__ __forceinline__ LogState term_grid(const T* A, long long lda, const GridLayout& L, long long item)
{
    const int block = L.along_rows ? L.mb : L.nb;
    const int peers = L.along_rows ? L.pr : L.pc;
    const int coord = L.along_rows ? L.row : L.col;
    const int src = L.along_rows ? L.rsrc : L.csrc;
    const int offset = (coord - src + peers) % peers;
    const long long g = (item / block * peers + offset) * block + item % block;
    if (g >= L.n || (L.rsrc + g / L.mb) % L.pr != L.row || (L.csrc + g / L.nb) % L.pc != L.col)
        return LogState{0.0, 0.0, 0, 0};
    const long long lr = g / ((long long)L.mb * L.pr) * L.mb + g % L.mb;
    const long long lc = g / ((long long)L.nb * L.pc) * L.nb + g % L.nb;
    return term_at<T>(A, lr + lc * lda);
}

template <class T>
__device__ __forceinline__ LogState term(const T* A, long long lda, long long i)
{
    return term_at<T>(A, i + i * lda);
}

template <class T>
__device__ __forceinline__ LogState term_at(const T* A, long long index)
{
    using R = real_t<T>;
    const R* d = reinterpret_cast<const R*>(A + index);
    const double x = (double)d[0];
    const double y = Traits<T>::cplx ? (double)d[1] : 0.0;
    const double lim = 1.7976931348623157e308;
    LogState s{0.0, 0.0, 0, 0};
    if (!(x <= lim && x >= -lim && y <= lim && y >= -lim)) { s.flags = 1; return s; }
    const double ax = fabs(x), ay = fabs(y);
    const double hi = ax > ay ? ax : ay, lo = ax > ay ? ay : ax;
    if (hi == 0.0) { s.flags = 2; return s; }
    const double ratio = lo / hi;
    s.mag = log(hi) + 0.5 * log1p(ratio * ratio);
    if (y == 0.0) { s.flags = x < 0.0 ? 4 : 0; return s; }
    s.phase = atan2(y, x);
    return s;
}

__device__ __forceinline__ LogState warp_join(LogState s)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        LogState t;
        t.mag = __shfl_down_sync(0xffffffffu, s.mag, o);
        t.phase = __shfl_down_sync(0xffffffffu, s.phase, o);
        t.flags = __shfl_down_sync(0xffffffffu, s.flags, o);
        t.pad = 0;
        s = join(s, t);
    }
    return s;
}

__device__ __forceinline__ LogState block_join(LogState s)
{
    __shared__ LogState part[32];
    s = warp_join(s);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) part[warp] = s;
    __syncthreads();
    if (warp == 0) {
        s = lane < (int)(blockDim.x >> 5) ? part[lane] : LogState{0.0, 0.0, 0, 0};
        s = warp_join(s);
    }
    return s;
}

template <class T>
__global__ void __launch_bounds__(256) k_logdet_partial(const T* __restrict__ A, long long lda, int n, LogState* partial)
{
    LogState s{0.0, 0.0, 0, 0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s = join(s, term<T>(A, lda, i));
    s = block_join(s);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

template <class T>
__global__ void __launch_bounds__(256) k_logdet_partial_grid(const T* __restrict__ A, long long lda, GridLayout L,
                                                             long long count, LogState* partial)
{
    LogState s{0.0, 0.0, 0, 0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        s = join(s, term_grid<T>(A, lda, L, i));
    s = block_join(s);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void __launch_bounds__(256) k_logdet_final(const LogState* partial, int count, LogState* out)
{
    LogState s{0.0, 0.0, 0, 0};
    for (int i = threadIdx.x; i < count; i += blockDim.x) s = join(s, partial[i]);
    s = block_join(s);
    if (threadIdx.x == 0) *out = s;
}

constexpr int kLogdetCtas = 296;  // two per SM on a 148-SM B200

template <class T>
cudaError_t logdet_typed(int n, const void* A, long long lda, void* work, cudaStream_t st)
{
    LogState* out = static_cast<LogState*>(work);
    LogState* partial = out + 1;
    long long ctas = ceil_div(n, 256);
    if (ctas > kLogdetCtas) ctas = kLogdetCtas;
    if (ctas < 1) ctas = 1;
    ProfScope ps(PK_LOGDET, st, 0.0, (double)sizeof(T) * n);
    k_logdet_partial<T><<<(unsigned)ctas, 256, 0, st>>>(static_cast<const T*>(A), lda, n, partial);
    k_logdet_final<<<1, 256, 0, st>>>(partial, (int)ctas, out);
    note_launches(2);
    return cudaGetLastError();
}

template <class T>
cudaError_t logdet_grid_typed(const void* A, long long lda, const GridLayout& L, long long count, void* work,
                              cudaStream_t st)
{
    LogState* out = static_cast<LogState*>(work);
    LogState* partial = out + 1;
    long long ctas = ceil_div(count, 256);
    if (ctas > kLogdetCtas) ctas = kLogdetCtas;
    if (ctas < 1) ctas = 1;
    ProfScope ps(PK_LOGDET, st, 0.0, (double)sizeof(T) * count);
    k_logdet_partial_grid<T><<<(unsigned)ctas, 256, 0, st>>>(static_cast<const T*>(A), lda, L, count, partial);
    k_logdet_final<<<1, 256, 0, st>>>(partial, (int)ctas, out);
    note_launches(2);
    return cudaGetLastError();
}

}  // namespace ddlak

// The same reduction over the diagonal entries one rank of a pr x pc block-cyclic
// grid holds (its local rows when pr >= pc, else its local columns; the reference's
// pdiag_logdet, src/PBLAS/pdiag_logdet.cpp:26-37): A is that rank's local matrix
// (leading dimension lld, local_rows x local_cols).  Same output as ddlak_diag_logsum.
extern "C" int ddlak_diag_logsum_grid(char type, int n, const void* A, long long lld, int local_rows, int local_cols,
                                      int mb, int nb, int pr, int pc, int row, int col, int rsrc, int csrc, void* work,
                                      void* stream)
{
    using namespace ddlak;
    if (n < 0 || mb <= 0 || nb <= 0 || pr <= 0 || pc <= 0 || row < 0 || row >= pr || col < 0 || col >= pc ||
        rsrc < 0 || rsrc >= pr || csrc < 0 || csrc >= pc)
        return (int)cudaErrorInvalidValue;
    GridLayout L{n, mb, nb, pr, pc, row, col, rsrc, csrc, pr >= pc};
    const long long count = (local_rows <= 0 || local_cols <= 0) ? 0 : (pr >= pc ? local_rows : local_cols);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (type) {
    case 's': return (int)logdet_grid_typed<float>(A, lld, L, count, work, st);
    case 'd': return (int)logdet_grid_typed<double>(A, lld, L, count, work, st);
    case 'c': return (int)logdet_grid_typed<cf32>(A, lld, L, count, work, st);
    case 'z': return (int)logdet_grid_typed<cf64>(A, lld, L, count, work, st);
    default: return (int)cudaErrorInvalidValue;
    }
}

extern "C" unsigned long long ddlak_logdet_workspace(void)
{
    return sizeof(ddlak::LogState) * (1 + ddlak::kLogdetCtas);
}

// Writes {double magnitude, double phase, int flags} (the first 20 bytes of
// the workspace) on the stream; the caller copies it back and finishes.
extern "C" int ddlak_diag_logsum(char type, int n, const void* A, long long lda, void* work, void* stream)
{
    using namespace ddlak;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (type) {
    case 's': return (int)logdet_typed<float>(n, A, lda, work, st);
    case 'd': return (int)logdet_typed<double>(n, A, lda, work, st);
    case 'c': return (int)logdet_typed<cf32>(n, A, lda, work, st);
    case 'z': return (int)logdet_typed<cf64>(n, A, lda, work, st);
    default: return (int)cudaErrorInvalidValue;
    }
}
