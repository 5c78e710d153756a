// Scalar traits and small device helpers shared by every Cholesky-path kernel.
//
// Storage types: float, double, cf32 (complex<float>) and cf64 (complex<double>).
// The complex types have the layout of std::complex<R> (two interleaved reals), so
// host pointers of std::complex<R> are reinterpreted at the C-ABI boundary.
//
// Every kernel addresses the factor through an "L view": L(i,j), i >= j, is
//   A[i + j*lda]            for uplo 'L' (A = L * L^H)
//   conj(A[j + i*lda])      for uplo 'U' (A = U^H * U, so L = U^H)
// which is how one kernel body serves both triangles of the reference's
// ppotrf/ppotrs (src/Cholesky/ppotrf.cpp:22-29, ppotrs.cpp:44-46).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ddlak {

struct __align__(8) cf32 { float x, y; };
struct __align__(16) cf64 { double x, y; };

template <class T> struct Traits;
template <> struct Traits<float>  { using R = float;  static constexpr bool cplx = false; };
template <> struct Traits<double> { using R = double; static constexpr bool cplx = false; };
template <> struct Traits<cf32>   { using R = float;  static constexpr bool cplx = true; };
template <> struct Traits<cf64>   { using R = double; static constexpr bool cplx = true; };

template <class T> using real_t = typename Traits<T>::R;

__host__ __device__ __forceinline__ float  re(float a)  { return a; }
__host__ __device__ __forceinline__ double re(double a) { return a; }
__host__ __device__ __forceinline__ float  re(cf32 a)   { return a.x; }
__host__ __device__ __forceinline__ double re(cf64 a)   { return a.x; }

__host__ __device__ __forceinline__ float  cj(float a)  { return a; }
__host__ __device__ __forceinline__ double cj(double a) { return a; }
__host__ __device__ __forceinline__ cf32 cj(cf32 a) { return {a.x, -a.y}; }
__host__ __device__ __forceinline__ cf64 cj(cf64 a) { return {a.x, -a.y}; }

template <class T> __host__ __device__ __forceinline__ T zero();
template <> __host__ __device__ __forceinline__ float  zero<float>()  { return 0.f; }
template <> __host__ __device__ __forceinline__ double zero<double>() { return 0.0; }
template <> __host__ __device__ __forceinline__ cf32 zero<cf32>() { return {0.f, 0.f}; }
template <> __host__ __device__ __forceinline__ cf64 zero<cf64>() { return {0.0, 0.0}; }

template <class T> __host__ __device__ __forceinline__ T from_real(real_t<T> r);
template <> __host__ __device__ __forceinline__ float  from_real<float>(float r)   { return r; }
template <> __host__ __device__ __forceinline__ double from_real<double>(double r) { return r; }
template <> __host__ __device__ __forceinline__ cf32 from_real<cf32>(float r)  { return {r, 0.f}; }
template <> __host__ __device__ __forceinline__ cf64 from_real<cf64>(double r) { return {r, 0.0}; }

__host__ __device__ __forceinline__ float  add(float a, float b)   { return a + b; }
__host__ __device__ __forceinline__ double add(double a, double b) { return a + b; }
__host__ __device__ __forceinline__ cf32 add(cf32 a, cf32 b) { return {a.x + b.x, a.y + b.y}; }
__host__ __device__ __forceinline__ cf64 add(cf64 a, cf64 b) { return {a.x + b.x, a.y + b.y}; }

__host__ __device__ __forceinline__ float  sub(float a, float b)   { return a - b; }
__host__ __device__ __forceinline__ double sub(double a, double b) { return a - b; }
__host__ __device__ __forceinline__ cf32 sub(cf32 a, cf32 b) { return {a.x - b.x, a.y - b.y}; }
__host__ __device__ __forceinline__ cf64 sub(cf64 a, cf64 b) { return {a.x - b.x, a.y - b.y}; }

__host__ __device__ __forceinline__ float  scal(float a, float r)    { return a * r; }
__host__ __device__ __forceinline__ double scal(double a, double r) { return a * r; }
__host__ __device__ __forceinline__ cf32 scal(cf32 a, float r)  { return {a.x * r, a.y * r}; }
__host__ __device__ __forceinline__ cf64 scal(cf64 a, double r) { return {a.x * r, a.y * r}; }

__host__ __device__ __forceinline__ float  divr(float a, float r)    { return a / r; }
__host__ __device__ __forceinline__ double divr(double a, double r) { return a / r; }
__host__ __device__ __forceinline__ cf32 divr(cf32 a, float r)  { return {a.x / r, a.y / r}; }
__host__ __device__ __forceinline__ cf64 divr(cf64 a, double r) { return {a.x / r, a.y / r}; }

// acc - a*b
__host__ __device__ __forceinline__ float  fms(float acc, float a, float b)    { return fmaf(-a, b, acc); }
__host__ __device__ __forceinline__ double fms(double acc, double a, double b) { return fma(-a, b, acc); }
__host__ __device__ __forceinline__ cf32 fms(cf32 acc, cf32 a, cf32 b)
{
    acc.x = fmaf(-a.x, b.x, acc.x); acc.x = fmaf(a.y, b.y, acc.x);
    acc.y = fmaf(-a.x, b.y, acc.y); acc.y = fmaf(-a.y, b.x, acc.y);
    return acc;
}
__host__ __device__ __forceinline__ cf64 fms(cf64 acc, cf64 a, cf64 b)
{
    acc.x = fma(-a.x, b.x, acc.x); acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(-a.x, b.y, acc.y); acc.y = fma(-a.y, b.x, acc.y);
    return acc;
}
// acc - a*conj(b)
template <class T> __host__ __device__ __forceinline__ T fmsc(T acc, T a, T b) { return fms(acc, a, cj(b)); }
// acc + a*b
template <class T> __host__ __device__ __forceinline__ T fma_(T acc, T a, T b)
{
    return fms(acc, sub(zero<T>(), a), b);
}

// Element (i,j) of the L view (i >= j is the only half ever addressed).
template <class T, bool UP>
__device__ __forceinline__ T lview_ld(const T* A, long long lda, long long i, long long j)
{
    if (UP) return cj(A[j + i * lda]);
    return A[i + j * lda];
}
template <class T, bool UP>
__device__ __forceinline__ void lview_st(T* A, long long lda, long long i, long long j, T v)
{
    if (UP) A[j + i * lda] = cj(v);
    else A[i + j * lda] = v;
}

// Status words written by kernels that wait on other CTAs.  A wait gives up
// after a clock budget and records one of these instead of spinning forever.
enum : int {
    DDLAK_OK = 0,
    DDLAK_WAIT_TIMEOUT = 1,
};

// The clock budget of a flag wait, in SM clock cycles (default 4e9, about 2 s at
// 1.9 GHz).  Every translation unit holds its own copy; ddlak_set_wait_budget
// sets all of them on the current device through the setters registered below.
constexpr long long kDefaultWaitBudget = 4000000000LL;
static __device__ long long g_wait_budget = kDefaultWaitBudget;
__device__ __forceinline__ long long wait_budget_cycles() { return *(volatile const long long*)&g_wait_budget; }

// Host side: registry of the per-translation-unit setters (profile.cu).
bool register_wait_budget_setter(cudaError_t (*setter)(long long));
namespace {
inline cudaError_t set_tu_wait_budget(long long cycles)
{
    return cudaMemcpyToSymbol(g_wait_budget, &cycles, sizeof cycles);
}
[[maybe_unused]] const bool g_wait_budget_registered = register_wait_budget_setter(&set_tu_wait_budget);
}  // namespace

__device__ __forceinline__ int ld_acquire(const int* p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int* p, int v)
{
    asm volatile("st.release.gpu.global.b32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

// *p += v with release semantics at GPU scope (no return value)
__device__ __forceinline__ void red_release_add(int* p, int v)
{
    asm volatile("red.release.gpu.global.add.s32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

// Spin (one thread) until *flag >= want or the budget runs out.  Returns false
// on timeout after recording DDLAK_WAIT_TIMEOUT in *status.
__device__ __forceinline__ bool bounded_wait_geq(const int* flag, int want, int* status)
{
    if (ld_acquire(flag) >= want) return true;
    const long long t0 = clock64();
    const long long budget = wait_budget_cycles();
    // a short tight spin first: the producer is usually microseconds away
    for (int it = 0; it < 4096; ++it) {
        if (ld_acquire(flag) >= want) return true;
        if ((it & 63) == 63 && clock64() - t0 > budget) break;
    }
    unsigned ns = 32;
    while (true) {
        if (ld_acquire(flag) >= want) return true;
        if (ld_acquire(status) != DDLAK_OK) return false;
        if (clock64() - t0 > budget) {
            atomicCAS(status, DDLAK_OK, DDLAK_WAIT_TIMEOUT);
            return false;
        }
        __nanosleep(ns);
        if (ns < 1024) ns <<= 1;
    }
}

__host__ __device__ __forceinline__ long long ceil_div(long long a, long long b) { return (a + b - 1) / b; }

// Asynchronous global -> shared copy of one element (zero-filled when !valid).
template <int BYTES>
__device__ __forceinline__ void cp_async_elem(void* smem, const void* gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(s), "l"(gmem), "n"(BYTES),
                 "r"(valid ? BYTES : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_group_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_group_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_commit_wait_all()
{
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// Load the L-view block L(r0+i, c0+j), i < rows, j < cols (and i >= j when
// lower), into s[i + j*ld] with cp.async (one copy per element, coalesced for
// either storage), then conjugate in place for 'U' complex storage.  Entries
// outside the block are zero.  Ends with __syncthreads().
template <class T, bool UP>
__device__ __forceinline__ void load_lview_block(T* s, int ld, const T* A, long long lda, long long r0, long long c0,
                                                 int rows, int cols, int brows, int bcols, bool lower)
{
    auto elem = [&](int i, int j) {
        const bool valid = i < rows && j < cols && (!lower || i >= j);
        const T* src = UP ? A + (c0 + j) + (r0 + i) * lda : A + (r0 + i) + (c0 + j) * lda;
        cp_async_elem<sizeof(T)>(&s[i + j * ld], valid ? src : A, valid);
    };
    if (brows == 128 && bcols == 128) {
        // the full block: index arithmetic by shifts (consecutive threads on the contiguous index)
        for (int idx = threadIdx.x; idx < 128 * 128; idx += blockDim.x) {
            if (UP) elem(idx >> 7, idx & 127);
            else elem(idx & 127, idx >> 7);
        }
    } else {
        for (int idx = threadIdx.x; idx < brows * bcols; idx += blockDim.x) {
            if (UP) elem(idx / bcols, idx % bcols);
            else elem(idx % brows, idx / brows);
        }
    }
    cp_async_commit_wait_all();
    __syncthreads();
    if (UP && Traits<T>::cplx) {
        for (int idx = threadIdx.x; idx < brows * bcols; idx += blockDim.x) {
            const int i = idx % brows, j = idx / brows;
            s[i + j * ld] = cj(s[i + j * ld]);
        }
        __syncthreads();
    }
}

// Linear index b over the lower triangle of a tile grid (row-major: (0,0),
// (1,0),(1,1),(2,0),...) -> tile (I, J) with J <= I.
__device__ __forceinline__ void tile_of_tri(long long b, int& I, int& J)
{
    long long i = (long long)((sqrt(8.0 * (double)b + 1.0) - 1.0) * 0.5);
    while ((i + 1) * (i + 2) / 2 <= b) ++i;
    while (i * (i + 1) / 2 > b) --i;
    I = (int)i;
    J = (int)(b - i * (i + 1) / 2);
}

}  // namespace ddlak
