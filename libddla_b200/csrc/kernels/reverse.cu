// A <- J A J on the leading n x n of a column-major matrix, J the order-
// reversing permutation: element (i, j) trades places with (n-1-i, n-1-j).
//
// The bottom-right Cholesky of the reference (src/Cholesky/potrf_bottom_right.cpp,
// the per-block reverse packing of src/Cholesky/potrf_bottom_right_transform.cpp:18-47)
// factors A = U U^H ('U') or A = L^H L ('L') starting from the last column.
// Since J A J = (J U J)(J U J)^H with J U J lower triangular, that factor is
// the ordinary Cholesky factor of J A J with the triangles exchanged, so the
// path here is one swap pass, the standard blocked factorization of the
// opposite triangle, and a second swap pass.  The swap is a permutation of
// the n x n block: the other triangle and the padding rows beyond n come back
// bit for bit.  One thread per element pair; consecutive threads touch
// consecutive rows of both partners, so loads and stores stay coalesced.
#include <cuda_runtime.h>

#include <cstdint>

#include <ddla_kernels.h>

#include "common.cuh"
#include "profile.h"

namespace ddlak {
namespace {

struct __align__(8) Pair16 {
    unsigned long long lo, hi;
};

template <class W>
__global__ void __launch_bounds__(256) k_reverse_swap(int n, W* __restrict__ A, long long lda)
{
    const long long total = (long long)n * n;
    const long long pairs = total / 2;  // an odd n^2 leaves the centre element, its own partner
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < pairs;
         p += (long long)gridDim.x * blockDim.x) {
        const long long q = total - 1 - p;  // (n-1-j)*n + (n-1-i) for p = j*n + i
        W* a = A + (p % n) + (p / n) * lda;
        W* b = A + (q % n) + (q / n) * lda;
        const W t = *a;
        *a = *b;
        *b = t;
    }
}

template <class W>
int launch(int n, void* A, long long lda, cudaStream_t st)
{
    const long long pairs = (long long)n * n / 2;
    if (pairs == 0) return 0;
    const long long blocks = ceil_div(pairs, 256) < 148 * 16 ? ceil_div(pairs, 256) : 148 * 16;
    k_reverse_swap<W><<<(unsigned)blocks, 256, 0, st>>>(n, static_cast<W*>(A), lda);
    note_launches(1);
    return (int)cudaGetLastError();
}

}  // namespace
}  // namespace ddlak

extern "C" int ddlak_reverse_swap(char type, int n, void* A, long long lda, void* stream)
{
    using namespace ddlak;
    if (n < 0 || (n > 0 && (!A || lda < n))) return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (type) {
    case 's': return launch<unsigned int>(n, A, lda, st);
    case 'd':
    case 'c': return launch<unsigned long long>(n, A, lda, st);
    case 'z': return launch<Pair16>(n, A, lda, st);
    default: return (int)cudaErrorInvalidValue;
    }
}
