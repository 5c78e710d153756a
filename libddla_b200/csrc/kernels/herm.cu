// Hermitian completion of the leading n x n (the reference's herm_complete,
// used by src/Eigensolver/phegst.cpp:140-176): the triangle opposite uplo is
// overwritten with the conjugate transpose of the uplo triangle and the
// diagonal's imaginary part is zeroed.  One CTA per 32 x 32 tile pair: the
// source tile (in the uplo triangle) is read coalesced into shared memory and
// its conjugate transpose written coalesced into the mirror tile.
#include <cuda_runtime.h>

#include <ddla_kernels.h>

#include "common.cuh"
#include "profile.h"

namespace ddlak {
namespace {

constexpr int HT = 32;  // tile edge; blocks of 32 x 8 threads

template <class T, bool UP>
__global__ void __launch_bounds__(256) k_herm_complete(T* __restrict__ A, long long lda, int n)
{
    __shared__ T s[HT][HT + 1];
    const int I = blockIdx.x, J = blockIdx.y;  // tile row / column of the lower tile pair, I >= J
    if (I < J) return;
    const int tx = threadIdx.x, ty = threadIdx.y;
    // source block origin (rows, cols) in the uplo triangle; its mirror has the transposed origin
    const long long rs0 = (long long)(UP ? J : I) * HT, cs0 = (long long)(UP ? I : J) * HT;
    auto src_valid = [&](long long r, long long c) { return r < n && c < n && (UP ? r < c : r > c); };
    for (int c = ty; c < HT; c += 8) {
        const long long r = rs0 + tx, col = cs0 + c;
        if (src_valid(r, col)) s[c][tx] = A[r + col * lda];
        if (I == J && r == col && r < n) A[r + r * lda] = from_real<T>(re(A[r + r * lda]));
    }
    __syncthreads();
    // mirror element (cs0 + tx, rs0 + c) is the conjugate of source element (rs0 + c, cs0 + tx)
    for (int c = ty; c < HT; c += 8) {
        if (src_valid(rs0 + c, cs0 + tx)) A[(cs0 + tx) + (rs0 + c) * lda] = cj(s[tx][c]);
    }
}

template <class T>
cudaError_t herm_typed(char uplo, int n, void* A, long long lda, cudaStream_t st)
{
    const int nt = (int)ceil_div(n, HT);
    const dim3 grid((unsigned)nt, (unsigned)nt), block(HT, 8);
    if (uplo == 'U') k_herm_complete<T, true><<<grid, block, 0, st>>>(static_cast<T*>(A), lda, n);
    else k_herm_complete<T, false><<<grid, block, 0, st>>>(static_cast<T*>(A), lda, n);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace
}  // namespace ddlak

extern "C" int ddlak_herm_complete(char type, char uplo, int n, void* A, long long lda, void* stream)
{
    using namespace ddlak;
    if (n <= 0) return 0;
    if (!A || lda < n || (uplo != 'L' && uplo != 'U') || ceil_div(n, HT) > 65535) return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (type) {
    case 's': return (int)herm_typed<float>(uplo, n, A, lda, st);
    case 'd': return (int)herm_typed<double>(uplo, n, A, lda, st);
    case 'c': return (int)herm_typed<cf32>(uplo, n, A, lda, st);
    case 'z': return (int)herm_typed<cf64>(uplo, n, A, lda, st);
    default: return (int)cudaErrorInvalidValue;
    }
}
