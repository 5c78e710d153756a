// Declarations shared between the kernel translation units (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"

namespace ddlak {

// C(i,j) -= sum_{k0 <= c < k0+nbk} L(i,c) conj(L(j,c)) for the lower-triangle
// entries of the region rows [t0, n) x columns [t0, n) (cols == 0) or
// columns [t0, t0+cols) (cols > 0), in the L view of common.cuh.
template <class T, bool UP>
cudaError_t trailing_update(T* A, long long lda, int k0, int nbk, int n, long long t0, int cols, const int* dinfo,
                            cudaStream_t st);

// X * L11^H = A21 for the rows below the diagonal block [k0, k0+nbk) (potrf.cu).
template <class T, bool UP>
cudaError_t launch_trsm_panel(T* A, long long lda, int k0, int nbk, int n, const int* dinfo, cudaStream_t s);

// The FP64 lower update of the region from row / column t0 (all of it, or its
// first cols columns when cols > 0) over a batch of equal-order matrices
// (astride elements apart, info per matrix) by the TMA DMMA tile kernel
// (syrk.cu); false (nothing launched) when its conditions (even lda and
// astride, 16-byte aligned A, nbk a multiple of 32) do not hold.
bool launch_dmma_tma_batched(double* A, long long lda, long long astride, int batch, int k0, int nbk, int n,
                             long long t0, int cols, const int* dinfo, cudaStream_t st, cudaError_t* err);

template <class T, bool UP>
cudaError_t trailing_update_simt(T* A, long long lda, int k0, int nbk, int n, long long t0, int cols,
                                 const int* dinfo, cudaStream_t st);

}  // namespace ddlak
