// Declarations shared between the kernel translation units (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"

namespace ddlak {

// C -= L21 * L21^H on the lower tiles of the trailing matrix after block column
// [k0, k0+nbk) of an order-n factorization (L view, see common.cuh).
template <class T, bool UP>
cudaError_t trailing_update(T* A, long long lda, int k0, int nbk, int n, const int* dinfo, cudaStream_t st);

template <class T, bool UP>
cudaError_t trailing_update_simt(T* A, long long lda, int k0, int nbk, int n, const int* dinfo, cudaStream_t st);

}  // namespace ddlak
