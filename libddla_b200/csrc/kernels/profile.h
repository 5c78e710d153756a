// Launch accounting / optional CUDA-event timing shared by the kernel launchers.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

namespace ddlak {

// Kernel kinds reported by ddlak_profile_read.
enum ProfKind : int {
    PK_POTRF_DIAG = 0,
    PK_TRSM_PANEL = 1,
    PK_SYRK_UPDATE = 2,
    PK_POTRS_FUSED = 3,
    PK_LOGDET = 4,
    PK_MIXED_UPDATE = 5,
    PK_MIXED_OTHER = 6,
    PK_SYMM_RESIDUAL = 7,
    PK_BATCHED = 8,
    PK_ADJOINT = 9,
    PK_TRTRI = 10,
    PK_COUNT = 11
};

void note_launches(int count);
bool profiling();

// Raise kernel `func`'s dynamic shared-memory limit to `bytes` on the current
// device.  cudaFuncSetAttribute applies to one device only, so the raise is
// recorded per (kernel, device) and made again on every other device; thread
// safe; returns the attribute call's error, if any.
cudaError_t smem_optin(const void* func, std::size_t bytes);
template <class K>
cudaError_t smem_optin(K* func, std::size_t bytes)
{
    return smem_optin(reinterpret_cast<const void*>(func), bytes);
}

// Brackets the launches made while it lives with two events on st (profiling on only).
class ProfScope {
public:
    ProfScope(int kind, cudaStream_t st, double flops, double bytes);
    ~ProfScope();
    ProfScope(const ProfScope&) = delete;
    ProfScope& operator=(const ProfScope&) = delete;

private:
    cudaStream_t st_;
    bool active_;
    std::size_t idx_ = 0;
};

}  // namespace ddlak
