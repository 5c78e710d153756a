// Private definition of the opaque handle (the reference's DdlaStream,
// src/ddla_stream.h:18-128, reduced to what a 1x1-grid GPU handle owns):
// the device, one compute stream, a pinned host word for info / status
// read-backs, and the grid coordinates of the single rank.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <stdexcept>
#include <string>

#include <ddla/ddla_handle_t.h>

#include <memory>

#include "grid_comm.h"

namespace ddla {

class DdlaStream {
public:
    DdlaBackend backend = DdlaBackend::GPU;
    DdlaCommunication communication = DdlaCommunication::MPI;
    bool initialized = false;   // ddlaSet done
    int device = 0;
    cudaStream_t stream = nullptr;
    bool owns_stream = false;
    int* host_word = nullptr;   // pinned, 64 bytes
    MPI_Comm comm = MPI_COMM_WORLD;
    int nprows_ = 1, npcols_ = 1, myprow_ = 0, mypcol_ = 0, rank = 0, nprocs = 1;
    char major = 'R';
    int host_threads = 1;
    // collectives of a grid of more than one rank (null on a 1x1 grid)
    std::shared_ptr<detail::GridComm> grid;
};

namespace detail {

// Throw std::runtime_error carrying the CUDA message (DDLA_CHECK semantics).
inline void cuda_check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess)
        throw std::runtime_error(std::string("ddla: ") + what + ": " + cudaGetErrorString(e));
}
inline void kernel_check(int e, const char* what) { cuda_check(static_cast<cudaError_t>(e), what); }

void require_gpu(const DdlaHandle_t& h, const char* routine);
void note_workspace(int delta);
void check_desc(const int* desc, const DdlaHandle_t& handle);
void remember_cuda_error(cudaError_t e);

// Bytes take<T>(cursor, count) consumes: padded to 256 so every buffer stays
// aligned (the reference's detail::padded_bytes, src/plan_util.h:30-43).
template <typename T>
constexpr std::size_t padded_bytes(std::size_t count)
{
    return (count * sizeof(T) + 255) / 256 * 256;
}
template <typename T>
inline T* take(char*& cursor, std::size_t count)
{
    T* p = reinterpret_cast<T*>(cursor);
    cursor += padded_bytes<T>(count);
    return p;
}

// Testing aid for the allocation-failure paths (the reference reaches them with
// an LD_PRELOAD allocator shim, tests/pblas_alloc_failure.cpp; with the CUDA
// runtime linked statically the shim cannot reach this library's calls, so
// the hook sits at the library's own allocation points).  When armed with n,
// the n-th device or pinned allocation from then on (workspace, ddlaMalloc,
// ddlaMallocHost, the handle's pinned word) fails as cudaErrorMemoryAllocation
// and the hook disarms.  live_workspaces() counts workspace allocations not
// yet released.
void arm_allocation_failure(long long nth);
bool allocation_fails();
long long live_workspaces();

// Stream-ordered device scratch owned for the duration of one call
// (the reference allocates per call with cudaMallocAsync, ddla_handle_t.cpp:322-338).
class DeviceScratch {
public:
    DeviceScratch(const DdlaHandle_t& h, std::size_t bytes) : h_(h), bytes_(bytes)
    {
        if (!bytes_) return;
        if (allocation_fails()) cuda_check(cudaErrorMemoryAllocation, "workspace allocation");
        cuda_check(cudaMallocAsync(&p_, bytes_, h_->stream), "workspace allocation");
        note_workspace(+1);
    }
    ~DeviceScratch()
    {
        if (p_) {
            cudaFreeAsync(p_, h_->stream);
            note_workspace(-1);
        }
    }
    DeviceScratch(const DeviceScratch&) = delete;
    DeviceScratch& operator=(const DeviceScratch&) = delete;
    char* data() const { return static_cast<char*>(p_); }
    std::size_t size() const { return bytes_; }

private:
    DdlaHandle_t h_;
    std::size_t bytes_;
    void* p_ = nullptr;
};

}  // namespace detail
}  // namespace ddla
