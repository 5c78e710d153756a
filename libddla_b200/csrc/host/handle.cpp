// Handle lifecycle, memory and query API (reference src/ddla_handle_t.cpp and
// src/ddla_stream.cpp, restricted to a GPU handle on a 1x1 grid).
#include <cuda_runtime.h>

#include <functional>
#include <memory>

#include <atomic>
#include <cstring>
#include <mutex>
#include <string>

#include <ddla/ddla_desc.h>
#include <ddla/ddla_handle_t.h>

#include "ddla_stream.h"

namespace ddla {

namespace {
thread_local std::string g_last_cuda_message;

ddlaStatus_t from_cuda(cudaError_t e)
{
    if (e == cudaSuccess) return ddlaStatus_t::DDLA_STATUS_SUCCESS;
    detail::remember_cuda_error(e);
    return ddlaStatus_t::DDLA_STATUS_INTERNAL_ERROR;
}

bool gpu_present()
{
    int count = 0;
    const cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return count > 0;
}

bool is_device_pointer(const void* p)
{
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}
}  // namespace

namespace detail {
void remember_cuda_error(cudaError_t e) { g_last_cuda_message = cudaGetErrorString(e); }

namespace {
std::atomic<long long> g_alloc_countdown{0};  // 0: disarmed
std::atomic<long long> g_live_workspaces{0};
}  // namespace

void arm_allocation_failure(long long nth) { g_alloc_countdown.store(nth > 0 ? nth : 0); }

bool allocation_fails()
{
    long long c = g_alloc_countdown.load();
    while (c > 0) {
        if (g_alloc_countdown.compare_exchange_weak(c, c - 1)) return c == 1;
    }
    return false;
}

void note_workspace(int delta) { g_live_workspaces.fetch_add(delta); }
long long live_workspaces() { return g_live_workspaces.load(); }

void require_gpu(const DdlaHandle_t& h, const char* routine)
{
    if (h == nullptr) throw std::invalid_argument(std::string(routine) + ": null handle");
    if (!h->initialized) throw std::invalid_argument(std::string(routine) + ": handle has no process grid (call ddlaSet)");
    if (h->backend != DdlaBackend::GPU) throw std::invalid_argument(std::string(routine) + ": handle backend is not GPU");
    cuda_check(cudaSetDevice(h->device), "cudaSetDevice");
}

// Validation of a ScaLAPACK descriptor against the handle's grid, with the
// reference's messages (src/ddla_desc.cpp:9-59).
void check_desc(const int* desc, const DdlaHandle_t& handle)
{
    if (desc == nullptr) throw std::invalid_argument("ddla: null ScaLAPACK descriptor");
    if (handle == nullptr) throw std::invalid_argument("ddla: null handle for ScaLAPACK descriptor");
    if (desc[DDLA_DTYPE_] != DDLA_BLOCK_CYCLIC_2D)
        throw std::invalid_argument("ddla: unsupported descriptor type " + std::to_string(desc[DDLA_DTYPE_]) +
                                    "; only dense block-cyclic (DTYPE_ == 1) is supported");
    int nprows = 0, npcols = 0, myprow = -1, mypcol = -1;
    ddlaGetGridDims(handle, nprows, npcols);
    ddlaGetGridCoords(handle, myprow, mypcol);
    if (nprows <= 0 || npcols <= 0) throw std::invalid_argument("ddla: handle carries no process grid");
    if (desc[DDLA_M_] < 0 || desc[DDLA_N_] < 0)
        throw std::invalid_argument("ddla: descriptor M/N must be non-negative, got M=" + std::to_string(desc[DDLA_M_]) +
                                    " N=" + std::to_string(desc[DDLA_N_]));
    if (desc[DDLA_MB_] <= 0 || desc[DDLA_NB_] <= 0)
        throw std::invalid_argument("ddla: descriptor MB/NB must be positive, got MB=" +
                                    std::to_string(desc[DDLA_MB_]) + " NB=" + std::to_string(desc[DDLA_NB_]));
    if (desc[DDLA_RSRC_] < 0 || desc[DDLA_RSRC_] >= nprows || desc[DDLA_CSRC_] < 0 || desc[DDLA_CSRC_] >= npcols)
        throw std::invalid_argument("ddla: descriptor RSRC/CSRC outside the process grid (" + std::to_string(nprows) +
                                    "x" + std::to_string(npcols) + "), got RSRC=" + std::to_string(desc[DDLA_RSRC_]) +
                                    " CSRC=" + std::to_string(desc[DDLA_CSRC_]));
    const int required = std::max(1, num_loc(desc[DDLA_M_], desc[DDLA_MB_], myprow, desc[DDLA_RSRC_], nprows));
    if (desc[DDLA_LLD_] < required)
        throw std::invalid_argument("ddla: ScaLAPACK descriptor LLD_A=" + std::to_string(desc[DDLA_LLD_]) +
                                    " is smaller than the required max(1, LOCr(M_A))=" + std::to_string(required) +
                                    "; the descriptor does not match this handle's process grid");
}
}  // namespace detail

bool ddlaBackendAvailable(DdlaBackend backend)
{
    if (backend == DdlaBackend::GPU) return gpu_present();
    return false;  // no CPU implementation: the product has no CPU fallback
}

ddlaStatus_t ddlaInit(DdlaHandle_t& handle, DdlaBackend requested_backend)
{
    if (requested_backend != DdlaBackend::GPU && requested_backend != DdlaBackend::CPU)
        return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    if (!ddlaBackendAvailable(requested_backend))
        throw std::runtime_error(requested_backend == DdlaBackend::CPU
                                     ? "ddlaInit: the CPU backend is not part of this build"
                                     : "ddlaInit: no CUDA device is visible");
    auto* s = new DdlaStream;
    s->backend = requested_backend;
    cudaGetDevice(&s->device);
    handle = s;
    return ddlaStatus_t::DDLA_STATUS_SUCCESS;
}

// The handle's stream and pinned word, created once (the first ddlaSet*).
static ddlaStatus_t ensure_resources(DdlaHandle_t handle)
{
    if (!handle->initialized) {
        const cudaError_t e1 = cudaSetDevice(handle->device);
        if (e1 != cudaSuccess) return from_cuda(e1);
        const cudaError_t e2 = cudaStreamCreateWithFlags(&handle->stream, cudaStreamNonBlocking);
        if (e2 != cudaSuccess) return from_cuda(e2);
        handle->owns_stream = true;
        const cudaError_t e3 = detail::allocation_fails()
                                   ? cudaErrorMemoryAllocation
                                   : cudaMallocHost(reinterpret_cast<void**>(&handle->host_word), 64);
        if (e3 != cudaSuccess) {  // leave the handle as it was, so a retry starts clean
            cudaStreamDestroy(handle->stream);
            handle->stream = nullptr;
            handle->owns_stream = false;
            handle->host_word = nullptr;
            return from_cuda(e3);
        }
        // Workspace comes from the device's stream-ordered pool (cudaMallocAsync).
        // Keep freed blocks in the pool instead of unmapping them at every
        // synchronisation: the multi-GB workspaces of consecutive calls then reuse
        // the same mapped memory.
        cudaMemPool_t pool = nullptr;
        if (cudaDeviceGetDefaultMemPool(&pool, handle->device) == cudaSuccess) {
            unsigned long long keep = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    return ddlaStatus_t::DDLA_STATUS_SUCCESS;
}

static ddlaStatus_t set_impl(DdlaHandle_t handle, const MPI_Comm& comm, int nprows, int npcols, char major)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    if (major != 'R' && major != 'C') return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
#ifndef DDLA_SINGLE_RANK_MPI
    int size = 1;
    MPI_Comm_size(comm, &size);
    if (size != 1) return ddlaStatus_t::DDLA_STATUS_BACKEND_UNAVAILABLE;
#endif
    if (nprows * npcols != 1) return ddlaStatus_t::DDLA_STATUS_BACKEND_UNAVAILABLE;
    if (const ddlaStatus_t e = ensure_resources(handle); e != ddlaStatus_t::DDLA_STATUS_SUCCESS) return e;
    handle->grid.reset();
    handle->comm = comm;
    handle->nprows_ = handle->npcols_ = 1;
    handle->myprow_ = handle->mypcol_ = 0;
    handle->rank = 0;
    handle->nprocs = 1;
    handle->major = major;
    handle->initialized = true;
    return ddlaStatus_t::DDLA_STATUS_SUCCESS;
}

ddlaStatus_t ddlaSet(DdlaHandle_t handle, const MPI_Comm& comm, char major) { return set_impl(handle, comm, 1, 1, major); }
ddlaStatus_t ddlaSet(DdlaHandle_t handle, const MPI_Comm& comm, int nprows, int npcols, char major)
{
    if (nprows <= 0 || npcols <= 0) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    return set_impl(handle, comm, nprows, npcols, major);
}

// ---- grids of more than one rank -------------------------------------------
struct DdlaLocalGroup {
    std::shared_ptr<detail::LocalGroup> g;
};

ddlaStatus_t ddlaLocalGroupCreate(DdlaLocalGroup** group, int nranks, double timeout_s)
{
    if (group == nullptr || nranks < 1) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    *group = new DdlaLocalGroup{detail::make_local_group(nranks, timeout_s)};
    return ddlaStatus_t::DDLA_STATUS_SUCCESS;
}

ddlaStatus_t ddlaLocalGroupDestroy(DdlaLocalGroup* group)
{
    delete group;  // the members' handles keep the group alive until they are destroyed
    return ddlaStatus_t::DDLA_STATUS_SUCCESS;
}

static ddlaStatus_t set_grid(DdlaHandle_t handle, int rank, int nprows, int npcols, char major,
                             const std::function<std::unique_ptr<detail::GridComm>()>& make)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    if ((major != 'R' && major != 'C') || nprows <= 0 || npcols <= 0 || rank < 0 || rank >= nprows * npcols)
        return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    const cudaError_t e = cudaSetDevice(handle->device);
    if (e != cudaSuccess) return from_cuda(e);
    if (const ddlaStatus_t s = ensure_resources(handle); s != ddlaStatus_t::DDLA_STATUS_SUCCESS) return s;
    std::shared_ptr<detail::GridComm> comm;
    if (nprows * npcols > 1) comm = make();
    handle->grid = std::move(comm);
    handle->comm = MPI_COMM_WORLD;
    handle->nprows_ = nprows;
    handle->npcols_ = npcols;
    handle->major = major;
    handle->rank = rank;
    handle->nprocs = nprows * npcols;
    if (major == 'C') {
        handle->myprow_ = rank % nprows;
        handle->mypcol_ = rank / nprows;
    } else {
        handle->myprow_ = rank / npcols;
        handle->mypcol_ = rank % npcols;
    }
    handle->initialized = true;
    return ddlaStatus_t::DDLA_STATUS_SUCCESS;
}

ddlaStatus_t ddlaSetLocalGroup(DdlaHandle_t handle, DdlaLocalGroup* group, int rank, int nprows, int npcols,
                               char major)
{
    if (group == nullptr || nprows * npcols != detail::local_group_size(*group->g)) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    const int dev = handle->device;
    return set_grid(handle, rank, nprows, npcols, major,
                    [&] { return detail::make_local_comm(group->g, rank, nprows, npcols, major, dev); });
}

bool ddlaNcclAvailable() { return detail::nccl_available(); }

ddlaStatus_t ddlaNcclUniqueId(void* id128)
{
    if (id128 == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    if (!detail::nccl_available()) return ddlaStatus_t::DDLA_STATUS_BACKEND_UNAVAILABLE;
    detail::nccl_unique_id(id128);
    return ddlaStatus_t::DDLA_STATUS_SUCCESS;
}

ddlaStatus_t ddlaSetNccl(DdlaHandle_t handle, const void* id128, int nranks, int rank, int nprows, int npcols,
                         char major)
{
    if (id128 == nullptr || nprows * npcols != nranks) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    if (nranks > 1 && !detail::nccl_available()) return ddlaStatus_t::DDLA_STATUS_BACKEND_UNAVAILABLE;
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    const int dev = handle->device;
    return set_grid(handle, rank, nprows, npcols, major,
                    [&] { return detail::make_nccl_comm(id128, nranks, rank, nprows, npcols, major, dev); });
}

ddlaStatus_t ddlaDestroy(DdlaHandle_t& handle)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_SUCCESS;
    DdlaStream* s = handle;
    if (s->initialized || s->stream || s->host_word) {
        cudaSetDevice(s->device);
        if (s->stream) cudaStreamSynchronize(s->stream);
        s->grid.reset();
        if (s->owns_stream && s->stream) cudaStreamDestroy(s->stream);
        if (s->host_word) cudaFreeHost(s->host_word);
    }
    delete s;
    handle = nullptr;
    return ddlaStatus_t::DDLA_STATUS_SUCCESS;
}

DdlaBackend ddlaGetBackend(const DdlaHandle_t& handle)
{
    if (handle == nullptr) throw std::runtime_error("ddlaGetBackend: null handle");
    return handle->backend;
}

ddlaStatus_t ddlaSetCommunication(const DdlaHandle_t& handle, DdlaCommunication mode)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    const int m = static_cast<int>(mode);
    if (m < 0 || m > 2) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    handle->communication = mode;  // a single rank never communicates
    return ddlaStatus_t::DDLA_STATUS_SUCCESS;
}
DdlaCommunication ddlaGetCommunication(const DdlaHandle_t& handle)
{
    if (handle == nullptr) throw std::runtime_error("ddlaGetCommunication: null handle");
    return handle->communication;
}
bool ddlaCommunicationAvailable(const DdlaHandle_t& handle, DdlaCommunication mode)
{
    const int m = static_cast<int>(mode);
    return handle != nullptr && m >= 0 && m <= 2;
}

ddlaStatus_t ddlaMalloc(const DdlaHandle_t& handle, void** ptr, std::size_t bytes)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    if (ptr == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    if (bytes == 0) {
        *ptr = nullptr;
        return ddlaStatus_t::DDLA_STATUS_SUCCESS;
    }
    if (detail::allocation_fails()) return from_cuda(cudaErrorMemoryAllocation);
    cudaSetDevice(handle->device);
    return from_cuda(cudaMallocAsync(ptr, bytes, handle->stream));
}
ddlaStatus_t ddlaFree(const DdlaHandle_t& handle, void* ptr)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    if (ptr == nullptr) return ddlaStatus_t::DDLA_STATUS_SUCCESS;
    return from_cuda(cudaFreeAsync(ptr, handle->stream));
}
ddlaStatus_t ddlaMallocHost(const DdlaHandle_t& handle, void** ptr, std::size_t bytes)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    if (ptr == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    if (bytes == 0) {
        *ptr = nullptr;
        return ddlaStatus_t::DDLA_STATUS_SUCCESS;
    }
    if (detail::allocation_fails()) return from_cuda(cudaErrorMemoryAllocation);
    return from_cuda(cudaMallocHost(ptr, bytes));
}
ddlaStatus_t ddlaFreeHost(const DdlaHandle_t& handle, void* ptr)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    if (ptr == nullptr) return ddlaStatus_t::DDLA_STATUS_SUCCESS;
    return from_cuda(cudaFreeHost(ptr));
}

ddlaStatus_t ddlaMemcpy(const DdlaHandle_t& handle, void* dst, const void* src, std::size_t bytes)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    if (bytes == 0) return ddlaStatus_t::DDLA_STATUS_SUCCESS;
    if (dst == nullptr || src == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    if (!is_device_pointer(dst) && !is_device_pointer(src)) {
        std::memcpy(dst, src, bytes);
        return ddlaStatus_t::DDLA_STATUS_SUCCESS;
    }
    return from_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, handle->stream));
}
ddlaStatus_t ddlaMemcpy2D(const DdlaHandle_t& handle, void* dst, std::size_t dpitch, const void* src,
                          std::size_t spitch, std::size_t width, std::size_t height)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    if (width == 0 || height == 0) return ddlaStatus_t::DDLA_STATUS_SUCCESS;
    if (dst == nullptr || src == nullptr || dpitch < width || spitch < width)
        return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    if (!is_device_pointer(dst) && !is_device_pointer(src)) {
        for (std::size_t r = 0; r < height; ++r)
            std::memcpy(static_cast<char*>(dst) + r * dpitch, static_cast<const char*>(src) + r * spitch, width);
        return ddlaStatus_t::DDLA_STATUS_SUCCESS;
    }
    return from_cuda(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, cudaMemcpyDefault, handle->stream));
}
ddlaStatus_t ddlaMemset(const DdlaHandle_t& handle, void* ptr, int value, std::size_t bytes)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    if (bytes == 0) return ddlaStatus_t::DDLA_STATUS_SUCCESS;
    if (ptr == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    return from_cuda(cudaMemsetAsync(ptr, value, bytes, handle->stream));
}
ddlaStatus_t ddlaSynchronize(const DdlaHandle_t& handle)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    return from_cuda(cudaStreamSynchronize(handle->stream));
}
ddlaStatus_t ddlaDeviceSynchronize(const DdlaHandle_t& handle)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    cudaSetDevice(handle->device);
    return from_cuda(cudaDeviceSynchronize());
}
ddlaStatus_t ddlaEventCreate(const DdlaHandle_t& handle, ddlaEvent_t* event)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    if (event == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    cudaEvent_t e = nullptr;
    const cudaError_t err = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    *event = e;
    return from_cuda(err);
}
ddlaStatus_t ddlaEventDestroy(const DdlaHandle_t& handle, ddlaEvent_t event)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    if (event == nullptr) return ddlaStatus_t::DDLA_STATUS_SUCCESS;
    return from_cuda(cudaEventDestroy(static_cast<cudaEvent_t>(event)));
}
ddlaStatus_t ddlaEventRecord(const DdlaHandle_t& handle, ddlaEvent_t event)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    if (event == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    return from_cuda(cudaEventRecord(static_cast<cudaEvent_t>(event), handle->stream));
}
ddlaStatus_t ddlaEventWait(const DdlaHandle_t& handle, ddlaEvent_t event)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    if (event == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    return from_cuda(cudaStreamWaitEvent(handle->stream, static_cast<cudaEvent_t>(event), 0));
}
ddlaStatus_t ddlaEventSynchronize(const DdlaHandle_t& handle, ddlaEvent_t event)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    if (event == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    return from_cuda(cudaEventSynchronize(static_cast<cudaEvent_t>(event)));
}
ddlaStatus_t ddlaGetLastError(const DdlaHandle_t& handle)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    return from_cuda(cudaGetLastError());
}
ddlaStatus_t ddlaSetDevice(const DdlaHandle_t& handle)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    return from_cuda(cudaSetDevice(handle->device));
}
ddlaStatus_t ddlaGetDeviceCount(const DdlaHandle_t& handle, int* count)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    if (count == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    return from_cuda(cudaGetDeviceCount(count));
}
ddlaStatus_t ddlaMemGetInfo(const DdlaHandle_t& handle, std::size_t* free_bytes, std::size_t* total_bytes)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    if (free_bytes == nullptr || total_bytes == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    cudaSetDevice(handle->device);
    return from_cuda(cudaMemGetInfo(free_bytes, total_bytes));
}
const char* ddlaGetErrorString(ddlaStatus_t status)
{
    switch (status) {
    case ddlaStatus_t::DDLA_STATUS_SUCCESS: return "DDLA_STATUS_SUCCESS";
    case ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE: return "DDLA_STATUS_INVALID_HANDLE";
    case ddlaStatus_t::DDLA_STATUS_INVALID_VALUE: return "DDLA_STATUS_INVALID_VALUE";
    case ddlaStatus_t::DDLA_STATUS_ALLOC_FAILED: return "DDLA_STATUS_ALLOC_FAILED";
    case ddlaStatus_t::DDLA_STATUS_BACKEND_UNAVAILABLE: return "DDLA_STATUS_BACKEND_UNAVAILABLE";
    case ddlaStatus_t::DDLA_STATUS_INTERNAL_ERROR: {
        static thread_local std::string msg;
        msg = "DDLA_STATUS_INTERNAL_ERROR";
        if (!g_last_cuda_message.empty()) msg += ": " + g_last_cuda_message;
        return msg.c_str();
    }
    }
    return "unknown ddla status";
}
ddlaStatus_t ddlaSetStream(const DdlaHandle_t& handle, void* stream)
{
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    if (!handle->initialized) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (s == handle->stream) return ddlaStatus_t::DDLA_STATUS_SUCCESS;
    const cudaError_t e = cudaStreamSynchronize(handle->stream);
    if (e != cudaSuccess) return from_cuda(e);
    if (handle->owns_stream && handle->stream) cudaStreamDestroy(handle->stream);
    handle->stream = s;
    handle->owns_stream = s != nullptr;
    return ddlaStatus_t::DDLA_STATUS_SUCCESS;
}
void* ddlaGetStream(const DdlaHandle_t& handle) { return handle ? static_cast<void*>(handle->stream) : nullptr; }

MPI_Comm ddlaGetCommunicator(const DdlaHandle_t& handle) { return handle ? handle->comm : MPI_COMM_NULL; }
MPI_Comm ddlaGetRowCommunicator(const DdlaHandle_t& handle) { return handle ? handle->comm : MPI_COMM_NULL; }
MPI_Comm ddlaGetColCommunicator(const DdlaHandle_t& handle) { return handle ? handle->comm : MPI_COMM_NULL; }
int ddlaGetRank(const DdlaHandle_t& handle) { return handle ? handle->rank : -1; }
int ddlaGetSize(const DdlaHandle_t& handle) { return handle ? handle->nprocs : -1; }
void ddlaGetGridCoords(const DdlaHandle_t& handle, int& myprow, int& mypcol)
{
    myprow = handle && handle->initialized ? handle->myprow_ : -1;
    mypcol = handle && handle->initialized ? handle->mypcol_ : -1;
}
void ddlaGetGridDims(const DdlaHandle_t& handle, int& nprows, int& npcols)
{
    nprows = handle && handle->initialized ? handle->nprows_ : 0;
    npcols = handle && handle->initialized ? handle->npcols_ : 0;
}
// rank <-> (row, col), row-major for 'R' and column-major for 'C' (src/ddla_stream.h:114-125);
// -1 outside the grid
void ddlaRankToRc(const DdlaHandle_t& handle, int rank, int& row, int& col)
{
    row = col = -1;
    if (handle == nullptr || !handle->initialized || rank < 0 || rank >= handle->nprocs) return;
    if (handle->major == 'C') {
        row = rank % handle->nprows_;
        col = rank / handle->nprows_;
    } else {
        row = rank / handle->npcols_;
        col = rank % handle->npcols_;
    }
}
int ddlaRcToRank(const DdlaHandle_t& handle, int row, int col)
{
    if (handle == nullptr || !handle->initialized || row < 0 || col < 0 || row >= handle->nprows_ ||
        col >= handle->npcols_)
        return -1;
    return handle->major == 'C' ? col * handle->nprows_ + row : row * handle->npcols_ + col;
}

}  // namespace ddla
