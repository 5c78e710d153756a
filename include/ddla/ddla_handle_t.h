// Handle, backend, status and memory API of the ddla Cholesky path.
//
// Same names, signatures and status semantics as the reference's
// include/ddla/ddla_handle_t.h (enums 16-36, lifecycle 51-67, queries 74-99,
// memory 130-204, synchronisation 252-300, grid accessors 307-337,
// DDLA_CHECK 343-352).  This library is built for B200 GPUs only: the GPU
// backend is available when a CUDA device is visible, the CPU backend is never
// available (there is no CPU fallback).  Without MPI in this build, a process
// grid of more than one rank is formed by ddlaSetLocalGroup (ranks that are
// threads of one process) or ddlaSetNccl (ranks that are processes joined by
// NCCL); ddlaSet itself serves the 1x1 grid.
#ifndef DDLA_HANDLE_T_H
#define DDLA_HANDLE_T_H

#include <cstddef>
#include <stdexcept>
#include <string>
#include <type_traits>

#include <ddla/ddla_mpi.h>

namespace ddla {

enum class DdlaBackend { CPU, GPU };

enum class DdlaCommunication { MPI = 0, HostStagedMPI = 1, CCL = 2 };

enum class ddlaStatus_t {
    DDLA_STATUS_SUCCESS = 0,
    DDLA_STATUS_INVALID_HANDLE,
    DDLA_STATUS_INVALID_VALUE,
    DDLA_STATUS_ALLOC_FAILED,
    DDLA_STATUS_BACKEND_UNAVAILABLE,
    DDLA_STATUS_INTERNAL_ERROR
};

class DdlaStream;
using DdlaHandle_t = DdlaStream*;

// Lifecycle.  ddlaInit throws std::runtime_error for an unavailable backend.
ddlaStatus_t ddlaInit(DdlaHandle_t& handle, DdlaBackend requested_backend);
// Only a 1x1 grid is served: a communicator of more than one rank, or an
// explicit grid other than 1x1, returns DDLA_STATUS_BACKEND_UNAVAILABLE.
ddlaStatus_t ddlaSet(DdlaHandle_t handle, const MPI_Comm& comm = MPI_COMM_WORLD, char major = 'R');
ddlaStatus_t ddlaSet(DdlaHandle_t handle, const MPI_Comm& comm, int nprows, int npcols, char major = 'R');
ddlaStatus_t ddlaDestroy(DdlaHandle_t& handle);

// Process grids of more than one rank, one rank per GPU (the handle's device),
// rank -> (row, col) by `major` as ddlaRankToRc.  Every rank of the grid calls
// the distributed routines (ppotrf, ppotrs side 'L', pposv side 'L',
// pdiag_logdet) with its local block-cyclic piece and the common descriptor.
//   Local group: the ranks are threads of this process.  A collective whose
//   members do not all arrive within timeout_s seconds raises
//   std::runtime_error on the ranks that wait, and the group is then unusable.
//   NCCL: the ranks are processes; rank 0 makes the clique id with
//   ddlaNcclUniqueId and every rank passes the same 128 bytes.
struct DdlaLocalGroup;
ddlaStatus_t ddlaLocalGroupCreate(DdlaLocalGroup** group, int nranks, double timeout_s = 120.0);
ddlaStatus_t ddlaLocalGroupDestroy(DdlaLocalGroup* group);
ddlaStatus_t ddlaSetLocalGroup(DdlaHandle_t handle, DdlaLocalGroup* group, int rank, int nprows, int npcols,
                               char major = 'R');
bool ddlaNcclAvailable();
ddlaStatus_t ddlaNcclUniqueId(void* id128);
ddlaStatus_t ddlaSetNccl(DdlaHandle_t handle, const void* id128, int nranks, int rank, int nprows, int npcols,
                         char major = 'R');

bool ddlaBackendAvailable(DdlaBackend backend);
DdlaBackend ddlaGetBackend(const DdlaHandle_t& handle);
ddlaStatus_t ddlaSetCommunication(const DdlaHandle_t& handle, DdlaCommunication mode);
DdlaCommunication ddlaGetCommunication(const DdlaHandle_t& handle);
bool ddlaCommunicationAvailable(const DdlaHandle_t& handle, DdlaCommunication mode);

// Memory (device memory, ordered on the handle's stream).
using ddlaEvent_t = void*;
ddlaStatus_t ddlaMalloc(const DdlaHandle_t& handle, void** ptr, std::size_t bytes);
template <typename T>
inline ddlaStatus_t ddlaMalloc(const DdlaHandle_t& handle, T** ptr, std::size_t bytes)
{
    return ddlaMalloc(handle, reinterpret_cast<void**>(ptr), bytes);
}
ddlaStatus_t ddlaFree(const DdlaHandle_t& handle, void* ptr);
ddlaStatus_t ddlaMallocHost(const DdlaHandle_t& handle, void** ptr, std::size_t bytes);
template <typename T>
inline ddlaStatus_t ddlaMallocHost(const DdlaHandle_t& handle, T** ptr, std::size_t bytes)
{
    return ddlaMallocHost(handle, reinterpret_cast<void**>(ptr), bytes);
}
ddlaStatus_t ddlaFreeHost(const DdlaHandle_t& handle, void* ptr);
ddlaStatus_t ddlaMemcpy(const DdlaHandle_t& handle, void* dst, const void* src, std::size_t bytes);
ddlaStatus_t ddlaMemcpy2D(const DdlaHandle_t& handle, void* dst, std::size_t dpitch, const void* src,
                          std::size_t spitch, std::size_t width, std::size_t height);
ddlaStatus_t ddlaMemset(const DdlaHandle_t& handle, void* ptr, int value, std::size_t bytes);
ddlaStatus_t ddlaSynchronize(const DdlaHandle_t& handle);
ddlaStatus_t ddlaDeviceSynchronize(const DdlaHandle_t& handle);
ddlaStatus_t ddlaEventCreate(const DdlaHandle_t& handle, ddlaEvent_t* event);
ddlaStatus_t ddlaEventDestroy(const DdlaHandle_t& handle, ddlaEvent_t event);
ddlaStatus_t ddlaEventRecord(const DdlaHandle_t& handle, ddlaEvent_t event);
ddlaStatus_t ddlaEventWait(const DdlaHandle_t& handle, ddlaEvent_t event);
ddlaStatus_t ddlaEventSynchronize(const DdlaHandle_t& handle, ddlaEvent_t event);
ddlaStatus_t ddlaGetLastError(const DdlaHandle_t& handle);
ddlaStatus_t ddlaSetDevice(const DdlaHandle_t& handle);
ddlaStatus_t ddlaGetDeviceCount(const DdlaHandle_t& handle, int* count);
ddlaStatus_t ddlaMemGetInfo(const DdlaHandle_t& handle, std::size_t* free_bytes, std::size_t* total_bytes);
const char* ddlaGetErrorString(ddlaStatus_t status);
// Replace the compute stream; the handle owns the new stream afterwards and
// destroys the previous non-null one.  A null stream selects the legacy default.
ddlaStatus_t ddlaSetStream(const DdlaHandle_t& handle, void* stream);
void* ddlaGetStream(const DdlaHandle_t& handle);

// Grid accessors.  The communicators are the single-rank stand-in of this build;
// the grid itself is the handle's (1x1 after ddlaSet).
MPI_Comm ddlaGetCommunicator(const DdlaHandle_t& handle);
MPI_Comm ddlaGetRowCommunicator(const DdlaHandle_t& handle);
MPI_Comm ddlaGetColCommunicator(const DdlaHandle_t& handle);
int ddlaGetRank(const DdlaHandle_t& handle);
int ddlaGetSize(const DdlaHandle_t& handle);
void ddlaGetGridCoords(const DdlaHandle_t& handle, int& myprow, int& mypcol);
void ddlaGetGridDims(const DdlaHandle_t& handle, int& nprows, int& npcols);
void ddlaRankToRc(const DdlaHandle_t& handle, int rank, int& row, int& col);
int ddlaRcToRank(const DdlaHandle_t& handle, int row, int col);

inline void DDLA_CHECK(ddlaStatus_t status, const char* file = __builtin_FILE(), int line = __builtin_LINE())
{
    if (status != ddlaStatus_t::DDLA_STATUS_SUCCESS) {
        throw std::runtime_error(std::string("ddla error ") + std::to_string(static_cast<int>(status)) + " (" +
                                 ddlaGetErrorString(status) + ") at " + file + ":" + std::to_string(line));
    }
}

}  // namespace ddla

#endif
