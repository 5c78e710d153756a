// Communication among the ranks of a P x Q process grid, one rank per GPU.
//
// The reference moves panels with MPI_Bcast / ncclBcast over the row and column
// communicators of its handle (src/comm_traits.h:45-56 -> src/communicator.cpp:246)
// and sums with MPI_Allreduce.  Here a grid handle owns a GridComm with the two
// collectives the distributed Cholesky and triangular solve need, both
// stream-ordered on the caller's stream:
//   bcast      -- the root's bytes into every member's buffer;
//   reduce_sum -- the element-wise sum of every member's reals into the root's
//                 buffer (the other members' buffers are left unchanged).
// Every member of a scope calls a collective with the same arguments except
// the buffer, in the same order.  Scopes: Row = the ranks of this rank's process
// row (member index = process column), Col = the ranks of its process column
// (member index = process row), All = every rank (member index = rank).
//
// Two implementations:
//   LocalGroupComm -- ranks that are threads of one process (one thread per GPU,
//                     or several ranks sharing a GPU): the transfers are
//                     cudaMemcpyPeerAsync between the members' buffers, ordered
//                     by CUDA events, so no kernel of one rank ever waits on
//                     another rank's kernel; the host rendezvous is bounded
//                     by a timeout (an absent rank raises instead of hanging).
//   NcclComm       -- ranks that are processes: NCCL (loaded at run time from
//                     libnccl.so.2) over a world communicator and its row and
//                     column splits.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <memory>

namespace ddla {
namespace detail {

enum class Scope : int { Row = 0, Col = 1, All = 2 };

class GridComm {
public:
    virtual ~GridComm() = default;
    virtual void bcast(Scope s, int root, void* buf, std::size_t bytes, cudaStream_t st) = 0;
    // real_type 's' (float) or 'd' (double); complex data is summed as pairs of reals
    virtual void reduce_sum(Scope s, int root, void* buf, std::size_t count, char real_type, cudaStream_t st) = 0;
    virtual const char* kind() const = 0;
};

// An in-process group of nranks ranks (opaque; shared by the members' handles).
struct LocalGroup;
std::shared_ptr<LocalGroup> make_local_group(int nranks, double timeout_s);
int local_group_size(const LocalGroup& group);
// The communicator of member `rank` of `group`, on a P x Q grid, rank -> (row, col) by `major`.
std::unique_ptr<GridComm> make_local_comm(std::shared_ptr<LocalGroup> group, int rank, int nprows, int npcols,
                                          char major, int device);

// NCCL: true when libnccl.so.2 loads and has every entry point used here.
bool nccl_available();
// 128-byte ncclUniqueId of a new clique (rank 0 makes it, the caller distributes it).
void nccl_unique_id(void* out128);
std::unique_ptr<GridComm> make_nccl_comm(const void* id128, int nranks, int rank, int nprows, int npcols, char major,
                                         int device);

}  // namespace detail
}  // namespace ddla
