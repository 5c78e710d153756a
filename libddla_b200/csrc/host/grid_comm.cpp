// GridComm implementations: an in-process group of ranks (threads) and NCCL.
#include "grid_comm.h"

#include <dlfcn.h>
#include <nccl.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include <ddla_kernels.h>

#include "ddla_stream.h"

namespace ddla {
namespace detail {

namespace {

void rank_rc(int rank, int P, int Q, char major, int& row, int& col)
{
    if (major == 'C') {
        row = rank % P;
        col = rank / P;
    } else {
        row = rank / Q;
        col = rank % Q;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// In-process group
// ---------------------------------------------------------------------------
struct LocalGroup {
    struct Part {
        const void* ptr;
        int dev;
        cudaEvent_t ready;
    };
    struct Slot {
        long gen = 0;
        int arrived = 0;
        bool root_in = false;
        const void* src = nullptr;
        int src_dev = 0;
        cudaEvent_t ready = nullptr;
        cudaEvent_t consumed = nullptr;
        std::vector<cudaEvent_t> dones;
        std::vector<Part> parts;
    };
    int nranks = 0;
    std::chrono::duration<double> timeout{120.0};
    std::mutex m;
    std::condition_variable cv;
    std::map<long long, Slot> slots;
    bool broken = false;
};

std::shared_ptr<LocalGroup> make_local_group(int nranks, double timeout_s)
{
    if (nranks < 1) throw std::invalid_argument("ddla grid: a local group needs at least one rank");
    auto g = std::make_shared<LocalGroup>();
    g->nranks = nranks;
    if (timeout_s > 0) g->timeout = std::chrono::duration<double>(timeout_s);
    return g;
}

int local_group_size(const LocalGroup& group) { return group.nranks; }

namespace {

class LocalGroupComm final : public GridComm {
public:
    LocalGroupComm(std::shared_ptr<LocalGroup> g, int rank, int P, int Q, char major, int dev)
        : g_(std::move(g)), rank_(rank), P_(P), Q_(Q), dev_(dev)
    {
        rank_rc(rank, P, Q, major, row_, col_);
        cuda_check(cudaEventCreateWithFlags(&ev_a_, cudaEventDisableTiming), "grid event");
        cuda_check(cudaEventCreateWithFlags(&ev_b_, cudaEventDisableTiming), "grid event");
    }
    ~LocalGroupComm() override
    {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(dev_);
        cudaEventDestroy(ev_a_);
        cudaEventDestroy(ev_b_);
        cudaSetDevice(prev);
    }
    const char* kind() const override { return "local"; }

    void bcast(Scope s, int root, void* buf, std::size_t bytes, cudaStream_t st) override
    {
        int members = 0, me = 0;
        long long key = scope_key(s, members, me);
        if (members == 1 || bytes == 0) return;
        std::unique_lock<std::mutex> lk(g_->m);
        LocalGroup::Slot& slot = g_->slots[key];
        const long my = gen_[key]++;
        wait(lk, [&] { return slot.gen == my; }, "bcast entry");
        if (me == root) {
            cuda_check(cudaEventRecord(ev_a_, st), "grid bcast record");
            slot.src = buf;
            slot.src_dev = dev_;
            slot.ready = ev_a_;
            slot.root_in = true;
            slot.arrived++;
            g_->cv.notify_all();
            wait(lk, [&] { return slot.arrived == members; }, "bcast receivers");
            for (cudaEvent_t e : slot.dones) cuda_check(cudaStreamWaitEvent(st, e, 0), "grid bcast join");
            slot.dones.clear();
            slot.arrived = 0;
            slot.root_in = false;
            slot.gen++;
            g_->cv.notify_all();
        } else {
            wait(lk, [&] { return slot.root_in; }, "bcast root");
            cuda_check(cudaStreamWaitEvent(st, slot.ready, 0), "grid bcast wait");
            cuda_check(cudaMemcpyPeerAsync(buf, dev_, slot.src, slot.src_dev, bytes, st), "grid bcast copy");
            cuda_check(cudaEventRecord(ev_b_, st), "grid bcast record");
            slot.dones.push_back(ev_b_);
            slot.arrived++;
            g_->cv.notify_all();
            // stay until the root has ordered its stream after every copy, so
            // that this rank's event is not re-recorded before the root used it
            wait(lk, [&] { return slot.gen > my; }, "bcast completion");
        }
    }

    void reduce_sum(Scope s, int root, void* buf, std::size_t count, char real_type, cudaStream_t st) override
    {
        if (real_type != 's' && real_type != 'd') throw std::invalid_argument("ddla grid: reduce of an unknown type");
        int members = 0, me = 0;
        long long key = scope_key(s, members, me);
        if (members == 1 || count == 0) return;
        const std::size_t bytes = count * (real_type == 's' ? 4 : 8);
        std::unique_lock<std::mutex> lk(g_->m);
        LocalGroup::Slot& slot = g_->slots[key];
        const long my = gen_[key]++;
        wait(lk, [&] { return slot.gen == my; }, "reduce entry");
        if (me == root) {
            slot.arrived++;
            wait(lk, [&] { return slot.arrived == members; }, "reduce contributions");
            void* stage = nullptr;
            cuda_check(cudaMallocAsync(&stage, bytes, st), "grid reduce staging");
            for (const LocalGroup::Part& p : slot.parts) {
                cuda_check(cudaStreamWaitEvent(st, p.ready, 0), "grid reduce wait");
                cuda_check(cudaMemcpyPeerAsync(stage, dev_, p.ptr, p.dev, bytes, st), "grid reduce copy");
                kernel_check(ddlak_grid_accumulate(real_type, count, stage, buf, st), "grid reduce sum");
            }
            cuda_check(cudaFreeAsync(stage, st), "grid reduce staging");
            cuda_check(cudaEventRecord(ev_a_, st), "grid reduce record");
            slot.consumed = ev_a_;
            slot.parts.clear();
            slot.arrived = 0;
            slot.gen++;
            g_->cv.notify_all();
        } else {
            cuda_check(cudaEventRecord(ev_b_, st), "grid reduce record");
            slot.parts.push_back({buf, dev_, ev_b_});
            slot.arrived++;
            g_->cv.notify_all();
            wait(lk, [&] { return slot.gen > my; }, "reduce completion");
            // the contribution stays untouched until the root's copies have run
            cuda_check(cudaStreamWaitEvent(st, slot.consumed, 0), "grid reduce join");
        }
    }

private:
    long long scope_key(Scope s, int& members, int& me) const
    {
        switch (s) {
        case Scope::Row: members = Q_; me = col_; return (long long)row_;
        case Scope::Col: members = P_; me = row_; return (1LL << 32) + col_;
        default: members = P_ * Q_; me = rank_; return 2LL << 32;
        }
    }
    template <class Pred>
    void wait(std::unique_lock<std::mutex>& lk, Pred pred, const char* what)
    {
        const bool ok = g_->cv.wait_for(lk, g_->timeout, [&] { return g_->broken || pred(); });
        if (ok && !g_->broken) return;
        if (ok && pred()) return;
        g_->broken = true;
        g_->cv.notify_all();
        throw std::runtime_error(std::string("ddla grid: ") +
                                 (ok ? "an earlier collective of the group failed" : "collective timed out") +
                                 " (" + what + ", rank " + std::to_string(rank_) + ")");
    }

    std::shared_ptr<LocalGroup> g_;
    int rank_, P_, Q_, row_ = 0, col_ = 0, dev_;
    std::map<long long, long> gen_;
    cudaEvent_t ev_a_ = nullptr, ev_b_ = nullptr;
};

}  // namespace

std::unique_ptr<GridComm> make_local_comm(std::shared_ptr<LocalGroup> group, int rank, int nprows, int npcols,
                                          char major, int device)
{
    if (!group) throw std::invalid_argument("ddla grid: null local group");
    if (nprows * npcols != group->nranks || rank < 0 || rank >= group->nranks)
        throw std::invalid_argument("ddla grid: rank or grid does not match the local group");
    return std::make_unique<LocalGroupComm>(std::move(group), rank, nprows, npcols, major, device);
}

// ---------------------------------------------------------------------------
// NCCL, loaded at run time
// ---------------------------------------------------------------------------
namespace {

struct NcclApi {
    bool ok = false;
    ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
    ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*comm_split)(ncclComm_t, int, int, ncclComm_t*, ncclConfig_t*) = nullptr;
    ncclResult_t (*broadcast)(const void*, void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*reduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, int, ncclComm_t,
                           cudaStream_t) = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
    const char* (*error_string)(ncclResult_t) = nullptr;
};

const NcclApi& nccl()
{
    static NcclApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        void* lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!lib) return;
        auto sym = [&](auto& fn, const char* name) {
            fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(lib, name));
            return fn != nullptr;
        };
        api.ok = sym(api.get_unique_id, "ncclGetUniqueId") && sym(api.comm_init_rank, "ncclCommInitRank") &&
                 sym(api.comm_split, "ncclCommSplit") && sym(api.broadcast, "ncclBroadcast") &&
                 sym(api.reduce, "ncclReduce") && sym(api.comm_destroy, "ncclCommDestroy") &&
                 sym(api.error_string, "ncclGetErrorString");
    });
    return api;
}

void nccl_check(ncclResult_t r, const char* what)
{
    if (r != ncclSuccess)
        throw std::runtime_error(std::string("ddla grid: ") + what + ": " + nccl().error_string(r));
}

class NcclComm final : public GridComm {
public:
    NcclComm(const void* id128, int nranks, int rank, int P, int Q, char major) : P_(P), Q_(Q)
    {
        const NcclApi& a = nccl();
        if (!a.ok) throw std::runtime_error("ddla grid: libnccl.so.2 is not available");
        rank_rc(rank, P, Q, major, row_, col_);
        ncclUniqueId id;
        std::memcpy(&id, id128, sizeof id);
        nccl_check(a.comm_init_rank(&world_, nranks, id, rank), "ncclCommInitRank");
        nccl_check(a.comm_split(world_, row_, col_, &row_comm_, nullptr), "ncclCommSplit (row)");
        nccl_check(a.comm_split(world_, col_, row_, &col_comm_, nullptr), "ncclCommSplit (column)");
    }
    ~NcclComm() override
    {
        const NcclApi& a = nccl();
        if (row_comm_) a.comm_destroy(row_comm_);
        if (col_comm_) a.comm_destroy(col_comm_);
        if (world_) a.comm_destroy(world_);
    }
    const char* kind() const override { return "nccl"; }
    void bcast(Scope s, int root, void* buf, std::size_t bytes, cudaStream_t st) override
    {
        if (bytes == 0 || members(s) == 1) return;
        nccl_check(nccl().broadcast(buf, buf, bytes, ncclInt8, root, comm(s), st), "ncclBroadcast");
    }
    void reduce_sum(Scope s, int root, void* buf, std::size_t count, char real_type, cudaStream_t st) override
    {
        if (count == 0 || members(s) == 1) return;
        nccl_check(nccl().reduce(buf, buf, count, real_type == 's' ? ncclFloat32 : ncclFloat64, ncclSum, root,
                                 comm(s), st),
                   "ncclReduce");
    }

private:
    int members(Scope s) const { return s == Scope::Row ? Q_ : s == Scope::Col ? P_ : P_ * Q_; }
    ncclComm_t comm(Scope s) const { return s == Scope::Row ? row_comm_ : s == Scope::Col ? col_comm_ : world_; }
    int P_, Q_, row_ = 0, col_ = 0;
    ncclComm_t world_ = nullptr, row_comm_ = nullptr, col_comm_ = nullptr;
};

}  // namespace

bool nccl_available() { return nccl().ok; }

void nccl_unique_id(void* out128)
{
    const NcclApi& a = nccl();
    if (!a.ok) throw std::runtime_error("ddla grid: libnccl.so.2 is not available");
    ncclUniqueId id;
    nccl_check(a.get_unique_id(&id), "ncclGetUniqueId");
    std::memcpy(out128, &id, sizeof id);
}

std::unique_ptr<GridComm> make_nccl_comm(const void* id128, int nranks, int rank, int nprows, int npcols, char major,
                                         int device)
{
    if (nprows * npcols != nranks || rank < 0 || rank >= nranks)
        throw std::invalid_argument("ddla grid: rank or grid does not match the NCCL clique");
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    return std::make_unique<NcclComm>(id128, nranks, rank, nprows, npcols, major);
}

}  // namespace detail
}  // namespace ddla
