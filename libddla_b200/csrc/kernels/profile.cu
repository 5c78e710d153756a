// Launch accounting and per-kernel CUDA-event timing for the kernel layer.
//
// Every launcher bumps a process-wide launch counter.  When profiling is
// switched on, launchers also bracket their kernels with CUDA events on the
// launching stream and record the algorithmic flops and bytes of that launch;
// ddlak_profile_read folds the records of one kernel kind into total device
// time, launch count, flops and bytes.  The reference has no tracing of its
// own; this is what bench.py uses for the live roofline numbers.
#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "common.cuh"
#include "profile.h"

namespace ddlak {

namespace {
std::atomic<long long> g_launches{0};
std::atomic<bool> g_on{false};
std::mutex g_mu;
struct Rec {
    int kind;
    cudaEvent_t a, b;
    double flops, bytes;
};
std::vector<Rec> g_recs;
std::vector<cudaEvent_t> g_free;

cudaEvent_t get_event()
{
    if (!g_free.empty()) {
        cudaEvent_t e = g_free.back();
        g_free.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}
}  // namespace

void note_launches(int count) { g_launches.fetch_add(count, std::memory_order_relaxed); }

bool profiling() { return g_on.load(std::memory_order_relaxed); }

namespace {
std::mutex& setter_mu()
{
    static std::mutex mu;
    return mu;
}
std::vector<cudaError_t (*)(long long)>& setters()
{
    static std::vector<cudaError_t (*)(long long)> v;
    return v;
}
std::atomic<long long> g_budget{4000000000LL};
}  // namespace

bool register_wait_budget_setter(cudaError_t (*setter)(long long))
{
    std::lock_guard<std::mutex> lk(setter_mu());
    setters().push_back(setter);
    return true;
}

cudaError_t smem_optin(const void* func, std::size_t bytes)
{
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, std::size_t> raised;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    auto it = raised.find({func, dev});
    if (it != raised.end() && it->second >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) raised[{func, dev}] = bytes;
    return e;
}

ProfScope::ProfScope(int kind, cudaStream_t st, double flops, double bytes) : st_(st), active_(profiling())
{
    if (!active_) return;
    std::lock_guard<std::mutex> lk(g_mu);
    Rec r{kind, get_event(), get_event(), flops, bytes};
    cudaEventRecord(r.a, st);
    idx_ = g_recs.size();
    g_recs.push_back(r);
}

ProfScope::~ProfScope()
{
    if (!active_) return;
    std::lock_guard<std::mutex> lk(g_mu);
    cudaEventRecord(g_recs[idx_].b, st_);
}

}  // namespace ddlak

extern "C" long long ddlak_launch_count(void) { return ddlak::g_launches.load(); }

extern "C" void ddlak_profile_enable(int on) { ddlak::g_on.store(on != 0); }

extern "C" int ddlak_profile_read(int kind, double* ms, long long* launches, double* flops, double* bytes, int reset)
{
    using namespace ddlak;
    std::lock_guard<std::mutex> lk(g_mu);
    double t = 0, f = 0, b = 0;
    long long c = 0;
    std::vector<Rec> keep;
    for (auto& r : g_recs) {
        if (kind >= 0 && r.kind != kind) {
            keep.push_back(r);
            continue;
        }
        const cudaError_t e = cudaEventSynchronize(r.b);
        if (e != cudaSuccess) return (int)e;
        float x = 0;
        cudaEventElapsedTime(&x, r.a, r.b);
        t += x;
        f += r.flops;
        b += r.bytes;
        ++c;
        if (reset) {
            g_free.push_back(r.a);
            g_free.push_back(r.b);
        } else {
            keep.push_back(r);
        }
    }
    g_recs.swap(keep);
    if (ms) *ms = t;
    if (launches) *launches = c;
    if (flops) *flops = f;
    if (bytes) *bytes = b;
    return 0;
}

// Clock budget (SM cycles) after which a kernel's flag wait gives up and
// records DDLAK_WAIT_TIMEOUT; cycles <= 0 restores the default (4e9, about
// 2 s).  Applies to the current device, for every kernel of the library.
extern "C" int ddlak_set_wait_budget(long long cycles)
{
    using namespace ddlak;
    const long long c = cycles > 0 ? cycles : kDefaultWaitBudget;
    std::lock_guard<std::mutex> lk(setter_mu());
    for (auto f : setters())
        if (cudaError_t e = f(c); e != cudaSuccess) return (int)e;
    g_budget.store(c);
    return 0;
}

extern "C" long long ddlak_get_wait_budget(void) { return ddlak::g_budget.load(); }
