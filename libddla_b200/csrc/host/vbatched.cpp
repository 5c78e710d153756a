// ddla::posvVbatched / VbatchedPlan / vbatchedAutotune (include/ddla/ddla_batched.h).
//
// Host side of the persistent batched kernel (ddlak_posv_vbatched): read the
// orders once, sort the work list by decreasing order (longest first), pick
// each matrix's block-column width from the tuning table of its order bucket,
// upload list + choices + the kernel's two work counters, and launch (directly,
// or captured once in a CUDA graph for VbatchedPlan).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include <ddla/ddla_batched.h>
#include <ddla_kernels.h>

#include "ddla_stream.h"

namespace ddla {

namespace {

constexpr int kBucket = 16;  // orders per tuning bucket

template <class T> constexpr char tcode();
template <> constexpr char tcode<float>() { return 's'; }
template <> constexpr char tcode<double>() { return 'd'; }

int nmax_for(int max_n) { return max_n <= 512 ? 512 : 1024; }

// ---- tuning tables ----------------------------------------------------------
using TuneKey = std::tuple<int, char, int>;  // device, type, nmax

std::mutex& tune_mutex()
{
    static std::mutex m;
    return m;
}
std::map<TuneKey, VbatchedTuning>& tune_tables()
{
    static std::map<TuneKey, VbatchedTuning> t;
    return t;
}
bool& tune_file_loaded()
{
    static bool loaded = false;
    return loaded;
}

const char* tune_file() { return std::getenv("DDLA_VBATCHED_TUNE_FILE"); }

// File format, one table per line:  <device> <type> <nmax> <grid> <v_0> ... <v_{nmax/16-1}>
void load_tune_file_locked()
{
    if (tune_file_loaded()) return;
    tune_file_loaded() = true;
    const char* path = tune_file();
    if (!path || !*path) return;
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    int dev, nmax, grid;
    char type;
    while (std::fscanf(f, "%d %c %d %d", &dev, &type, &nmax, &grid) == 4) {
        if ((nmax != 512 && nmax != 1024) || (type != 's' && type != 'd') || grid <= 0) break;
        VbatchedTuning tt;
        tt.nmax = nmax;
        tt.grid = grid;
        tt.variant.assign(nmax / kBucket, 0);
        bool ok = true;
        for (auto& v : tt.variant) {
            int x;
            if (std::fscanf(f, "%d", &x) != 1 || x < 0 || x > 1) { ok = false; break; }
            v = (unsigned char)x;
        }
        if (!ok) break;
        ddlak_vbatched_variants(type, nmax, tt.widths);
        tt.tuned = true;
        tune_tables()[TuneKey{dev, type, nmax}] = tt;
    }
    std::fclose(f);
}

void save_tune_file_locked()
{
    const char* path = tune_file();
    if (!path || !*path) return;
    FILE* f = std::fopen(path, "w");
    if (!f) return;
    for (const auto& kv : tune_tables()) {
        if (!kv.second.tuned) continue;
        std::fprintf(f, "%d %c %d %d", std::get<0>(kv.first), std::get<1>(kv.first), kv.second.nmax, kv.second.grid);
        for (unsigned char v : kv.second.variant) std::fprintf(f, " %d", (int)v);
        std::fprintf(f, "\n");
    }
    std::fclose(f);
}

// Built-in choice: the wider block column from order 64 up.
VbatchedTuning default_tuning(char type, int nmax)
{
    VbatchedTuning tt;
    tt.nmax = nmax;
    tt.grid = ddlak_vbatched_max_grid(type, nmax);
    if (tt.grid <= 0) throw std::runtime_error("posvVbatched: cannot size the persistent launch");
    ddlak_vbatched_variants(type, nmax, tt.widths);
    tt.variant.assign(nmax / kBucket, 0);
    for (int b = 0; b < nmax / kBucket; ++b) tt.variant[b] = (b + 1) * kBucket >= 64 ? 1 : 0;
    return tt;
}

VbatchedTuning lookup_tuning(int dev, char type, int nmax)
{
    std::lock_guard<std::mutex> lk(tune_mutex());
    load_tune_file_locked();
    auto it = tune_tables().find(TuneKey{dev, type, nmax});
    if (it != tune_tables().end()) return it->second;
    return default_tuning(type, nmax);
}

int bucket_of(int n) { return n <= 0 ? 0 : (n - 1) / kBucket; }

void check_args(const DdlaHandle_t& h, const char* routine, char uplo, const int* d_n, const void* d_A,
                const int* d_lda, const double* d_logdet, const int* d_info, int batch, int max_n)
{
    detail::require_gpu(h, routine);
    if (uplo != 'L') throw std::invalid_argument(std::string(routine) + ": only uplo 'L' is supported");
    if (batch < 0) throw std::invalid_argument(std::string(routine) + ": negative batch count");
    if (max_n < 0 || max_n > 1024) throw std::invalid_argument(std::string(routine) + ": max_n outside [0, 1024]");
    if (batch > 0 && (!d_n || !d_A || !d_lda || !d_logdet || !d_info))
        throw std::invalid_argument(std::string(routine) + ": null array");
}

}  // namespace

// ---- plan -------------------------------------------------------------------
struct VbatchedPlan::Impl {
    DdlaHandle_t h = nullptr;
    int device = 0;
    char type = 'd';
    int nmax = 512;
    int max_n = 0;
    int batch = 0;
    const int* d_n = nullptr;
    void* const* d_A = nullptr;
    const int* d_lda = nullptr;
    void* const* d_B = nullptr;
    double* d_logdet = nullptr;
    int* d_info = nullptr;
    void* dmem = nullptr;  // order | wsel | counters
    int* order = nullptr;
    unsigned char* wsel = nullptr;
    int* counters = nullptr;
    int grid = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;

    int launch(cudaStream_t st) const
    {
        return ddlak_posv_vbatched(type, nmax, batch, d_n, d_A, d_lda, d_B, d_logdet, d_info, order, wsel, counters,
                                   grid, st);
    }
};

namespace {

// Reads the orders, builds the work list and variants, uploads them into one
// device allocation (stream ordered when `ordered`, for one-shot calls).
void prepare(VbatchedPlan::Impl& p, double& flops, bool ordered)
{
    DdlaHandle_t h = p.h;
    cudaStream_t st = h->stream;
    std::vector<int> n(p.batch);
    detail::cuda_check(cudaMemcpyAsync(n.data(), p.d_n, sizeof(int) * p.batch, cudaMemcpyDeviceToHost, st),
                       "posvVbatched: order read-back");
    detail::cuda_check(cudaStreamSynchronize(st), "stream synchronisation");
    int mx = 0;
    flops = 0;
    for (int i = 0; i < p.batch; ++i) {
        if (n[i] < 0 || n[i] > 1024) throw std::invalid_argument("posvVbatched: matrix order outside [0, 1024]");
        mx = std::max(mx, n[i]);
        const double x = n[i];
        flops += x * x * x / 3.0 + x * x / 2.0 + x / 6.0 + (p.d_B ? 2.0 * x * x : 0.0);
    }
    if (mx > p.max_n) throw std::invalid_argument("posvVbatched: a matrix order exceeds max_n");
    const VbatchedTuning tt = lookup_tuning(h->device, p.type, p.nmax);
    p.grid = std::min(tt.grid, std::max(1, p.batch));
    std::vector<int> order(p.batch);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return n[a] > n[b]; });
    std::vector<unsigned char> wsel(p.batch);
    for (int i = 0; i < p.batch; ++i) wsel[i] = tt.variant[std::min<int>(bucket_of(n[i]), (int)tt.variant.size() - 1)];

    const size_t ob = detail::padded_bytes<int>(p.batch), wb = detail::padded_bytes<unsigned char>(p.batch),
                 cb = detail::padded_bytes<int>(2);
    if (ordered)
        detail::cuda_check(cudaMallocAsync(&p.dmem, ob + wb + cb, st), "posvVbatched: work list allocation");
    else
        detail::cuda_check(cudaMalloc(&p.dmem, ob + wb + cb), "posvVbatched: work list allocation");
    char* c = static_cast<char*>(p.dmem);
    p.order = reinterpret_cast<int*>(c);
    p.wsel = reinterpret_cast<unsigned char*>(c + ob);
    p.counters = reinterpret_cast<int*>(c + ob + wb);
    // pageable sources: the copies complete before the calls return
    detail::cuda_check(cudaMemcpyAsync(p.order, order.data(), sizeof(int) * p.batch, cudaMemcpyHostToDevice, st),
                       "posvVbatched: work list upload");
    detail::cuda_check(cudaMemcpyAsync(p.wsel, wsel.data(), p.batch, cudaMemcpyHostToDevice, st),
                       "posvVbatched: work list upload");
    detail::cuda_check(cudaMemsetAsync(p.counters, 0, sizeof(int) * 2, st), "posvVbatched: counters");
}

template <class T>
VbatchedPlan::Impl make_impl(const DdlaHandle_t& h, const int* d_n, T* const* d_A, const int* d_lda, T* const* d_B,
                             double* d_logdet, int* d_info, int batch, int max_n)
{
    VbatchedPlan::Impl p;
    p.h = h;
    p.device = h->device;
    p.type = tcode<T>();
    p.nmax = nmax_for(max_n);
    p.max_n = max_n;
    p.batch = batch;
    p.d_n = d_n;
    p.d_A = reinterpret_cast<void* const*>(d_A);
    p.d_lda = d_lda;
    p.d_B = reinterpret_cast<void* const*>(d_B);
    p.d_logdet = d_logdet;
    p.d_info = d_info;
    return p;
}

}  // namespace

template <typename T>
void posvVbatched(const DdlaHandle_t& h, char uplo, const int* d_n, T* const* d_A, const int* d_lda, T* const* d_B,
                  double* d_logdet, int* d_info, int batch, int max_n)
{
    check_args(h, "posvVbatched", uplo, d_n, d_A, d_lda, d_logdet, d_info, batch, max_n);
    if (batch == 0) return;
    VbatchedPlan::Impl p = make_impl<T>(h, d_n, d_A, d_lda, d_B, d_logdet, d_info, batch, max_n);
    double flops = 0;
    prepare(p, flops, true);
    const int e = p.launch(h->stream);
    cudaFreeAsync(p.dmem, h->stream);
    detail::kernel_check(e, "posvVbatched: launch");
}

template <typename T>
VbatchedPlan* VbatchedPlan::create(const DdlaHandle_t& h, char uplo, const int* d_n, T* const* d_A, const int* d_lda,
                                   T* const* d_B, double* d_logdet, int* d_info, int batch, int max_n)
{
    check_args(h, "VbatchedPlan", uplo, d_n, d_A, d_lda, d_logdet, d_info, batch, max_n);
    // owned until returned: any throw below releases the plan and what it holds
    std::unique_ptr<VbatchedPlan> plan(new VbatchedPlan());
    plan->impl_ = new Impl(make_impl<T>(h, d_n, d_A, d_lda, d_B, d_logdet, d_info, batch, max_n));
    Impl& p = *plan->impl_;
    {
        if (batch > 0) {
            prepare(p, plan->flops_, false);
            detail::cuda_check(cudaStreamSynchronize(h->stream), "stream synchronisation");
            // sets the kernel's shared-memory attribute outside the capture
            if (ddlak_vbatched_max_grid(p.type, p.nmax) <= 0)
                throw std::runtime_error("VbatchedPlan: cannot size the persistent launch");
            cudaStream_t cs = nullptr;
            detail::cuda_check(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "capture stream");
            cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                const int le = p.launch(cs);
                e = cudaStreamEndCapture(cs, &p.graph);
                if (le != 0 && e == cudaSuccess) e = static_cast<cudaError_t>(le);
            }
            cudaStreamDestroy(cs);
            detail::cuda_check(e, "VbatchedPlan: graph capture");
            detail::cuda_check(cudaGraphInstantiate(&p.exec, p.graph, 0), "VbatchedPlan: graph instantiation");
        }
        plan->grid_ = p.grid;
    }
    return plan.release();
}

void VbatchedPlan::run()
{
    if (!impl_ || impl_->batch == 0) return;
    detail::cuda_check(cudaSetDevice(impl_->h->device), "cudaSetDevice");
    detail::cuda_check(cudaGraphLaunch(impl_->exec, impl_->h->stream), "VbatchedPlan: graph launch");
}

VbatchedPlan::~VbatchedPlan()
{
    if (!impl_) return;
    if (impl_->exec) cudaGraphExecDestroy(impl_->exec);
    if (impl_->graph) cudaGraphDestroy(impl_->graph);
    // the handle may be gone by now: touch only the device (cudaFree waits for
    // the device's work, so a replay still in flight finishes first)
    if (impl_->dmem) {
        cudaSetDevice(impl_->device);
        cudaFree(impl_->dmem);
    }
    delete impl_;
}

// ---- autotuner -----------------------------------------------------------------
namespace {

// Times one launch configuration over a synthetic batch: median of `reps`.
template <class T>
float time_batch(const DdlaHandle_t& h, int nmax, int order, int count, int variant, int grid, T** d_ptrs,
                 T* d_mats, T* d_b, int* d_n, int* d_lda, double* d_logdet, int* d_info, unsigned char* d_wsel,
                 int* d_counters, int reps)
{
    cudaStream_t st = h->stream;
    std::vector<int> n(count, order), lda(count, order);
    std::vector<T*> ptrs(2 * count);
    for (int i = 0; i < count; ++i) {
        ptrs[i] = d_mats + (size_t)i * order * order;
        ptrs[count + i] = d_b + (size_t)i * order;
    }
    std::vector<unsigned char> ws(count, (unsigned char)variant);
    detail::cuda_check(cudaMemcpyAsync(d_n, n.data(), sizeof(int) * count, cudaMemcpyHostToDevice, st), "tune");
    detail::cuda_check(cudaMemcpyAsync(d_lda, lda.data(), sizeof(int) * count, cudaMemcpyHostToDevice, st), "tune");
    detail::cuda_check(cudaMemcpyAsync(d_ptrs, ptrs.data(), sizeof(T*) * 2 * count, cudaMemcpyHostToDevice, st),
                       "tune");
    detail::cuda_check(cudaMemcpyAsync(d_wsel, ws.data(), count, cudaMemcpyHostToDevice, st), "tune");
    detail::cuda_check(cudaStreamSynchronize(st), "stream synchronisation");
    struct Events {  // destroyed on every exit, a throw included
        cudaEvent_t e[2] = {nullptr, nullptr};
        ~Events()
        {
            for (cudaEvent_t x : e)
                if (x) cudaEventDestroy(x);
        }
    } ev;
    detail::cuda_check(cudaEventCreate(&ev.e[0]), "tune event");
    detail::cuda_check(cudaEventCreate(&ev.e[1]), "tune event");
    cudaEvent_t e0 = ev.e[0], e1 = ev.e[1];
    std::vector<float> ms;
    for (int r = 0; r < reps + 1; ++r) {
        detail::kernel_check(ddlak_fill_spd_vbatched(tcode<T>(), count, d_n, reinterpret_cast<void* const*>(d_ptrs),
                                                     d_lda, reinterpret_cast<void* const*>(d_ptrs + count), st),
                             "tune fill");
        detail::cuda_check(cudaEventRecord(e0, st), "tune event");
        detail::kernel_check(ddlak_posv_vbatched(tcode<T>(), nmax, count, d_n, reinterpret_cast<void* const*>(d_ptrs),
                                                 d_lda, reinterpret_cast<void* const*>(d_ptrs + count), d_logdet,
                                                 d_info, nullptr, d_wsel, d_counters, grid, st),
                             "tune launch");
        detail::cuda_check(cudaEventRecord(e1, st), "tune event");
        detail::cuda_check(cudaEventSynchronize(e1), "tune event");
        float t = 0;
        detail::cuda_check(cudaEventElapsedTime(&t, e0, e1), "tune event");
        if (r > 0) ms.push_back(t);  // first run warms up
    }
    std::sort(ms.begin(), ms.end());
    return ms[ms.size() / 2];
}

template <class T>
VbatchedTuning autotune_typed(const DdlaHandle_t& h, int nmax)
{
    VbatchedTuning tt = default_tuning(tcode<T>(), nmax);
    int dev = h->device, sms = 0;
    detail::cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    const int maxgrid = tt.grid;
    // enough matrices for a few waves of the largest grid
    const int count = 3 * maxgrid;
    const size_t mat_elems = (size_t)count * nmax * nmax;
    // the three buffers are freed on every exit, a throw included
    struct DeviceBuffers {
        void* p[3] = {nullptr, nullptr, nullptr};
        ~DeviceBuffers()
        {
            for (void* q : p)
                if (q) cudaFree(q);
        }
    } bufs;
    const size_t sb = sizeof(T*) * 2 * count + sizeof(int) * 2 * count + sizeof(double) * count + sizeof(int) * count +
                      count + 64;
    detail::cuda_check(cudaMalloc(&bufs.p[0], sizeof(T) * mat_elems), "tune allocation");
    detail::cuda_check(cudaMalloc(&bufs.p[1], sizeof(T) * (size_t)count * nmax), "tune allocation");
    detail::cuda_check(cudaMalloc(&bufs.p[2], sb + 256), "tune allocation");
    T* d_mats = static_cast<T*>(bufs.p[0]);
    T* d_b = static_cast<T*>(bufs.p[1]);
    char* small = static_cast<char*>(bufs.p[2]);
    char* c = small;
    T** d_ptrs = reinterpret_cast<T**>(c);
    c += sizeof(T*) * 2 * count;
    int* d_n = reinterpret_cast<int*>(c);
    c += sizeof(int) * count;
    int* d_lda = reinterpret_cast<int*>(c);
    c += sizeof(int) * count;
    double* d_logdet = reinterpret_cast<double*>(c);
    c += sizeof(double) * count;
    int* d_info = reinterpret_cast<int*>(c);
    c += sizeof(int) * count;
    int* d_counters = reinterpret_cast<int*>(c);
    c += 16;
    unsigned char* d_wsel = reinterpret_cast<unsigned char*>(c);
    detail::cuda_check(cudaMemset(d_counters, 0, 16), "tune counters");
    {
        // grid: time a mid-size order at one CTA per SM and at full residency
        if (maxgrid > sms) {
            const int mid = std::min(nmax, 256);
            const float tf = time_batch<T>(h, nmax, mid, count, 1, maxgrid, d_ptrs, d_mats, d_b, d_n, d_lda, d_logdet,
                                           d_info, d_wsel, d_counters, 3);
            const float t1 = time_batch<T>(h, nmax, mid, count, 1, sms, d_ptrs, d_mats, d_b, d_n, d_lda, d_logdet,
                                           d_info, d_wsel, d_counters, 3);
            tt.grid = t1 < tf ? sms : maxgrid;
        }
        for (int b = 0; b < nmax / kBucket; ++b) {
            const int order = b * kBucket + kBucket;  // the bucket's largest order
            const float t0 = time_batch<T>(h, nmax, order, count, 0, tt.grid, d_ptrs, d_mats, d_b, d_n, d_lda,
                                           d_logdet, d_info, d_wsel, d_counters, 3);
            const float t1 = time_batch<T>(h, nmax, order, count, 1, tt.grid, d_ptrs, d_mats, d_b, d_n, d_lda,
                                           d_logdet, d_info, d_wsel, d_counters, 3);
            tt.variant[b] = t1 < t0 ? 1 : 0;
        }
    }
    tt.tuned = true;
    return tt;
}

}  // namespace

void vbatchedAutotune(const DdlaHandle_t& h, char type, int max_n)
{
    detail::require_gpu(h, "vbatchedAutotune");
    if (type != 's' && type != 'd') throw std::invalid_argument("vbatchedAutotune: type must be 's' or 'd'");
    if (max_n < 1 || max_n > 1024) throw std::invalid_argument("vbatchedAutotune: max_n outside [1, 1024]");
    const int nmax = nmax_for(max_n);
    detail::cuda_check(cudaStreamSynchronize(h->stream), "stream synchronisation");
    VbatchedTuning tt = type == 'd' ? autotune_typed<double>(h, nmax) : autotune_typed<float>(h, nmax);
    std::lock_guard<std::mutex> lk(tune_mutex());
    load_tune_file_locked();
    tune_tables()[TuneKey{h->device, type, nmax}] = tt;
    save_tune_file_locked();
}

VbatchedTuning vbatchedTuning(const DdlaHandle_t& h, char type, int max_n)
{
    detail::require_gpu(h, "vbatchedTuning");
    if (type != 's' && type != 'd') throw std::invalid_argument("vbatchedTuning: type must be 's' or 'd'");
    if (max_n < 0 || max_n > 1024) throw std::invalid_argument("vbatchedTuning: max_n outside [0, 1024]");
    return lookup_tuning(h->device, type, nmax_for(max_n));
}

#define DDLA_VB_INST(T)                                                                                          \
    template void posvVbatched<T>(const DdlaHandle_t&, char, const int*, T* const*, const int*, T* const*,       \
                                  double*, int*, int, int);                                                      \
    template VbatchedPlan* VbatchedPlan::create<T>(const DdlaHandle_t&, char, const int*, T* const*, const int*, \
                                                   T* const*, double*, int*, int, int);
DDLA_VB_INST(float)
DDLA_VB_INST(double)
#undef DDLA_VB_INST

}  // namespace ddla
