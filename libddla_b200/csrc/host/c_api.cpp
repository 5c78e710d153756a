// C ABI over the ddla C++ API (declarations and reference citations in
// include/ddla_c.h).  Status codes and the exception-to-status wrapper follow
// the reference's generated shim (fortran/ddla_c_api.cpp:44-98).
#include <cuda_runtime.h>

#include <complex>
#include <cstring>
#include <exception>
#include <string>

#include <ddla/ddla.h>
#include <ddla/ddla_batched.h>
#include <ddla_c.h>
#include <ddla_kernels.h>

#include "ddla_stream.h"

namespace {

enum {
    ST_SUCCESS = 0,
    ST_INVALID_HANDLE = 1,
    ST_INVALID_VALUE = 2,
    ST_ALLOC_FAILED = 3,
    ST_BACKEND_UNAVAILABLE = 4,
    ST_INTERNAL_ERROR = 5,
    ST_EXCEPTION = 6
};

thread_local std::string g_last_error;

void record(const char* what)
{
    try {
        g_last_error = what ? what : "";
    } catch (...) {
        g_last_error.clear();
    }
}

template <typename F>
int guarded(const char* name, F&& body)
{
    try {
        return body();
    } catch (const std::exception& e) {
        record(e.what());
        return ST_EXCEPTION;
    } catch (...) {
        record((std::string("unknown C++ exception in ") + name).c_str());
        return ST_EXCEPTION;
    }
}

template <typename F>
int run(void* handle, F&& body)
{
    if (handle == nullptr) return ST_INVALID_HANDLE;
    return guarded("a ddla C API call", [&]() -> int {
        const ddla::DdlaHandle_t h = static_cast<ddla::DdlaHandle_t>(handle);
        const auto be = ddla::ddlaGetBackend(h);
        if (be != ddla::DdlaBackend::CPU && be != ddla::DdlaBackend::GPU) return ST_INVALID_VALUE;
        if (!ddla::ddlaBackendAvailable(be)) return ST_BACKEND_UNAVAILABLE;
        return body(h);
    });
}

ddla::DdlaHandle_t H(void* p) { return static_cast<ddla::DdlaHandle_t>(p); }

template <class T>
int gather_impl(void* handle, int m, int n, const void* A, int ia, int ja, const int* descA, int root, void* dst,
                int lddst)
{
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        ddla::detail::check_desc(descA, h);
        if (m < 0 || n < 0 || ia < 1 || ja < 1 || ia - 1 + m > descA[ddla::DDLA_M_] || ja - 1 + n > descA[ddla::DDLA_N_])
            throw std::invalid_argument("gather: invalid extents or offsets");
        if (h->nprocs > 1)
            throw std::invalid_argument("gather: served on a 1x1 grid only (on a grid every rank copies its local piece)");
        if (root != 0) throw std::invalid_argument("gather: root outside the 1x1 grid");
        if (m == 0 || n == 0) return ST_SUCCESS;
        if (!A || !dst || lddst < m) throw std::invalid_argument("gather: null pointer or short leading dimension");
        const long long lld = descA[ddla::DDLA_LLD_];
        const T* src = static_cast<const T*>(A) + (ia - 1) + (long long)(ja - 1) * lld;
        ddla::DDLA_CHECK(ddla::ddlaMemcpy2D(h, dst, (size_t)lddst * sizeof(T), src, (size_t)lld * sizeof(T),
                                            (size_t)m * sizeof(T), (size_t)n));
        ddla::DDLA_CHECK(ddla::ddlaSynchronize(h));
        return ST_SUCCESS;
    });
}

template <class T>
int scatter_impl(void* handle, int m, int n, void* A, int ia, int ja, const int* descA, int root, const void* src,
                 int ldsrc)
{
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        ddla::detail::check_desc(descA, h);
        if (m < 0 || n < 0 || ia < 1 || ja < 1 || ia - 1 + m > descA[ddla::DDLA_M_] || ja - 1 + n > descA[ddla::DDLA_N_])
            throw std::invalid_argument("scatter: invalid extents or offsets");
        if (h->nprocs > 1)
            throw std::invalid_argument("scatter: served on a 1x1 grid only (on a grid every rank copies its local piece)");
        if (root != 0) throw std::invalid_argument("scatter: root outside the 1x1 grid");
        if (m == 0 || n == 0) return ST_SUCCESS;
        if (!A || !src || ldsrc < m) throw std::invalid_argument("scatter: null pointer or short leading dimension");
        const long long lld = descA[ddla::DDLA_LLD_];
        T* dst = static_cast<T*>(A) + (ia - 1) + (long long)(ja - 1) * lld;
        ddla::DDLA_CHECK(ddla::ddlaMemcpy2D(h, dst, (size_t)lld * sizeof(T), src, (size_t)ldsrc * sizeof(T),
                                            (size_t)m * sizeof(T), (size_t)n));
        ddla::DDLA_CHECK(ddla::ddlaSynchronize(h));
        return ST_SUCCESS;
    });
}

template <class T>
int diag_logdet_impl(void* handle, int n, const void* A, int lda, void* result)
{
    using R = ddla::real_type_t<T>;
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        if (result == nullptr) return ST_INVALID_VALUE;
        std::complex<R> r;
        std::memcpy(&r, result, sizeof(r));
        ddla::diag_logdet<T>(h, n, static_cast<const T*>(A), lda, r);
        std::memcpy(result, &r, sizeof(r));
        return ST_SUCCESS;
    });
}

template <class T>
int pdiag_logdet_impl(void* handle, int n, const void* A, const int* descA, void* result)
{
    using R = ddla::real_type_t<T>;
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        if (result == nullptr) return ST_INVALID_VALUE;
        std::complex<R> r;
        std::memcpy(&r, result, sizeof(r));
        ddla::pdiag_logdet<T>(h, n, static_cast<const T*>(A), descA, r);
        std::memcpy(result, &r, sizeof(r));
        return ST_SUCCESS;
    });
}

template <class T>
int pdiag_logdet_local_impl(void* handle, int n, const void* A, const int* descA, int pr, int pc, int row, int col,
                            double* state)
{
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        if (state == nullptr) return ST_INVALID_VALUE;
        ddla::pdiag_logdet_local<T>(h, n, static_cast<const T*>(A), descA, pr, pc, row, col, state);
        return ST_SUCCESS;
    });
}

template <class T>
int gemm_vbatched_impl(void* handle, char ta, char tb, int* d_m, int* d_n, int* d_k, const void* alpha,
                       const void* const* d_A, int* d_lda, const void* const* d_B, int* d_ldb, const void* beta,
                       void** d_C, int* d_ldc, int batch_count)
{
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        if (alpha == nullptr || beta == nullptr) return ST_INVALID_VALUE;
        T al, be;
        std::memcpy(&al, alpha, sizeof(T));
        std::memcpy(&be, beta, sizeof(T));
        ddla::gemmVbatched<T>(h, ta, tb, d_m, d_n, d_k, al, reinterpret_cast<const T* const*>(d_A), d_lda,
                              reinterpret_cast<const T* const*>(d_B), d_ldb, be, reinterpret_cast<T**>(d_C), d_ldc,
                              batch_count);
        return ST_SUCCESS;
    });
}

template <class R, bool ComplexLeft>
int gemm_vbatched_mixed_impl(void* handle, char ta, char tb, int* d_m, int* d_n, int* d_k, const void* alpha,
                             const void* const* d_A, int* d_lda, const void* const* d_B, int* d_ldb,
                             const void* beta, void** d_C, int* d_ldc, int batch_count)
{
    using Z = std::complex<R>;
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        if (alpha == nullptr || beta == nullptr) return ST_INVALID_VALUE;
        Z al, be;
        std::memcpy(&al, alpha, sizeof(Z));
        std::memcpy(&be, beta, sizeof(Z));
        if constexpr (ComplexLeft)
            ddla::gemmVbatched<R>(h, ta, tb, d_m, d_n, d_k, al, reinterpret_cast<const Z* const*>(d_A), d_lda,
                                  reinterpret_cast<const R* const*>(d_B), d_ldb, be, reinterpret_cast<Z**>(d_C), d_ldc,
                                  batch_count);
        else
            ddla::gemmVbatched<R>(h, ta, tb, d_m, d_n, d_k, al, reinterpret_cast<const R* const*>(d_A), d_lda,
                                  reinterpret_cast<const Z* const*>(d_B), d_ldb, be, reinterpret_cast<Z**>(d_C), d_ldc,
                                  batch_count);
        return ST_SUCCESS;
    });
}

template <class R, class TA, class TB, class T0, class TX>
int gemm_vbatched2s_mixed_impl(void* handle, char ta0, char tb0, int* m0, int* n0, int* k0, const void* alpha0,
                               const void* const* A0, int* lda0, const void* const* B0, int* ldb0, const void* beta0,
                               void** C0, int* ldc0, char ta1, char tb1, int* m1, int* n1, int* k1,
                               const void* alpha1, const void* const* AB1, int* lda1, int* ldb1, const void* beta1,
                               void** C1, int* ldc1, int c0_left, int batch_count, const int* segment_sizes,
                               int segment_count)
{
    using Z = std::complex<R>;
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        if (!alpha0 || !beta0 || !alpha1 || !beta1) return ST_INVALID_VALUE;
        T0 a0, b0;
        Z a1, b1;
        std::memcpy(&a0, alpha0, sizeof(T0));
        std::memcpy(&b0, beta0, sizeof(T0));
        std::memcpy(&a1, alpha1, sizeof(Z));
        std::memcpy(&b1, beta1, sizeof(Z));
        ddla::gemmVbatched2s<R>(h, ta0, tb0, m0, n0, k0, a0, reinterpret_cast<const TA* const*>(A0), lda0,
                                reinterpret_cast<const TB* const*>(B0), ldb0, b0, reinterpret_cast<T0**>(C0), ldc0,
                                ta1, tb1, m1, n1, k1, a1, reinterpret_cast<const TX* const*>(AB1), lda1, ldb1, b1,
                                reinterpret_cast<Z**>(C1), ldc1, c0_left != 0, batch_count, segment_sizes,
                                segment_count);
        return ST_SUCCESS;
    });
}

template <class T>
int phegst_impl(void* handle, char uplo, int n, void* A, const int* descA, const void* F, const int* descF)
{
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        ddla::phegst<T>(h, uplo, n, static_cast<T*>(A), descA, static_cast<const T*>(F), descF);
        return ST_SUCCESS;
    });
}

template <class T>
int gemm_vbatched2s_impl(void* handle, char ta0, char tb0, int* m0, int* n0, int* k0, const void* alpha0,
                         const void* const* A0, int* lda0, const void* const* B0, int* ldb0, const void* beta0,
                         void** C0, int* ldc0, char ta1, char tb1, int* m1, int* n1, int* k1, const void* alpha1,
                         const void* const* AB1, int* lda1, int* ldb1, const void* beta1, void** C1, int* ldc1,
                         int c0_left, int batch_count, const int* segment_sizes, int segment_count)
{
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        if (!alpha0 || !beta0 || !alpha1 || !beta1) return ST_INVALID_VALUE;
        T a0, b0, a1, b1;
        std::memcpy(&a0, alpha0, sizeof(T));
        std::memcpy(&b0, beta0, sizeof(T));
        std::memcpy(&a1, alpha1, sizeof(T));
        std::memcpy(&b1, beta1, sizeof(T));
        ddla::gemmVbatched2s<T>(h, ta0, tb0, m0, n0, k0, a0, reinterpret_cast<const T* const*>(A0), lda0,
                                reinterpret_cast<const T* const*>(B0), ldb0, b0, reinterpret_cast<T**>(C0), ldc0, ta1,
                                tb1, m1, n1, k1, a1, reinterpret_cast<const T* const*>(AB1), lda1, ldb1, b1,
                                reinterpret_cast<T**>(C1), ldc1, c0_left != 0, batch_count, segment_sizes,
                                segment_count);
        return ST_SUCCESS;
    });
}

template <class T>
int ppotrf_ws_impl(void* handle, char uplo, int n, const int* descA, long long* bytes)
{
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        if (!bytes) return ST_INVALID_VALUE;
        std::size_t bb = 0, hb = 0;
        ddla::cholesky_impl::ppotrf_workspace_size<T>(h, uplo, n, nullptr, descA, &bb, &hb);
        *bytes = (long long)bb;
        return ST_SUCCESS;
    });
}
template <class T>
int ppotrf_run_impl(void* handle, char uplo, int n, void* A, const int* descA, int* info, void* work, long long bytes)
{
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        if (!info || bytes < 0) return ST_INVALID_VALUE;
        ddla::detail::require_gpu(h, "ppotrf_run");
        ddla::cholesky_impl::ppotrf_run<T>(h, uplo, n, static_cast<T*>(A), 1, 1, descA, *info, work, (size_t)bytes,
                                           nullptr, 0);
        return ST_SUCCESS;
    });
}
template <class T>
int ppotrs_ws_impl(void* handle, char side, int n, int nrhs, const int* descA, const int* descB, long long* bytes)
{
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        if (!bytes) return ST_INVALID_VALUE;
        std::size_t bb = 0, hb = 0;
        ddla::cholesky_impl::ppotrs_workspace_size<T>(h, side, n, nrhs, descA, descB, &bb, &hb);
        *bytes = (long long)bb;
        return ST_SUCCESS;
    });
}

}  // namespace

extern "C" {

const char* ddla_c_error_string(int status)
{
    if (status == ST_EXCEPTION && !g_last_error.empty()) return g_last_error.c_str();
    if (status >= 0 && status <= 5) return ddla::ddlaGetErrorString(static_cast<ddla::ddlaStatus_t>(status));
    return "unknown LibDDLA C API status";
}

int ddla_c_init_backend(void** handle, int backend)
{
    return guarded("ddla_c_init_backend", [&]() -> int {
        if (handle == nullptr) return ST_INVALID_VALUE;
        if (backend < 0 || backend > 1) return ST_INVALID_VALUE;
        const ddla::DdlaBackend be = backend == 0 ? ddla::DdlaBackend::CPU : ddla::DdlaBackend::GPU;
        if (!ddla::ddlaBackendAvailable(be)) return ST_BACKEND_UNAVAILABLE;
        ddla::DdlaHandle_t h = nullptr;
        const auto st = ddla::ddlaInit(h, be);
        if (st != ddla::ddlaStatus_t::DDLA_STATUS_SUCCESS) return static_cast<int>(st);
        *handle = h;
        return ST_SUCCESS;
    });
}

int ddla_c_set(void* handle, int f_comm, int nprows, int npcols, char major)
{
    return guarded("ddla_c_set", [&]() -> int {
        if (handle == nullptr) return ST_INVALID_HANDLE;
        const MPI_Comm comm = MPI_Comm_f2c(static_cast<MPI_Fint>(f_comm));
        ddla::ddlaStatus_t st;
        if (nprows > 0 && npcols > 0) st = ddla::ddlaSet(H(handle), comm, nprows, npcols, major);
        else st = ddla::ddlaSet(H(handle), comm, major);
        return static_cast<int>(st);
    });
}

int ddla_c_local_group_create(void** group, int nranks, double timeout_s)
{
    return guarded("ddla_c_local_group_create", [&]() -> int {
        if (group == nullptr) return ST_INVALID_VALUE;
        ddla::DdlaLocalGroup* g = nullptr;
        const ddla::ddlaStatus_t st = ddla::ddlaLocalGroupCreate(&g, nranks, timeout_s);
        *group = g;
        return static_cast<int>(st);
    });
}

int ddla_c_local_group_destroy(void* group)
{
    return guarded("ddla_c_local_group_destroy", [&]() -> int {
        return static_cast<int>(ddla::ddlaLocalGroupDestroy(static_cast<ddla::DdlaLocalGroup*>(group)));
    });
}

int ddla_c_set_local_group(void* handle, void* group, int rank, int nprows, int npcols, char major)
{
    return guarded("ddla_c_set_local_group", [&]() -> int {
        if (handle == nullptr) return ST_INVALID_HANDLE;
        return static_cast<int>(ddla::ddlaSetLocalGroup(H(handle), static_cast<ddla::DdlaLocalGroup*>(group), rank,
                                                        nprows, npcols, major));
    });
}

int ddla_c_nccl_available(void) { return ddla::ddlaNcclAvailable() ? 1 : 0; }

int ddla_c_nccl_unique_id(void* id128)
{
    return guarded("ddla_c_nccl_unique_id", [&]() -> int { return static_cast<int>(ddla::ddlaNcclUniqueId(id128)); });
}

int ddla_c_set_nccl(void* handle, const void* id128, int nranks, int rank, int nprows, int npcols, char major)
{
    return guarded("ddla_c_set_nccl", [&]() -> int {
        if (handle == nullptr) return ST_INVALID_HANDLE;
        return static_cast<int>(ddla::ddlaSetNccl(H(handle), id128, nranks, rank, nprows, npcols, major));
    });
}

int ddla_c_set_communication(void* handle, int communication)
{
    return guarded("ddla_c_set_communication", [&]() -> int {
        return static_cast<int>(
            ddla::ddlaSetCommunication(H(handle), static_cast<ddla::DdlaCommunication>(communication)));
    });
}

int ddla_c_get_communication(void* handle, int* communication)
{
    if (handle == nullptr) return ST_INVALID_HANDLE;
    if (communication == nullptr) return ST_INVALID_VALUE;
    return guarded("ddla_c_get_communication", [&]() -> int {
        *communication = static_cast<int>(ddla::ddlaGetCommunication(H(handle)));
        return ST_SUCCESS;
    });
}

int ddla_c_communication_available(void* handle, int communication)
{
    return ddla::ddlaCommunicationAvailable(H(handle), static_cast<ddla::DdlaCommunication>(communication)) ? 1 : 0;
}

int ddla_c_destroy(void** handle)
{
    return guarded("ddla_c_destroy", [&]() -> int {
        if (handle == nullptr || *handle == nullptr) return ST_SUCCESS;
        ddla::DdlaHandle_t h = H(*handle);
        const auto st = ddla::ddlaDestroy(h);
        *handle = h;
        return static_cast<int>(st);
    });
}

int ddla_c_backend_available(int backend)
{
    if (backend < 0 || backend > 1) return 0;
    return ddla::ddlaBackendAvailable(backend == 0 ? ddla::DdlaBackend::CPU : ddla::DdlaBackend::GPU) ? 1 : 0;
}

int ddla_c_get_backend(void* handle)
{
    if (handle == nullptr) return -ST_INVALID_HANDLE;
    return static_cast<int>(ddla::ddlaGetBackend(H(handle)));
}

int ddla_c_grid_dims(void* handle, int* nprows, int* npcols)
{
    if (handle == nullptr) return ST_INVALID_HANDLE;
    if (!nprows || !npcols) return ST_INVALID_VALUE;
    ddla::ddlaGetGridDims(H(handle), *nprows, *npcols);
    return ST_SUCCESS;
}

int ddla_c_grid_coords(void* handle, int* myprow, int* mypcol)
{
    if (handle == nullptr) return ST_INVALID_HANDLE;
    if (!myprow || !mypcol) return ST_INVALID_VALUE;
    ddla::ddlaGetGridCoords(H(handle), *myprow, *mypcol);
    return ST_SUCCESS;
}

int ddla_c_rank(void* handle) { return handle ? ddla::ddlaGetRank(H(handle)) : -1; }
int ddla_c_size(void* handle) { return handle ? ddla::ddlaGetSize(H(handle)) : -1; }

int ddla_c_descinit(int* desc, void* handle, int m, int n, int mb, int nb, int irsrc, int icsrc, int lld)
{
    if (handle == nullptr) return ST_INVALID_HANDLE;
    return static_cast<int>(ddla::ddlaDescInit(desc, H(handle), m, n, mb, nb, irsrc, icsrc, lld));
}

int ddla_c_numloc(int n, int nb, int iproc, int srcproc, int nprocs)
{
    return ddla::num_loc(n, nb, iproc, srcproc, nprocs);
}

int ddla_c_malloc(void* handle, void** ptr, long long bytes)
{
    if (handle == nullptr) return ST_INVALID_HANDLE;
    if (bytes < 0) return ST_INVALID_VALUE;
    return static_cast<int>(ddla::ddlaMalloc(H(handle), ptr, static_cast<std::size_t>(bytes)));
}
int ddla_c_free(void* handle, void* ptr)
{
    if (handle == nullptr) return ST_INVALID_HANDLE;
    return static_cast<int>(ddla::ddlaFree(H(handle), ptr));
}
int ddla_c_memcpy(void* handle, void* dst, const void* src, long long bytes)
{
    if (handle == nullptr) return ST_INVALID_HANDLE;
    if (bytes < 0) return ST_INVALID_VALUE;
    return static_cast<int>(ddla::ddlaMemcpy(H(handle), dst, src, static_cast<std::size_t>(bytes)));
}
int ddla_c_memcpy2d(void* handle, void* dst, long long dpitch, const void* src, long long spitch, long long width,
                    long long height)
{
    if (handle == nullptr) return ST_INVALID_HANDLE;
    if (dpitch < 0 || spitch < 0 || width < 0 || height < 0) return ST_INVALID_VALUE;
    return static_cast<int>(ddla::ddlaMemcpy2D(H(handle), dst, (std::size_t)dpitch, src, (std::size_t)spitch,
                                               (std::size_t)width, (std::size_t)height));
}
int ddla_c_memset(void* handle, void* ptr, int value, long long bytes)
{
    if (handle == nullptr) return ST_INVALID_HANDLE;
    if (bytes < 0) return ST_INVALID_VALUE;
    return static_cast<int>(ddla::ddlaMemset(H(handle), ptr, value, static_cast<std::size_t>(bytes)));
}
int ddla_c_synchronize(void* handle)
{
    if (handle == nullptr) return ST_INVALID_HANDLE;
    return static_cast<int>(ddla::ddlaSynchronize(H(handle)));
}

int ddla_c_default_comm(void) { return static_cast<int>(MPI_Comm_c2f(MPI_COMM_WORLD)); }
int ddla_c_comm_rank(int) { return 0; }
int ddla_c_comm_size(int) { return 1; }
void ddla_c_finalize(void) {}
int ddla_c_bcast_dims(int, int* m, int* n, int* type_char, int root)
{
    if (!m || !n || !type_char) return ST_INVALID_VALUE;
    return root == 0 ? ST_SUCCESS : ST_INVALID_VALUE;  // a single rank already holds the values
}

#define DDLA_C_TYPED(P, T)                                                                                           \
    int ddla_##P##_gather(void* h, int m, int n, const void* A, int ia, int ja, const int* descA, int root,          \
                          void* dst, int lddst)                                                                      \
    {                                                                                                                \
        return gather_impl<T>(h, m, n, A, ia, ja, descA, root, dst, lddst);                                          \
    }                                                                                                                \
    int ddla_##P##_scatter(void* h, int m, int n, void* A, int ia, int ja, const int* descA, int root,               \
                           const void* src, int ldsrc)                                                               \
    {                                                                                                                \
        return scatter_impl<T>(h, m, n, A, ia, ja, descA, root, src, ldsrc);                                         \
    }                                                                                                                \
    int ddla_##P##_ppotrf(void* handle, char uplo, int n, void* A, int ia, int ja, const int* descA, int* info)    \
    {                                                                                                                \
        return run(handle, [&](ddla::DdlaHandle_t h) -> int {                                                        \
            if (!info) return ST_INVALID_VALUE;                                                                      \
            ddla::ppotrf<T>(h, uplo, n, static_cast<T*>(A), ia, ja, descA, *info);                                   \
            return ST_SUCCESS;                                                                                       \
        });                                                                                                          \
    }                                                                                                                \
    int ddla_##P##_ppotrs(void* handle, char side, char uplo, char trans, int n, int nrhs, const void* A,          \
                          const int* descA, void* B, const int* descB)                                               \
    {                                                                                                                \
        return run(handle, [&](ddla::DdlaHandle_t h) -> int {                                                        \
            ddla::ppotrs<T>(h, side, uplo, trans, n, nrhs, static_cast<const T*>(A), descA, static_cast<T*>(B),      \
                            descB);                                                                                  \
            return ST_SUCCESS;                                                                                       \
        });                                                                                                          \
    }                                                                                                                \
    int ddla_##P##_pposv(void* handle, char side, char uplo, char trans, int n, int nrhs, void* A, int ia, int ja, \
                         const int* descA, void* B, int ib, int jb, const int* descB, int* info)                     \
    {                                                                                                                \
        return run(handle, [&](ddla::DdlaHandle_t h) -> int {                                                        \
            if (!info) return ST_INVALID_VALUE;                                                                      \
            ddla::pposv<T>(h, side, uplo, trans, n, nrhs, static_cast<T*>(A), ia, ja, descA, static_cast<T*>(B), ib, \
                           jb, descB, *info);                                                                        \
            return ST_SUCCESS;                                                                                       \
        });                                                                                                          \
    }                                                                                                                \
    int ddla_##P##_potrf(void* handle, char uplo, int n, void* A, int lda, void* info)                             \
    {                                                                                                                \
        return run(handle, [&](ddla::DdlaHandle_t h) -> int {                                                        \
            ddla::potrf<T>(h, uplo, n, static_cast<T*>(A), lda, static_cast<int*>(info));                            \
            return ST_SUCCESS;                                                                                       \
        });                                                                                                          \
    }                                                                                                                \
    int ddla_##P##_potrf_bottom_right(void* handle, char uplo, int n, void* A, int lda, int* info)                 \
    {                                                                                                                \
        return run(handle, [&](ddla::DdlaHandle_t h) -> int {                                                        \
            if (!info) return ST_INVALID_VALUE;                                                                      \
            ddla::potrf_bottom_right<T>(uplo, n, static_cast<T*>(A), lda, *info, h);                                 \
            return ST_SUCCESS;                                                                                       \
        });                                                                                                          \
    }                                                                                                                \
    int ddla_##P##_ppotrf_bottom_right(void* handle, char uplo, int n, void* A, const int* descA, int* info)       \
    {                                                                                                                \
        return run(handle, [&](ddla::DdlaHandle_t h) -> int {                                                        \
            if (!info) return ST_INVALID_VALUE;                                                                      \
            ddla::ppotrf_bottom_right<T>(h, uplo, n, static_cast<T*>(A), descA, *info);                              \
            return ST_SUCCESS;                                                                                       \
        });                                                                                                          \
    }                                                                                                                \
    int ddla_##P##_diag_logdet(void* handle, int n, const void* A, int lda, void* result)                          \
    {                                                                                                                \
        return diag_logdet_impl<T>(handle, n, A, lda, result);                                                       \
    }                                                                                                                \
    int ddla_##P##_pdiag_logdet(void* handle, int n, const void* A, const int* descA, void* result)                \
    {                                                                                                                \
        return pdiag_logdet_impl<T>(handle, n, A, descA, result);                                                    \
    }                                                                                                                \
    int ddla_##P##_pdiag_logdet_local(void* handle, int n, const void* A, const int* descA, int pr, int pc,       \
                                      int row, int col, double* state)                                             \
    {                                                                                                                \
        return pdiag_logdet_local_impl<T>(handle, n, A, descA, pr, pc, row, col, state);                            \
    }                                                                                                                \
    int ddla_##P##_gemm_vbatched(void* handle, char ta, char tb, int* d_m, int* d_n, int* d_k, const void* alpha,  \
                                 const void* const* d_A, int* d_lda, const void* const* d_B, int* d_ldb,             \
                                 const void* beta, void** d_C, int* d_ldc, int batch_count)                          \
    {                                                                                                                \
        return gemm_vbatched_impl<T>(handle, ta, tb, d_m, d_n, d_k, alpha, d_A, d_lda, d_B, d_ldb, beta, d_C, d_ldc, \
                                     batch_count);                                                                   \
    }                                                                                                                \
    int ddla_##P##_phegst(void* handle, char uplo, int n, void* A, const int* descA, const void* F,                \
                          const int* descF)                                                                          \
    {                                                                                                                \
        return phegst_impl<T>(handle, uplo, n, A, descA, F, descF);                                                  \
    }                                                                                                                \
    int ddla_##P##_gemm_vbatched2s(DDLA_GEMM_VBATCHED2S_ARGS)                                                      \
    {                                                                                                                \
        return gemm_vbatched2s_impl<T>(handle, transA_0, transB_0, d_m_0, d_n_0, d_k_0, alpha_0, d_A_0, d_lda_0,    \
                                       d_B_0, d_ldb_0, beta_0, d_C_0, d_ldc_0, transA_1, transB_1, d_m_1, d_n_1,    \
                                       d_k_1, alpha_1, d_AB_1, d_lda_1, d_ldb_1, beta_1, d_C_1, d_ldc_1, c0_left,    \
                                       batch_count, segment_sizes, segment_count);                                   \
    }                                                                                                                \
    int ddla_##P##_ppotrf_workspace_size(void* handle, char uplo, int n, const int* descA, long long* bytes)       \
    {                                                                                                                \
        return ppotrf_ws_impl<T>(handle, uplo, n, descA, bytes);                                                     \
    }                                                                                                                \
    int ddla_##P##_ppotrf_run(void* handle, char uplo, int n, void* A, const int* descA, int* info, void* work,    \
                              long long bytes)                                                                       \
    {                                                                                                                \
        return ppotrf_run_impl<T>(handle, uplo, n, A, descA, info, work, bytes);                                     \
    }                                                                                                                \
    int ddla_##P##_ppotrs_workspace_size(void* handle, char side, int n, int nrhs, const int* descA,               \
                                         const int* descB, long long* bytes)                                         \
    {                                                                                                                \
        return ppotrs_ws_impl<T>(handle, side, n, nrhs, descA, descB, bytes);                                        \
    }

DDLA_C_TYPED(s, float)
DDLA_C_TYPED(d, double)
DDLA_C_TYPED(c, std::complex<float>)
DDLA_C_TYPED(z, std::complex<double>)
#undef DDLA_C_TYPED

#define DDLA_GVM_C(P, R)                                                                                          \
    int ddla_##P##_gemm_vbatched_rc(void* handle, char ta, char tb, int* m, int* n, int* k, const void* alpha,      \
                                    const void* const* A, int* lda, const void* const* B, int* ldb,                \
                                    const void* beta, void** C, int* ldc, int batch_count)                         \
    {                                                                                                              \
        return gemm_vbatched_mixed_impl<R, false>(handle, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,    \
                                                  batch_count);                                                    \
    }                                                                                                              \
    int ddla_##P##_gemm_vbatched_cr(void* handle, char ta, char tb, int* m, int* n, int* k, const void* alpha,      \
                                    const void* const* A, int* lda, const void* const* B, int* ldb,                \
                                    const void* beta, void** C, int* ldc, int batch_count)                         \
    {                                                                                                              \
        return gemm_vbatched_mixed_impl<R, true>(handle, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,     \
                                                 batch_count);                                                     \
    }
DDLA_GVM_C(c, float)
DDLA_GVM_C(z, double)
#undef DDLA_GVM_C

#define DDLA_GV2M_C(P, R, CODE, TA, TB, T0, TX)                                                               \
    int ddla_##P##_gemm_vbatched2s_##CODE(DDLA_GEMM_VBATCHED2S_ARGS)                                             \
    {                                                                                                            \
        return gemm_vbatched2s_mixed_impl<R, TA, TB, T0, TX>(                                                    \
            handle, transA_0, transB_0, d_m_0, d_n_0, d_k_0, alpha_0, d_A_0, d_lda_0, d_B_0, d_ldb_0, beta_0,    \
            d_C_0, d_ldc_0, transA_1, transB_1, d_m_1, d_n_1, d_k_1, alpha_1, d_AB_1, d_lda_1, d_ldb_1, beta_1,  \
            d_C_1, d_ldc_1, c0_left, batch_count, segment_sizes, segment_count);                                 \
    }
#define DDLA_GV2M_C_ALL(P, R)                                                                                    \
    DDLA_GV2M_C(P, R, rzzr, R, std::complex<R>, std::complex<R>, R)                                              \
    DDLA_GV2M_C(P, R, zrzr, std::complex<R>, R, std::complex<R>, R)                                              \
    DDLA_GV2M_C(P, R, rzzz, R, std::complex<R>, std::complex<R>, std::complex<R>)                                \
    DDLA_GV2M_C(P, R, zrzz, std::complex<R>, R, std::complex<R>, std::complex<R>)                                \
    DDLA_GV2M_C(P, R, zzzr, std::complex<R>, std::complex<R>, std::complex<R>, R)                                \
    DDLA_GV2M_C(P, R, rrrz, R, R, R, std::complex<R>)
DDLA_GV2M_C_ALL(c, float)
DDLA_GV2M_C_ALL(z, double)
#undef DDLA_GV2M_C_ALL
#undef DDLA_GV2M_C

int ddla_d_ppotrs_noalloc(void* handle, char side, char uplo, char trans, int n, int nrhs, const void* A,
                          const int* descA, void* B, const int* descB)
{
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        ddla::ppotrs_noalloc(h, side, uplo, trans, n, nrhs, static_cast<const double*>(A), descA,
                             static_cast<double*>(B), descB);
        return ST_SUCCESS;
    });
}

int ddla_c_get_stream(void* handle, void** stream)
{
    if (handle == nullptr) return ST_INVALID_HANDLE;
    if (stream == nullptr) return ST_INVALID_VALUE;
    *stream = ddla::ddlaGetStream(H(handle));
    return ST_SUCCESS;
}
long long ddla_c_launch_count(void) { return ddlak_launch_count(); }

int ddla_c_pdiag_logdet_finish(const double* total, int single, void* result)
{
    if (total == nullptr || result == nullptr) return ST_INVALID_VALUE;
    return guarded("ddla_c_pdiag_logdet_finish", [&]() -> int {
        double re = 0, im = 0;
        ddla::pdiag_logdet_finish(total, re, im);
        if (single) {
            const float r[2] = {static_cast<float>(re), static_cast<float>(im)};
            std::memcpy(result, r, sizeof(r));
        } else {
            const double r[2] = {re, im};
            std::memcpy(result, r, sizeof(r));
        }
        return ST_SUCCESS;
    });
}
int ddla_c_fail_allocation(long long nth)
{
    ddla::detail::arm_allocation_failure(nth);
    return ST_SUCCESS;
}
long long ddla_c_live_workspaces(void) { return ddla::detail::live_workspaces(); }
int ddla_c_set_wait_budget(void* handle, long long cycles)
{
    if (handle == nullptr) return ST_INVALID_HANDLE;
    if (cudaSetDevice(H(handle)->device) != cudaSuccess) return ST_INTERNAL_ERROR;
    return ddlak_set_wait_budget(cycles) == 0 ? ST_SUCCESS : ST_INTERNAL_ERROR;
}
void ddla_c_profile_enable(int on) { ddlak_profile_enable(on); }
int ddla_c_profile_read(int kind, double* ms, long long* launches, double* flops, double* bytes, int reset)
{
    const int e = ddlak_profile_read(kind, ms, launches, flops, bytes, reset);
    return e == 0 ? ST_SUCCESS : ST_INTERNAL_ERROR;
}

int ddla_d_pposv_mixed_host(void* handle, char uplo, char precision, int n, int nrhs, const void* A, int lda,
                            const void* B, int ldb, void* X, int ldx, int* info, double* report)
{
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        if (!info) return ST_INVALID_VALUE;
        ddla::MixedReport rep;
        ddla::pposv_mixed_host(h, uplo, precision, n, nrhs, static_cast<const double*>(A), lda,
                               static_cast<const double*>(B), ldb, static_cast<double*>(X), ldx, *info, &rep);
        if (report) {
            report[0] = rep.iter;
            report[1] = rep.gmres;
            report[2] = rep.shift;
            report[3] = rep.backward_error;
        }
        return ST_SUCCESS;
    });
}

int ddla_d_pposv_mixed(void* handle, char uplo, char precision, int n, int nrhs, void* A, const int* descA,
                       const void* B, const int* descB, void* X, const int* descX, int* info, double* report)
{
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        if (!info) return ST_INVALID_VALUE;
        ddla::MixedReport rep;
        ddla::pposv_mixed(h, uplo, precision, n, nrhs, static_cast<double*>(A), descA, static_cast<const double*>(B),
                          descB, static_cast<double*>(X), descX, *info, &rep);
        if (report) {
            report[0] = rep.iter;
            report[1] = rep.gmres;
            report[2] = rep.shift;
            report[3] = rep.backward_error;
        }
        return ST_SUCCESS;
    });
}

int ddla_s_posv_vbatched(void* handle, char uplo, const int* d_n, float* const* d_A, const int* d_lda,
                         float* const* d_B, double* d_logdet, int* d_info, int batch_count, int max_n)
{
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        ddla::posvVbatched<float>(h, uplo, d_n, d_A, d_lda, d_B, d_logdet, d_info, batch_count, max_n);
        return ST_SUCCESS;
    });
}

int ddla_d_posv_vbatched(void* handle, char uplo, const int* d_n, double* const* d_A, const int* d_lda,
                         double* const* d_B, double* d_logdet, int* d_info, int batch_count, int max_n)
{
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        ddla::posvVbatched<double>(h, uplo, d_n, d_A, d_lda, d_B, d_logdet, d_info, batch_count, max_n);
        return ST_SUCCESS;
    });
}

int ddla_s_posv_vbatched_plan(void* handle, char uplo, const int* d_n, float* const* d_A, const int* d_lda,
                              float* const* d_B, double* d_logdet, int* d_info, int batch_count, int max_n,
                              void** plan)
{
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        if (!plan) return ST_INVALID_VALUE;
        *plan = ddla::VbatchedPlan::create<float>(h, uplo, d_n, d_A, d_lda, d_B, d_logdet, d_info, batch_count,
                                                  max_n);
        return ST_SUCCESS;
    });
}

int ddla_d_posv_vbatched_plan(void* handle, char uplo, const int* d_n, double* const* d_A, const int* d_lda,
                              double* const* d_B, double* d_logdet, int* d_info, int batch_count, int max_n,
                              void** plan)
{
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        if (!plan) return ST_INVALID_VALUE;
        *plan = ddla::VbatchedPlan::create<double>(h, uplo, d_n, d_A, d_lda, d_B, d_logdet, d_info, batch_count,
                                                   max_n);
        return ST_SUCCESS;
    });
}

int ddla_vbatched_plan_run(void* plan)
{
    if (!plan) return ST_INVALID_VALUE;
    return guarded("ddla_vbatched_plan_run", [&]() -> int {
        static_cast<ddla::VbatchedPlan*>(plan)->run();
        return ST_SUCCESS;
    });
}

int ddla_vbatched_plan_info(void* plan, int* grid, double* flops)
{
    if (!plan) return ST_INVALID_VALUE;
    const auto* p = static_cast<ddla::VbatchedPlan*>(plan);
    if (grid) *grid = p->grid();
    if (flops) *flops = p->flops();
    return ST_SUCCESS;
}

int ddla_vbatched_plan_destroy(void* plan)
{
    return guarded("ddla_vbatched_plan_destroy", [&]() -> int {
        delete static_cast<ddla::VbatchedPlan*>(plan);
        return ST_SUCCESS;
    });
}

int ddla_vbatched_autotune(void* handle, char type, int max_n)
{
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        ddla::vbatchedAutotune(h, type, max_n);
        return ST_SUCCESS;
    });
}

int ddla_vbatched_tuning(void* handle, char type, int max_n, int* grid, int* widths, unsigned char* variant, int len,
                         int* tuned)
{
    return run(handle, [&](ddla::DdlaHandle_t h) -> int {
        const ddla::VbatchedTuning t = ddla::vbatchedTuning(h, type, max_n);
        if (grid) *grid = t.grid;
        if (widths) {
            widths[0] = t.widths[0];
            widths[1] = t.widths[1];
        }
        if (variant) {
            if (len < (int)t.variant.size()) return ST_INVALID_VALUE;
            std::memcpy(variant, t.variant.data(), t.variant.size());
        }
        if (tuned) *tuned = t.tuned ? 1 : 0;
        return ST_SUCCESS;
    });
}

#define DDLA_GP_C(P, T)                                                                                             \
    int ddla_##P##_chol_nll_batched(void* handle, int batch, int n, T* A, const T* y, T* alpha, double* logdet,      \
                                    double* quad, int* info)                                                        \
    {                                                                                                               \
        return run(handle, [&](ddla::DdlaHandle_t h) -> int {                                                       \
            ddla::cholNllBatched<T>(h, batch, n, A, y, alpha, logdet, quad, info);                                  \
            return ST_SUCCESS;                                                                                      \
        });                                                                                                         \
    }                                                                                                               \
    int ddla_##P##_gp_nll_batched(void* handle, int batch, int n, int d, const T* X, const double* theta,           \
                                  int theta_stride, const T* y, T* A, T* alpha, double* logdet, double* quad,        \
                                  int* info)                                                                        \
    {                                                                                                               \
        return run(handle, [&](ddla::DdlaHandle_t h) -> int {                                                       \
            ddla::gpNllBatched<T>(h, batch, n, d, X, theta, theta_stride, y, A, alpha, logdet, quad, info);         \
            return ST_SUCCESS;                                                                                      \
        });                                                                                                         \
    }                                                                                                               \
    int ddla_##P##_chol_nll_grad_batched(void* handle, int batch, int n, const T* L, const T* alpha, T* W, T* G)    \
    {                                                                                                               \
        return run(handle, [&](ddla::DdlaHandle_t h) -> int {                                                       \
            ddla::cholNllGradBatched<T>(h, batch, n, L, alpha, W, G);                                               \
            return ST_SUCCESS;                                                                                      \
        });                                                                                                         \
    }                                                                                                               \
    int ddla_##P##_gp_nll_grad_batched(void* handle, int batch, int n, int d, const T* X, const double* theta,      \
                                       int theta_stride, const T* L, const T* alpha, T* W, double* grad)            \
    {                                                                                                               \
        return run(handle, [&](ddla::DdlaHandle_t h) -> int {                                                       \
            ddla::gpNllGradBatched<T>(h, batch, n, d, X, theta, theta_stride, L, alpha, W, grad);                   \
            return ST_SUCCESS;                                                                                      \
        });                                                                                                         \
    }
DDLA_GP_C(s, float)
DDLA_GP_C(d, double)
#undef DDLA_GP_C

}  // extern "C"
