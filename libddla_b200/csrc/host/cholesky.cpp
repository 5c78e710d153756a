// ddla::ppotrf / ppotrs / pposv / potrf / diag_logdet on a GPU handle (1x1 grid).
//
// Argument checks, exception types and messages follow the reference's
// check components (src/Cholesky/ppotrf.cpp:21-29, ppotrs.cpp:14-30,
// pposv.cpp:15-21, potrf.cpp:122-135, src/diag_logdet.cpp:42-55); the run
// components replace the vendor calls with the kernels of include/ddla_kernels.h.
// ppotrf/ppotrs/pposv return with the handle's stream synchronised and info
// on the host (ppotrf.cpp:49-52, ppotrs.cpp:84, pposv.cpp:62); potrf is
// asynchronous with a device info (ddla.h:2150-2160).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>

#include <ddla/ddla.h>
#include <ddla_kernels.h>

#include "ddla_stream.h"
#include "grid.h"

namespace ddla {

namespace {

template <class T> constexpr char tcode();
template <> constexpr char tcode<float>() { return 's'; }
template <> constexpr char tcode<double>() { return 'd'; }
template <> constexpr char tcode<std::complex<float>>() { return 'c'; }
template <> constexpr char tcode<std::complex<double>>() { return 'z'; }

void ppotrf_check(const DdlaHandle_t& h, char uplo, int n, const void* A, int ia, int ja, const int* d)
{
    detail::check_desc(d, h);
    detail::require_gpu(h, "ppotrf");
    if ((uplo != 'L' && uplo != 'U') || n < 0 || n > d[DDLA_M_] || n > d[DDLA_N_] || d[DDLA_MB_] != d[DDLA_NB_] ||
        ia != 1 || ja != 1)
        throw std::invalid_argument("ppotrf: invalid triangle, dimensions, blocks or offsets");
    if (n && !A) throw std::invalid_argument("ppotrf: null local matrix");
}

void ppotrs_check(const DdlaHandle_t& h, char side, char uplo, char trans, int n, int nrhs, const void* A,
                  const int* da, const void* B, const int* db)
{
    detail::check_desc(da, h);
    detail::check_desc(db, h);
    detail::require_gpu(h, "ppotrs");
    if ((side != 'L' && side != 'R') || (uplo != 'L' && uplo != 'U') || (trans != 'N' && trans != 'C') || n < 0 ||
        nrhs < 0 || n > da[DDLA_M_] || n > da[DDLA_N_] || da[DDLA_MB_] != da[DDLA_NB_])
        throw std::invalid_argument("ppotrs: invalid flags, dimensions or factor blocks");
    if (db[DDLA_MB_] != da[DDLA_MB_] || (side == 'L' && db[DDLA_RSRC_] != da[DDLA_RSRC_]) ||
        (side == 'R' && (db[DDLA_NB_] != da[DDLA_NB_] || db[DDLA_CSRC_] != da[DDLA_CSRC_])))
        throw std::invalid_argument("ppotrs: B must be distributed like A along the solved dimension");
    const int rows = side == 'L' ? n : nrhs, cols = side == 'L' ? nrhs : n;
    if (rows > db[DDLA_M_] || cols > db[DDLA_N_]) throw std::invalid_argument("ppotrs: invalid right-hand side");
    if (n && !A) throw std::invalid_argument("ppotrs: null local factor");
    if (rows && cols && !B) throw std::invalid_argument("ppotrs: null local right-hand side");
}

void pposv_check(const DdlaHandle_t& h, char side, char uplo, char trans, int n, int nrhs, const void* A, int ia,
                 int ja, const int* da, const void* B, int ib, int jb, const int* db)
{
    ppotrf_check(h, uplo, n, A, ia, ja, da);
    ppotrs_check(h, side, uplo, trans, n, nrhs, A, da, B, db);
    if (ib != 1 || jb != 1) throw std::invalid_argument("pposv: offsets must be one");
}

// potrf_bottom_right_check (src/Cholesky/potrf_bottom_right.cpp:171-187): real throws, runtime_error
void potrf_bottom_right_check(const DdlaHandle_t& h, char uplo, int n, const void* A, int lda)
{
    detail::require_gpu(h, "potrf_bottom_right");
    if (uplo != 'U' && uplo != 'L') throw std::runtime_error("potrf_bottom_right: uplo must be 'U' or 'L'");
    if (n < 0) throw std::runtime_error("potrf_bottom_right: negative matrix size");
    if (n == 0) return;
    if (A == nullptr) throw std::runtime_error("potrf_bottom_right: null A");
    if (lda < n) throw std::runtime_error("potrf_bottom_right: lda too small");
}

// ppotrf_bottom_right_check (src/Cholesky/ppotrf_bottom_right.cpp:62-70) on a 1x1 grid
void ppotrf_bottom_right_check(const DdlaHandle_t& h, char uplo, int n, const void* A, const int* d)
{
    detail::check_desc(d, h);
    detail::require_gpu(h, "ppotrf_bottom_right");
    if ((uplo != 'L' && uplo != 'U') || n < 0 || n > d[DDLA_M_] || n > d[DDLA_N_] || d[DDLA_MB_] != d[DDLA_NB_] ||
        h->nprows_ != h->npcols_ || h->nprocs > 1)
        throw std::invalid_argument("ppotrf_bottom_right: invalid triangle, dimensions, blocks or grid");
    if (n && !A) throw std::invalid_argument("ppotrf_bottom_right: null local matrix");
}

int read_device_int(const DdlaHandle_t& h, const int* dptr)
{
    detail::cuda_check(cudaMemcpyAsync(h->host_word, dptr, sizeof(int), cudaMemcpyDeviceToHost, h->stream),
                       "info read-back");
    detail::cuda_check(cudaStreamSynchronize(h->stream), "stream synchronisation");
    return *h->host_word;
}

}  // namespace

namespace cholesky_impl {

template <typename T>
void ppotrf_workspace_size(const DdlaHandle_t&, char, int n, const T*, const int*, std::size_t* backend_bytes,
                           std::size_t* host_bytes)
{
    *backend_bytes = n > 0 ? detail::padded_bytes<int>(1) : 0;  // the device info word
    *host_bytes = 0;
}

template <typename T>
void ppotrf_run(const DdlaHandle_t& h, char uplo, int n, T* A, int, int, const int* descA, int& info,
                void* backend_work, std::size_t backend_bytes, void*, std::size_t)
{
    if (n == 0) {
        info = 0;
        return;
    }
    if (h->nprocs > 1) {  // a grid of several ranks: the distributed factorization (its own scratch)
        grid::ppotrf_grid<T>(h, uplo, n, A, descA, info);
        return;
    }
    if (backend_bytes < detail::padded_bytes<int>(1) || backend_work == nullptr)
        throw std::invalid_argument("ppotrf: workspace smaller than ppotrf_workspace_size");
    char* w = static_cast<char*>(backend_work);
    int* dinfo = detail::take<int>(w, 1);
    detail::kernel_check(ddlak_potrf(tcode<T>(), uplo, n, A, descA[DDLA_LLD_], dinfo, h->stream), "potrf kernels");
    info = read_device_int(h, dinfo);
}

// The plain FP64 solve at large orders with few right-hand sides (uplo 'L', side 'L',
// nrhs <= 16) runs as the persistent solve by inverted 1024-row diagonal blocks
// (ddlak_bis_inverse_f64 + ddlak_bis_solve_f64): a few dozen diagonal blocks instead
// of a chain of n / 64 block rows per direction.  Below kBisMinOrder the fused
// 64-row solve is faster (the inverses cost O(n * 1024^2)).
constexpr int kBisMinOrder = 4096;

template <typename T>
bool bis_candidate(char side, int n, int nrhs)
{
    return std::is_same<T, double>::value && side == 'L' && n >= kBisMinOrder && nrhs >= 1 && nrhs <= 16;
}

std::size_t bis_bytes(int n, int nrhs)
{
    return detail::padded_bytes<char>(static_cast<std::size_t>(ddlak_bis_inverse_bytes(n))) +
           static_cast<std::size_t>(ddlak_bis_solve_workspace(n, nrhs));
}

template <typename T>
void ppotrs_workspace_size(const DdlaHandle_t&, char side, int n, int nrhs, const int*, const int*,
                           std::size_t* backend_bytes, std::size_t* host_bytes)
{
    *host_bytes = 0;
    *backend_bytes = (n > 0 && nrhs > 0) ? static_cast<std::size_t>(ddlak_potrs_workspace(n, nrhs)) : 0;
    if (bis_candidate<T>(side, n, nrhs)) *backend_bytes = std::max(*backend_bytes, bis_bytes(n, nrhs));
}

template <typename T>
void ppotrs_run(const DdlaHandle_t& h, char side, char uplo, char, int n, int nrhs, const T* A, const int* descA,
                T* B, const int* descB, void* backend_work, std::size_t backend_bytes, void*, std::size_t)
{
    if (n == 0 || nrhs == 0) return;
    if (h->nprocs > 1) {  // a grid of several ranks: the distributed solve (its own scratch)
        grid::ppotrs_grid<T>(h, side, uplo, n, nrhs, A, descA, B, descB);
        return;
    }
    const long long lda = descA[DDLA_LLD_];
    if (bis_candidate<T>(side, n, nrhs) && uplo == 'L' && !(lda & 1) &&
        !(reinterpret_cast<std::uintptr_t>(A) & 15) && backend_work != nullptr && backend_bytes >= bis_bytes(n, nrhs)) {
        char* w = static_cast<char*>(backend_work);
        void* Dinv = w;
        void* swork = w + detail::padded_bytes<char>(static_cast<std::size_t>(ddlak_bis_inverse_bytes(n)));
        const std::size_t sbytes = backend_bytes - static_cast<std::size_t>(static_cast<char*>(swork) - w);
        detail::kernel_check(ddlak_bis_inverse_f64(n, A, lda, Dinv, h->stream), "diagonal block inverses");
        detail::kernel_check(ddlak_bis_solve_f64(n, nrhs, A, lda, Dinv, B, descB[DDLA_LLD_], swork, sbytes, h->stream),
                             "persistent solve");
        if (read_device_int(h, static_cast<const int*>(swork)) != 0)
            throw std::runtime_error("ppotrs: a device wait in the persistent solve timed out");
        return;
    }
    const unsigned long long need = ddlak_potrs_workspace(n, nrhs);
    if (backend_bytes < need || backend_work == nullptr)
        throw std::invalid_argument("ppotrs: workspace smaller than ppotrs_workspace_size");
    detail::kernel_check(ddlak_potrs(tcode<T>(), uplo, side, n, nrhs, A, descA[DDLA_LLD_], B, descB[DDLA_LLD_],
                                     backend_work, need, h->stream),
                         "potrs kernel");
    const int status = read_device_int(h, static_cast<const int*>(backend_work));
    if (status != 0) throw std::runtime_error("ppotrs: a device wait in the fused solve timed out");
}

}  // namespace cholesky_impl

namespace cholesky_impl {

// The bottom-right factorization (src/Cholesky/potrf_bottom_right.cpp:208-256 on one
// rank): J A J (J reverses the order) is factored by the standard kernels on the
// opposite triangle, then swapped back.  A pivot that fails at reversed position k
// is the pivot n - k + 1 counted from the top, the reference's
// global_offset + n - solver_info + 1 (potrf_bottom_right.cpp:97).
template <typename T>
void bottom_right_core(const DdlaHandle_t& h, char uplo, int n, T* A, long long lda, int& info, void* backend_work,
                       std::size_t backend_bytes)
{
    info = 0;
    if (n == 0) return;
    if (backend_bytes < detail::padded_bytes<int>(1) || backend_work == nullptr)
        throw std::invalid_argument("ppotrf_bottom_right: workspace smaller than ppotrf_bottom_right_workspace_size");
    char* w = static_cast<char*>(backend_work);
    int* dinfo = detail::take<int>(w, 1);
    detail::kernel_check(ddlak_reverse_swap(tcode<T>(), n, A, lda, h->stream), "reverse swap");
    detail::kernel_check(ddlak_potrf(tcode<T>(), uplo == 'U' ? 'L' : 'U', n, A, lda, dinfo, h->stream),
                         "potrf kernels");
    detail::kernel_check(ddlak_reverse_swap(tcode<T>(), n, A, lda, h->stream), "reverse swap");
    const int r = read_device_int(h, dinfo);
    info = r == 0 ? 0 : n - r + 1;
}

template <typename T>
void ppotrf_bottom_right_workspace_size(const DdlaHandle_t&, char, int n, T*, const int*, std::size_t* backend_bytes,
                                        std::size_t* host_bytes)
{
    *backend_bytes = n > 0 ? detail::padded_bytes<int>(1) : 0;  // the device info word
    *host_bytes = 0;
}

template <typename T>
void ppotrf_bottom_right_run(const DdlaHandle_t& h, char uplo, int n, T* A, const int* descA, int& info,
                             void* backend_work, std::size_t backend_bytes, void*, std::size_t)
{
    bottom_right_core<T>(h, uplo, n, A, descA[DDLA_LLD_], info, backend_work, backend_bytes);
}

}  // namespace cholesky_impl

template <typename T>
void potrf_bottom_right(char uplo, int n, T* A, int lda, int& info, const DdlaHandle_t& handle)
{
    potrf_bottom_right_check(handle, uplo, n, A, lda);
    info = 0;
    if (n == 0) return;
    detail::DeviceScratch work(handle, detail::padded_bytes<int>(1));
    cholesky_impl::bottom_right_core<T>(handle, uplo, n, A, lda, info, work.data(), detail::padded_bytes<int>(1));
}

template <typename T>
void ppotrf_bottom_right(const DdlaHandle_t& handle, char uplo, int n, T* A, const int* descA, int& info)
{
    ppotrf_bottom_right_check(handle, uplo, n, A, descA);
    info = 0;
    if (n == 0) return;
    std::size_t bb = 0, hb = 0;
    cholesky_impl::ppotrf_bottom_right_workspace_size<T>(handle, uplo, n, A, descA, &bb, &hb);
    detail::DeviceScratch work(handle, bb);
    cholesky_impl::ppotrf_bottom_right_run<T>(handle, uplo, n, A, descA, info, work.data(), bb, nullptr, 0);
}

template <typename T>
void ppotrf(const DdlaHandle_t& handle, char uplo, int n, T* A, int ia, int ja, const int* descA, int& info)
{
    ppotrf_check(handle, uplo, n, A, ia, ja, descA);
    info = 0;
    if (n == 0) return;
    std::size_t bb = 0, hb = 0;
    cholesky_impl::ppotrf_workspace_size<T>(handle, uplo, n, A, descA, &bb, &hb);
    detail::DeviceScratch work(handle, bb);
    cholesky_impl::ppotrf_run<T>(handle, uplo, n, A, ia, ja, descA, info, work.data(), bb, nullptr, 0);
}

template <typename T>
void ppotrs(const DdlaHandle_t& h, char side, char uplo, char trans, int n, int nrhs, const T* A, const int* da, T* B,
            const int* db)
{
    ppotrs_check(h, side, uplo, trans, n, nrhs, A, da, B, db);
    if (n == 0 || nrhs == 0) return;
    std::size_t bb = 0, hb = 0;
    cholesky_impl::ppotrs_workspace_size<T>(h, side, n, nrhs, da, db, &bb, &hb);
    detail::DeviceScratch work(h, bb);
    cholesky_impl::ppotrs_run<T>(h, side, uplo, trans, n, nrhs, A, da, B, db, work.data(), bb, nullptr, 0);
    detail::cuda_check(cudaStreamSynchronize(h->stream), "stream synchronisation");
}

template <typename T>
void pposv(const DdlaHandle_t& h, char side, char uplo, char trans, int n, int nrhs, T* A, int ia, int ja,
           const int* da, T* B, int ib, int jb, const int* db, int& info)
{
    pposv_check(h, side, uplo, trans, n, nrhs, A, ia, ja, da, B, ib, jb, db);
    if (n == 0) {
        info = 0;
        return;
    }
    std::size_t fb = 0, fh = 0, sb = 0, sh = 0;
    cholesky_impl::ppotrf_workspace_size<T>(h, uplo, n, A, da, &fb, &fh);
    cholesky_impl::ppotrs_workspace_size<T>(h, side, n, nrhs, da, db, &sb, &sh);
    const std::size_t bb = std::max(fb, sb);
    detail::DeviceScratch work(h, bb);
    cholesky_impl::ppotrf_run<T>(h, uplo, n, A, ia, ja, da, info, work.data(), bb, nullptr, 0);
    if (info == 0) cholesky_impl::ppotrs_run<T>(h, side, uplo, trans, n, nrhs, A, da, B, db, work.data(), bb, nullptr, 0);
    detail::cuda_check(cudaStreamSynchronize(h->stream), "stream synchronisation");
}

// ppotrs with the solve's flags in the library's fixed device array: no
// allocation.  For callers that cannot allocate device memory while running.
void ppotrs_noalloc(const DdlaHandle_t& h, char side, char uplo, char trans, int n, int nrhs, const double* A,
                    const int* da, double* B, const int* db)
{
    ppotrs_check(h, side, uplo, trans, n, nrhs, A, da, B, db);
    if (n == 0 || nrhs == 0) return;
    int max_n = 0, max_rhs = 0;
    ddlak_potrs_fixed_scratch_limits(&max_n, &max_rhs);
    if (n > max_n || nrhs > max_rhs)
        throw std::invalid_argument("ppotrs_noalloc: the fixed scratch serves n <= " + std::to_string(max_n) +
                                    " and nrhs <= " + std::to_string(max_rhs));
    int* status = nullptr;
    detail::kernel_check(ddlak_potrs_fixed_scratch('d', uplo, side, n, nrhs, A, da[DDLA_LLD_], B, db[DDLA_LLD_],
                                                   &status, h->stream),
                         "potrs kernel (fixed scratch)");
    if (read_device_int(h, status) != 0) throw std::runtime_error("ppotrs_noalloc: a device wait timed out");
}

template <typename T>
void potrf(const DdlaHandle_t& h, char uplo, int n, T* A, int lda, int* info)
{
    detail::require_gpu(h, "potrf");
    char u;
    if (uplo == 'U' || uplo == 'u') u = 'U';
    else if (uplo == 'L' || uplo == 'l') u = 'L';
    else throw std::runtime_error("ddla: invalid uplo flag (expected 'U' or 'L')");
    if (n < 0) throw std::runtime_error("potrf: negative matrix size");
    if (info == nullptr) throw std::runtime_error("potrf: null info");
    if (n > 0) {
        if (A == nullptr) throw std::runtime_error("potrf: null A");
        if (lda < std::max(1, n)) throw std::runtime_error("potrf: lda too small");
    }
    detail::kernel_check(ddlak_potrf(tcode<T>(), u, n, A, lda, info, h->stream), "potrf kernels");
}

namespace {
// DiagLogTerm / DiagLogJoin over the diagonal, then finish_diagonal_log
// (src/diag_logdet_impl.h:42-113); `who` names the routine in the domain_error.
template <typename T>
void logdet_core(const DdlaHandle_t& h, int n, const T* a, long long lda, std::complex<real_type_t<T>>& result,
                 const char* who)
{
    using R = real_type_t<T>;
    if (n > 0) {
        // the reference's check_diag_span (src/diag_logdet_impl.h:33-40)
        const auto last = std::uint64_t(n - 1) * std::uint64_t(lda) + std::uint64_t(n) - 1;
        if (last > std::uint64_t(std::numeric_limits<std::ptrdiff_t>::max()) / sizeof(T))
            throw std::overflow_error(std::string(who) + ": matrix address span is not representable");
    }
    double magnitude = 0, phase = 0;
    int flags = 0;
    if (n > 0) {
        detail::DeviceScratch work(h, static_cast<std::size_t>(ddlak_logdet_workspace()));
        detail::kernel_check(ddlak_diag_logsum(tcode<T>(), n, a, lda, work.data(), h->stream), "diag_logdet kernels");
        struct {
            double mag, phase;
            int flags, pad;
        } st{};
        static_assert(sizeof(st) == 24, "state layout");
        detail::cuda_check(cudaMemcpyAsync(h->host_word, work.data(), sizeof(st), cudaMemcpyDeviceToHost, h->stream),
                           "logdet read-back");
        detail::cuda_check(cudaStreamSynchronize(h->stream), "stream synchronisation");
        std::memcpy(&st, h->host_word, sizeof(st));
        magnitude = st.mag;
        phase = st.phase;
        flags = st.flags;
    }
    if (flags & 1) throw std::domain_error(std::string(who) + ": nonfinite diagonal");
    // finish_diagonal_log (src/diag_logdet_impl.h:104-113)
    if (flags & 2) {
        result = {-std::numeric_limits<R>::infinity(), R(0)};
        return;
    }
    const double pi = std::acos(-1.0);
    phase = std::remainder(phase + ((flags >> 2) & 1) * pi, 2 * pi);
    if (phase <= -pi) phase = pi;
    result = {static_cast<R>(magnitude), static_cast<R>(phase)};
}
}  // namespace

template <typename T>
void diag_logdet(const DdlaHandle_t& h, int n, const T* a, int lda, std::complex<real_type_t<T>>& result)
{
    detail::require_gpu(h, "diag_logdet");
    if (n < 0 || lda < std::max(1, n) || (n > 0 && !a))
        throw std::invalid_argument("diag_logdet: invalid order, leading dimension or pointer");
    logdet_core<T>(h, n, a, lda, result, "diag_logdet");
}

// The descriptor form (src/PBLAS/pdiag_logdet.cpp:11-48).  On a 1x1 grid the local
// block is the whole matrix and the all-reduce of the four partial sums is the
// identity, so the result is diag_logdet's with LLD_ as the leading dimension; on a
// grid of several ranks every rank's state is summed over the grid (grid.cpp).
template <typename T>
void pdiag_logdet(const DdlaHandle_t& h, int n, const T* a, const int* desc, std::complex<real_type_t<T>>& result)
{
    detail::require_gpu(h, "pdiag_logdet");
    detail::check_desc(desc, h);
    if (n < 0 || n > desc[DDLA_M_] || n > desc[DDLA_N_])
        throw std::invalid_argument("pdiag_logdet: order exceeds descriptor");
    if (h->nprocs > 1) {  // every rank's local state, summed over the grid, finished on every rank
        double total[5], re = 0, im = 0;
        grid::pdiag_logdet_grid<T>(h, n, a, desc, total);
        pdiag_logdet_finish(total, re, im);
        result = std::complex<real_type_t<T>>(static_cast<real_type_t<T>>(re), static_cast<real_type_t<T>>(im));
        return;
    }
    if (n > 0 && !a) throw std::invalid_argument("pdiag_logdet: null local matrix");
    logdet_core<T>(h, n, a, desc[DDLA_LLD_], result, "pdiag_logdet");
}

// One rank's share of pdiag_logdet on a pr x pc grid (src/PBLAS/pdiag_logdet.cpp:11-48):
// the descriptor is checked against that grid (not the handle's), then the
// DiagLogTerm / DiagLogJoin reduction runs over the diagonal entries the rank
// holds.  state = {magnitude, phase, zero, negative parity, nonfinite}: the four
// doubles the reference all-reduces (pdiag_logdet.cpp:41-45) plus the nonfinite
// flag, which the reference raises on the rank that sees it before the
// reduction; carried through the sum, it lets every rank raise together.
template <typename T>
void pdiag_logdet_local(const DdlaHandle_t& h, int n, const T* a, const int* desc, int pr, int pc, int row, int col,
                        double state[5])
{
    detail::require_gpu(h, "pdiag_logdet");
    if (desc == nullptr) throw std::invalid_argument("ddla: null ScaLAPACK descriptor");
    if (pr <= 0 || pc <= 0 || row < 0 || row >= pr || col < 0 || col >= pc)
        throw std::invalid_argument("pdiag_logdet: grid coordinates outside the grid");
    if (desc[DDLA_DTYPE_] != DDLA_BLOCK_CYCLIC_2D || desc[DDLA_M_] < 0 || desc[DDLA_N_] < 0 || desc[DDLA_MB_] <= 0 ||
        desc[DDLA_NB_] <= 0 || desc[DDLA_RSRC_] < 0 || desc[DDLA_RSRC_] >= pr || desc[DDLA_CSRC_] < 0 ||
        desc[DDLA_CSRC_] >= pc)
        throw std::invalid_argument("pdiag_logdet: descriptor does not describe a matrix on this grid");
    const int rows = num_loc(desc[DDLA_M_], desc[DDLA_MB_], row, desc[DDLA_RSRC_], pr);
    if (desc[DDLA_LLD_] < std::max(1, rows))
        throw std::invalid_argument("pdiag_logdet: LLD_ smaller than the local row count");
    if (n < 0 || n > desc[DDLA_M_] || n > desc[DDLA_N_])
        throw std::invalid_argument("pdiag_logdet: order exceeds descriptor");
    const int lr = num_loc(n, desc[DDLA_MB_], row, desc[DDLA_RSRC_], pr);
    const int lc = num_loc(n, desc[DDLA_NB_], col, desc[DDLA_CSRC_], pc);
    if (lr > 0 && lc > 0 && !a) throw std::invalid_argument("pdiag_logdet: null local matrix");
    if (lr > 0 && lc > 0) {
        const auto last = std::uint64_t(lc - 1) * std::uint64_t(desc[DDLA_LLD_]) + std::uint64_t(lr) - 1;
        if (last > std::uint64_t(std::numeric_limits<std::ptrdiff_t>::max()) / sizeof(T))
            throw std::overflow_error("pdiag_logdet: matrix address span is not representable");
    }
    struct {
        double mag, phase;
        int flags, pad;
    } st{};
    if (lr > 0 && lc > 0) {
        detail::DeviceScratch work(h, static_cast<std::size_t>(ddlak_logdet_workspace()));
        detail::kernel_check(ddlak_diag_logsum_grid(tcode<T>(), n, a, desc[DDLA_LLD_], lr, lc, desc[DDLA_MB_],
                                                    desc[DDLA_NB_], pr, pc, row, col, desc[DDLA_RSRC_],
                                                    desc[DDLA_CSRC_], work.data(), h->stream),
                             "pdiag_logdet kernels");
        detail::cuda_check(cudaMemcpyAsync(h->host_word, work.data(), sizeof(st), cudaMemcpyDeviceToHost, h->stream),
                           "logdet read-back");
        detail::cuda_check(cudaStreamSynchronize(h->stream), "stream synchronisation");
        std::memcpy(&st, h->host_word, sizeof(st));
    }
    state[0] = st.mag;
    state[1] = st.phase;
    state[2] = double((st.flags & 2) != 0);
    state[3] = double((st.flags & 4) != 0);
    state[4] = double((st.flags & 1) != 0);
}

// finish_diagonal_log of the summed states (src/diag_logdet_impl.h:104-113;
// pdiag_logdet.cpp:46-47): zero wins, else the negative-real parity adds pi and
// the phase is wrapped to (-pi, pi]; a nonfinite entry on any rank throws.
void pdiag_logdet_finish(const double total[5], double& re, double& im)
{
    if (total[4] != 0) throw std::domain_error("pdiag_logdet: nonfinite diagonal");
    if (total[2] != 0) {
        re = -std::numeric_limits<double>::infinity();
        im = 0;
        return;
    }
    const double pi = std::acos(-1.0);
    double phase = std::remainder(total[1] + (static_cast<long long>(total[3]) & 1) * pi, 2 * pi);
    if (phase <= -pi) phase = pi;
    re = total[0];
    im = phase;
}

#define DDLA_INSTANTIATE(T)                                                                                          \
    template void pdiag_logdet_local<T>(const DdlaHandle_t&, int, const T*, const int*, int, int, int, int,          \
                                        double*);                                                                    \
    template void ppotrf<T>(const DdlaHandle_t&, char, int, T*, int, int, const int*, int&);                         \
    template void ppotrs<T>(const DdlaHandle_t&, char, char, char, int, int, const T*, const int*, T*, const int*); \
    template void pposv<T>(const DdlaHandle_t&, char, char, char, int, int, T*, int, int, const int*, T*, int, int, \
                           const int*, int&);                                                                        \
    template void potrf<T>(const DdlaHandle_t&, char, int, T*, int, int*);                                          \
    template void diag_logdet<T>(const DdlaHandle_t&, int, const T*, int, std::complex<real_type_t<T>>&);           \
    template void pdiag_logdet<T>(const DdlaHandle_t&, int, const T*, const int*, std::complex<real_type_t<T>>&);   \
    template void cholesky_impl::ppotrf_workspace_size<T>(const DdlaHandle_t&, char, int, const T*, const int*,      \
                                                          std::size_t*, std::size_t*);                               \
    template void cholesky_impl::ppotrf_run<T>(const DdlaHandle_t&, char, int, T*, int, int, const int*, int&,       \
                                               void*, std::size_t, void*, std::size_t);                              \
    template void cholesky_impl::ppotrs_workspace_size<T>(const DdlaHandle_t&, char, int, int, const int*,           \
                                                          const int*, std::size_t*, std::size_t*);                   \
    template void cholesky_impl::ppotrs_run<T>(const DdlaHandle_t&, char, char, char, int, int, const T*,           \
                                               const int*, T*, const int*, void*, std::size_t, void*, std::size_t); \
    template void potrf_bottom_right<T>(char, int, T*, int, int&, const DdlaHandle_t&);                             \
    template void ppotrf_bottom_right<T>(const DdlaHandle_t&, char, int, T*, const int*, int&);                     \
    template void cholesky_impl::ppotrf_bottom_right_workspace_size<T>(const DdlaHandle_t&, char, int, T*,           \
                                                                       const int*, std::size_t*, std::size_t*);     \
    template void cholesky_impl::ppotrf_bottom_right_run<T>(const DdlaHandle_t&, char, int, T*, const int*, int&,    \
                                                            void*, std::size_t, void*, std::size_t);

DDLA_INSTANTIATE(float)
DDLA_INSTANTIATE(double)
DDLA_INSTANTIATE(std::complex<float>)
DDLA_INSTANTIATE(std::complex<double>)
#undef DDLA_INSTANTIATE

}  // namespace ddla
