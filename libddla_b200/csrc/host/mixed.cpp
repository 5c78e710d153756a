// ddla::pposv_mixed -- FP64-accurate Hermitian positive-definite solve from a
// low-precision tensor-core Cholesky factor plus refinement (no reference
// counterpart; the contract of LAPACK ?sposv).
//
//   1. W = fl32(A) (lower), ||A||_inf from the full symmetric A;
//   2. W = L L^T with the trailing updates on the tensor cores (BF16 or TF32
//      operands, FP32 accumulation and storage, FP64 diagonal blocks); when the
//      low-precision factorization breaks down, W is rebuilt with the diagonal
//      scaled by 1 + c*u (a relative shift) and factored again;
//   3. X = L^-T L^-1 B with the FP32 factor (FP32 solves by inverted diagonal
//      super-blocks for up to 16 right-hand sides, as ?sposv's single-precision
//      solves; the fused chain with FP64 vectors beyond);
//   4. refinement: R = B - A X in FP64 against the untouched A, D = L^-T L^-1 R,
//      X += D, until every column meets ||r|| <= ||x|| ||A|| eps sqrt(n) (the
//      ?sposv test); when a sweep fails to halve the scaled residual the
//      correction is computed by GMRES preconditioned by the factor instead;
//   5. if neither converges within the budget, the FP64 path (ppotrf/ppotrs on A)
//      produces X and iter = -(sweeps + 1).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include <ddla/ddla.h>
#include <ddla/ddla_desc.h>
#include <ddla_kernels.h>

#include "ddla_stream.h"
#include "gmres.h"

namespace ddla {

namespace {

constexpr int kMaxSweeps = 30;        // as ?sposv's ITERMAX
constexpr int kMaxShiftTries = 4;

void ck(int e, const char* what) { detail::kernel_check(e, what); }

struct Scalars {
    double anrm;
    int info;
    int status;
};

}  // namespace

namespace {

// Where the first factorization takes A from when A is still in host memory:
// the lower part arrives by column panels on copy_stream while the panels that
// have arrived are factored (ddlak_potrf_mixed_stream).
struct HostSource {
    const double* A;
    long long lda;
    cudaStream_t copy_stream;
};

void mixed_core(const DdlaHandle_t& h, char precision, int n, int nrhs, double* A, long long lda, const double* B,
                long long ldb, double* X, long long ldx, int& info, MixedReport* report, const HostSource* src)
{
    MixedReport rep;
    info = 0;
    if (report) *report = rep;
    if (n == 0) return;
    cudaStream_t st = h->stream;
    // descriptors of the device-resident operands for the FP64 path (1x1 grid)
    const int nbd = 256;
    const int descA[9] = {DDLA_BLOCK_CYCLIC_2D, 0, n, n, nbd, nbd, 0, 0, (int)lda};
    const int descX[9] = {DDLA_BLOCK_CYCLIC_2D, 0, n, std::max(1, nrhs), nbd, nbd, 0, 0, (int)ldx};
    auto copy_b_to_x = [&] {
        if (nrhs)
            detail::cuda_check(cudaMemcpy2DAsync(X, ldx * sizeof(double), B, ldb * sizeof(double),
                                                 n * sizeof(double), nrhs, cudaMemcpyDeviceToDevice, st),
                               "copy B to X");
    };
    auto fp64_path = [&](int sweeps) {
        copy_b_to_x();
        pposv<double>(h, 'L', 'L', 'N', n, nrhs, A, 1, 1, descA, X, 1, 1, descX, info);
        rep.iter = precision == 'D' ? 0 : -(sweeps + 1);
        if (report) *report = rep;
    };
    if (precision == 'D') {
        fp64_path(0);
        return;
    }
    if (nrhs == 0) return;

    // ---- workspace ----------------------------------------------------------
    const long long ldw = (n + 3) / 4 * 4;
    const std::size_t pbytes = ddlak_mixed_panel_bytes(n);
    // refinement solves: inverted diagonal super-blocks for up to 16 right-hand
    // sides, the fused chain with 64-row block inverses beyond
    const bool blocked = nrhs <= 16;
    const std::size_t sbytes = blocked ? ddlak_bis_solve_workspace(n, std::max(1, nrhs))
                                       : ddlak_potrs_workspace(n, std::max(1, nrhs));
    const std::size_t dinv_bytes = blocked ? ddlak_bis_inverse_bytes(n) : ddlak_inv_diag_bytes(n);
    const std::size_t dinv32_bytes = blocked ? detail::padded_bytes<float>(ddlak_bis_inverse_bytes(n) / 8) : 0;
    const int kry = GmresIR::kRestart;
    long long ldk = 0;
    const std::size_t lk_bytes = src ? (std::size_t)ddlak_mixed_lk_bytes(precision, n, &ldk) : 0;
    const std::size_t bytes = detail::padded_bytes<float>((std::size_t)ldw * n) + 2 * pbytes +
                              (lk_bytes ? (lk_bytes + 255) / 256 * 256 : 0) +
                              3 * detail::padded_bytes<double>((std::size_t)n * std::max(1, nrhs)) +
                              detail::padded_bytes<double>(n) + detail::padded_bytes<Scalars>(1) +
                              2 * detail::padded_bytes<double>(std::max(1, nrhs)) + sbytes +
                              GmresIR::workspace_bytes(n, std::max(1, nrhs), kry) + dinv_bytes + dinv32_bytes + 256;
    detail::DeviceScratch ws(h, bytes);
    char* w = ws.data();
    float* W = detail::take<float>(w, (std::size_t)ldw * n);
    void* Lk = w;
    w += lk_bytes ? (lk_bytes + 255) / 256 * 256 : 0;
    void* P0 = w;
    w += pbytes;
    void* P1 = w;
    w += pbytes;
    double* R = detail::take<double>(w, (std::size_t)n * std::max(1, nrhs));
    double* D = detail::take<double>(w, (std::size_t)n * std::max(1, nrhs));
    double* Bc = detail::take<double>(w, (std::size_t)n * std::max(1, nrhs));
    double* colsum = detail::take<double>(w, n);
    double* Dinv = detail::take<double>(w, dinv_bytes / sizeof(double));
    float* Dinv32 = blocked ? detail::take<float>(w, ddlak_bis_inverse_bytes(n) / 8) : nullptr;
    Scalars* sc = detail::take<Scalars>(w, 1);
    double* xn = detail::take<double>(w, std::max(1, nrhs));
    double* rn = detail::take<double>(w, std::max(1, nrhs));
    void* swork = w;
    w += sbytes;
    void* gwork = w;

    Scalars hs{};
    auto read_scalars = [&] {
        detail::cuda_check(cudaMemcpyAsync(h->host_word, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st),
                           "scalar read-back");
        detail::cuda_check(cudaStreamSynchronize(st), "stream synchronisation");
        std::memcpy(&hs, h->host_word, sizeof(Scalars));
    };

    // ---- 1 + 2: convert and factor (with a relative diagonal shift on breakdown) ----
    const double u = precision == 'B' ? std::ldexp(1.0, -8) : std::ldexp(1.0, -11);
    double shift = 0.0;
    bool factored = false;
    for (int attempt = 0; attempt < kMaxShiftTries && !factored; ++attempt) {
        if (attempt == 0 && src) {
            // A arrives from host memory while it is factored; every later attempt
            // (a shifted diagonal) starts from the device copy it leaves behind
            ck(ddlak_potrf_mixed_stream(precision, DDLAK_MIXED_GROUP, n, src->A, src->lda, A, lda, W, ldw, Lk, ldk,
                                        colsum, &sc->anrm, &sc->info, &sc->status, src->copy_stream, st),
               "streamed mixed factorization");
        } else {
            ck(ddlak_convert_lower(n, A, lda, W, ldw, 1.0 + shift, colsum, &sc->anrm, st), "convert to FP32");
            ck(ddlak_potrf_mixed(precision, n, W, ldw, P0, P1, &sc->info, &sc->status, st), "mixed factorization");
        }
        read_scalars();
        if (hs.status != 0) throw std::runtime_error("pposv_mixed: a tensor-core update wait timed out");
        if (hs.info == 0) factored = true;
        else shift = shift == 0.0 ? 2.0 * u : shift * 8.0;
    }
    rep.shift = factored ? shift : 0.0;
    const double anrm = hs.anrm;
    if (!factored || !(anrm > 0) || !std::isfinite(anrm) || nrhs == 0) {
        fp64_path(0);
        return;
    }

    // ---- 3: initial solve ----------------------------------------------------------
    const double eps = std::numeric_limits<double>::epsilon() / 2;  // unit roundoff, as LAPACK dlamch('E')
    const double cte = anrm * eps * std::sqrt((double)n);
    detail::cuda_check(cudaMemcpy2DAsync(Bc, n * sizeof(double), B, ldb * sizeof(double), n * sizeof(double), nrhs,
                                         cudaMemcpyDeviceToDevice, st),
                       "copy B");
    detail::cuda_check(cudaMemcpy2DAsync(X, ldx * sizeof(double), Bc, n * sizeof(double), n * sizeof(double), nrhs,
                                         cudaMemcpyDeviceToDevice, st),
                       "copy B to X");
    if (blocked) {
        detail::DeviceScratch tmp(h, ddlak_bis_inverse_bytes(n));
        ck(ddlak_bis_inverse(n, W, ldw, Dinv, tmp.data(), st), "diagonal block inverses");
        ck(ddlak_bis_inverse_narrow(n, Dinv, Dinv32, st), "FP32 diagonal block inverses");
    } else {
        ck(ddlak_inv_diag_blocks(n, W, ldw, Dinv, st), "diagonal block inverses");
    }
    MixedPreconditioner M;
    M.h = h;
    M.n = n;
    M.nrhs = nrhs;
    M.L = W;
    M.ldl = ldw;
    M.Dinv = Dinv;
    M.Dinv32 = Dinv32;
    M.blocked = blocked;
    M.single = blocked;  // classic sweeps: FP32 solves; GmresIR keeps its copy in FP64
    M.work = swork;
    M.bytes = sbytes;
    M.apply(X, ldx);

    std::vector<double> hx(nrhs), hr(nrhs);
    auto residual_check = [&](double& worst) -> bool {
        ck(ddlak_symm_residual(n, nrhs, A, lda, X, ldx, Bc, n, R, n, st), "residual");
        ck(ddlak_colmax(n, nrhs, X, ldx, xn, st), "norm x");
        ck(ddlak_colmax(n, nrhs, R, n, rn, st), "norm r");
        detail::cuda_check(cudaMemcpyAsync(hx.data(), xn, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, st), "norms");
        detail::cuda_check(cudaMemcpyAsync(hr.data(), rn, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, st), "norms");
        detail::cuda_check(cudaStreamSynchronize(st), "stream synchronisation");
        bool ok = true;
        worst = 0;
        for (int j = 0; j < nrhs; ++j) {
            if (!std::isfinite(hr[j]) || !std::isfinite(hx[j])) return false;
            ok = ok && hr[j] <= hx[j] * cte;
            worst = std::max(worst, hx[j] > 0 ? hr[j] / (hx[j] * anrm) : (hr[j] > 0 ? INFINITY : 0.0));
        }
        return ok;
    };

    // ---- 4: refinement ---------------------------------------------------------------
    double worst = 0, prev = INFINITY;
    int sweeps = 0;
    bool use_gmres = false;
    GmresIR gmres(h, n, nrhs, A, lda, M, gwork, kry);
    while (true) {
        const bool ok = residual_check(worst);
        rep.backward_error = worst;
        if (ok) {
            rep.iter = sweeps;
            rep.gmres = use_gmres ? 1 : 0;
            if (report) *report = rep;
            return;
        }
        if (!std::isfinite(worst) || sweeps >= kMaxSweeps) break;
        if (!use_gmres && sweeps > 0 && worst > 0.5 * prev) use_gmres = true;  // IR stagnates: switch to GMRES-IR
        prev = worst;
        if (use_gmres) {
            // D = A^-1 R by left-preconditioned GMRES; each Krylov iteration counts as a sweep
            const int its = gmres.solve(R, D, std::min(kry, kMaxSweeps - sweeps));
            sweeps += std::max(1, its);
        } else {
            detail::cuda_check(cudaMemcpyAsync(D, R, sizeof(double) * n * nrhs, cudaMemcpyDeviceToDevice, st),
                               "copy residual");
            M.apply(D, n);
            ++sweeps;
        }
        ck(ddlak_axpy(n, nrhs, 1.0, D, n, X, ldx, st), "update x");
    }
    rep.gmres = use_gmres ? 1 : 0;
    // ---- 5: FP64 fallback ---------------------------------------------------------------
    fp64_path(sweeps);
}

}  // namespace

void pposv_mixed(const DdlaHandle_t& h, char uplo, char precision, int n, int nrhs, double* A, const int* descA,
                 const double* B, const int* descB, double* X, const int* descX, int& info, MixedReport* report)
{
    detail::check_desc(descA, h);
    detail::check_desc(descB, h);
    detail::check_desc(descX, h);
    detail::require_gpu(h, "pposv_mixed");
    if (h->nprocs > 1) throw std::invalid_argument("pposv_mixed: served on a 1x1 grid only");
    if (uplo != 'L' || (precision != 'B' && precision != 'T' && precision != 'D') || n < 0 || nrhs < 0 ||
        n > descA[DDLA_M_] || n > descA[DDLA_N_] || n > descB[DDLA_M_] || nrhs > descB[DDLA_N_] ||
        n > descX[DDLA_M_] || nrhs > descX[DDLA_N_])
        throw std::invalid_argument("pposv_mixed: invalid triangle, precision or dimensions");
    if (n && (!A || (nrhs && (!B || !X)))) throw std::invalid_argument("pposv_mixed: null matrix");
    mixed_core(h, precision, n, nrhs, A, descA[DDLA_LLD_], B, descB[DDLA_LLD_], X, descX[DDLA_LLD_], info, report,
               nullptr);
}

void pposv_mixed_host(const DdlaHandle_t& h, char uplo, char precision, int n, int nrhs, const double* A, int lda,
                      const double* B, int ldb, double* X, int ldx, int& info, MixedReport* report)
{
    detail::require_gpu(h, "pposv_mixed_host");
    if (h->nprocs > 1) throw std::invalid_argument("pposv_mixed_host: served on a 1x1 grid only");
    if (uplo != 'L' || (precision != 'B' && precision != 'T' && precision != 'D') || n < 0 || nrhs < 0 ||
        lda < std::max(1, n) || ldb < std::max(1, n) || ldx < std::max(1, n))
        throw std::invalid_argument("pposv_mixed_host: invalid triangle, precision, dimensions or leading dimensions");
    if (n && (!A || (nrhs && (!B || !X)))) throw std::invalid_argument("pposv_mixed_host: null matrix");
    info = 0;
    if (report) *report = MixedReport{};
    if (n == 0) return;
    cudaStream_t st = h->stream;
    // device copies: A (lower part only is ever written or read; even leading
    // dimension for the FP64 tile maps of the residual), B and X
    const long long ldad = n + (n & 1);
    const std::size_t rhs_bytes = detail::padded_bytes<double>((std::size_t)n * std::max(1, nrhs));
    detail::DeviceScratch dev(h, detail::padded_bytes<double>((std::size_t)ldad * n) + 2 * rhs_bytes);
    double* dA = reinterpret_cast<double*>(dev.data());
    double* dB = reinterpret_cast<double*>(dev.data() + detail::padded_bytes<double>((std::size_t)ldad * n));
    double* dX = reinterpret_cast<double*>(reinterpret_cast<char*>(dB) + rhs_bytes);
    if (nrhs)
        detail::cuda_check(cudaMemcpy2DAsync(dB, sizeof(double) * n, B, sizeof(double) * ldb, sizeof(double) * n,
                                             nrhs, cudaMemcpyHostToDevice, st),
                           "copy B to the device");
    // the copy stream starts after the allocations on the handle stream
    struct CopyStream {
        cudaStream_t s = nullptr;
        cudaEvent_t ready = nullptr;
        ~CopyStream()
        {
            if (ready) cudaEventDestroy(ready);
            if (s) cudaStreamDestroy(s);
        }
    } cs;
    detail::cuda_check(cudaStreamCreateWithFlags(&cs.s, cudaStreamNonBlocking), "copy stream");
    detail::cuda_check(cudaEventCreateWithFlags(&cs.ready, cudaEventDisableTiming), "copy stream event");
    detail::cuda_check(cudaEventRecord(cs.ready, st), "copy stream event");
    detail::cuda_check(cudaStreamWaitEvent(cs.s, cs.ready, 0), "copy stream event");
    try {
        if (precision == 'D' || nrhs == 0) {
            // no tensor-core factor to overlap: the lower part of A in column panels, then the device routine
            const long long pw = 1024;
            for (long long c0 = 0; c0 < n; c0 += pw)
                detail::cuda_check(cudaMemcpy2DAsync(dA + c0 + c0 * ldad, sizeof(double) * ldad, A + c0 + c0 * lda,
                                                     sizeof(double) * lda, sizeof(double) * (n - c0),
                                                     (size_t)std::min(pw, n - c0), cudaMemcpyHostToDevice, st),
                                   "copy A to the device");
            mixed_core(h, precision, n, nrhs, dA, ldad, dB, n, dX, n, info, report, nullptr);
        } else {
            const HostSource src{A, lda, cs.s};
            mixed_core(h, precision, n, nrhs, dA, ldad, dB, n, dX, n, info, report, &src);
        }
        if (nrhs)
            detail::cuda_check(cudaMemcpy2DAsync(X, sizeof(double) * ldx, dX, sizeof(double) * n,
                                                 sizeof(double) * n, nrhs, cudaMemcpyDeviceToHost, st),
                               "copy X to the host");
        detail::cuda_check(cudaStreamSynchronize(st), "stream synchronisation");
        detail::cuda_check(cudaStreamSynchronize(cs.s), "stream synchronisation");
    } catch (...) {
        cudaStreamSynchronize(cs.s);
        cudaStreamSynchronize(st);
        throw;
    }
}

}  // namespace ddla
