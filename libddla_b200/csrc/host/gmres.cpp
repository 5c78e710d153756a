// GMRES-IR correction solves (see gmres.h).
#include "gmres.h"

#include <cmath>
#include <cstring>
#include <vector>

#include <ddla_kernels.h>

#include "ddla_stream.h"

namespace ddla {

namespace {
constexpr double kInnerTol = 1e-6;  // relative drop of the preconditioned residual per correction solve
void ck(int e, const char* what) { detail::kernel_check(e, what); }
}  // namespace

std::size_t GmresIR::workspace_bytes(int n, int nrhs, int m)
{
    const std::size_t blk = detail::padded_bytes<double>((std::size_t)n * nrhs);
    return (std::size_t)(m + 1) * blk + 2 * blk + detail::padded_bytes<double>(2 * (std::size_t)(m + 1) * nrhs) +
           detail::padded_bytes<double>(nrhs);
}

void MixedPreconditioner::apply(double* B, long long ldb) const
{
    if (blocked && single)
        ck(ddlak_bis_solve_f32(n, nrhs, L, ldl, Dinv32, B, ldb, work, bytes, h->stream), "preconditioner");
    else if (blocked)
        ck(ddlak_bis_solve(n, nrhs, L, ldl, Dinv, B, ldb, work, bytes, h->stream), "preconditioner");
    else
        ck(ddlak_potrs_mixed(n, nrhs, L, ldl, Dinv, B, ldb, work, bytes, h->stream), "preconditioner");
}

GmresIR::GmresIR(const DdlaHandle_t& h, int n, int nrhs, const double* A, long long lda, const MixedPreconditioner& M,
                 void* work, int m)
    : h_(h), n_(n), nrhs_(nrhs), m_(m), A_(A), lda_(lda), M_(M)
{
    M_.single = false;  // the Krylov basis needs the preconditioner applied in FP64
    char* w = static_cast<char*>(work);
    V_ = detail::take<double>(w, (std::size_t)(m + 1) * 0 + (std::size_t)n * nrhs);
    for (int i = 1; i <= m; ++i) (void)detail::take<double>(w, (std::size_t)n * nrhs);
    Wv_ = detail::take<double>(w, (std::size_t)n * nrhs);
    Z_ = detail::take<double>(w, (std::size_t)n * nrhs);
    coef_ = detail::take<double>(w, 2 * (std::size_t)(m + 1) * nrhs);
    nrm2_ = detail::take<double>(w, nrhs);
}

int GmresIR::solve(const double* R, double* D, int maxit)
{
    cudaStream_t st = h_->stream;
    const int n = n_, nc = nrhs_;
    const long long vstride = (long long)(detail::padded_bytes<double>((std::size_t)n * nc) / sizeof(double));
    auto Vi = [&](int i) { return V_ + i * vstride; };
    maxit = maxit < m_ ? maxit : m_;
    if (maxit < 1) maxit = 1;
    detail::cuda_check(cudaMemsetAsync(Z_, 0, sizeof(double) * n * nc, st), "zero block");

    // V_0 = M^-1 r / ||M^-1 r||
    detail::cuda_check(cudaMemcpyAsync(Vi(0), R, sizeof(double) * n * nc, cudaMemcpyDeviceToDevice, st), "copy r");
    M_.apply(Vi(0), n);
    ck(ddlak_multidot(Vi(0), 0, 1, Vi(0), n, nc, nrm2_, st), "norm");
    std::vector<double> beta(nc);
    detail::cuda_check(cudaMemcpyAsync(beta.data(), nrm2_, sizeof(double) * nc, cudaMemcpyDeviceToHost, st), "norm");
    ck(ddlak_scale_cols(Vi(0), Vi(0), n, nc, 1.0, nrm2_, st), "normalize");
    detail::cuda_check(cudaStreamSynchronize(st), "stream synchronisation");
    for (double& b : beta) b = std::sqrt(b);

    // per column: Hessenberg (m+1) x m, rotations, residual vector g
    std::vector<std::vector<double>> H(nc, std::vector<double>((std::size_t)(m_ + 1) * m_, 0.0));
    std::vector<std::vector<double>> cs(nc, std::vector<double>(m_)), sn(nc, std::vector<double>(m_));
    std::vector<std::vector<double>> g(nc, std::vector<double>(m_ + 1, 0.0));
    std::vector<int> kcol(nc, 0);
    std::vector<char> done(nc, 0);
    for (int c = 0; c < nc; ++c) {
        g[c][0] = beta[c];
        if (!(beta[c] > 0) || !std::isfinite(beta[c])) done[c] = 1;
    }
    std::vector<double> hc(2 * (std::size_t)(m_ + 1) * nc), hn(nc);
    double* c1 = coef_;
    double* c2 = coef_ + (std::size_t)(m_ + 1) * nc;
    int steps = 0;
    for (int j = 0; j < maxit; ++j) {
        bool all = true;
        for (int c = 0; c < nc; ++c) all = all && done[c];
        if (all) break;
        // w = M^-1 A V_j  (the residual kernel gives 0 - A V_j; the solve is linear)
        ck(ddlak_symm_residual(n, nc, A_, lda_, Vi(j), n, Z_, n, Wv_, n, st), "A v");
        M_.apply(Wv_, n);
        ck(ddlak_scale_cols(Wv_, Wv_, n, nc, -1.0, nullptr, st), "sign");
        // CGS2
        ck(ddlak_multidot(V_, vstride, j + 1, Wv_, n, nc, c1, st), "cgs dots");
        ck(ddlak_multi_axpy(V_, vstride, j + 1, c1, Wv_, n, nc, st), "cgs update");
        ck(ddlak_multidot(V_, vstride, j + 1, Wv_, n, nc, c2, st), "cgs dots");
        ck(ddlak_multi_axpy(V_, vstride, j + 1, c2, Wv_, n, nc, st), "cgs update");
        ck(ddlak_multidot(Wv_, 0, 1, Wv_, n, nc, nrm2_, st), "norm");
        ck(ddlak_scale_cols(Wv_, Vi(j + 1), n, nc, 1.0, nrm2_, st), "normalize");
        detail::cuda_check(cudaMemcpyAsync(hc.data(), c1, sizeof(double) * (j + 1) * nc, cudaMemcpyDeviceToHost, st),
                           "hessenberg");
        detail::cuda_check(cudaMemcpyAsync(hc.data() + (std::size_t)(m_ + 1) * nc, c2,
                                           sizeof(double) * (j + 1) * nc, cudaMemcpyDeviceToHost, st),
                           "hessenberg");
        detail::cuda_check(cudaMemcpyAsync(hn.data(), nrm2_, sizeof(double) * nc, cudaMemcpyDeviceToHost, st),
                           "hessenberg");
        detail::cuda_check(cudaStreamSynchronize(st), "stream synchronisation");
        ++steps;
        for (int c = 0; c < nc; ++c) {
            if (done[c]) continue;
            double* Hc = H[c].data();
            auto h = [&](int i, int k) -> double& { return Hc[(std::size_t)k * (m_ + 1) + i]; };
            for (int i = 0; i <= j; ++i)
                h(i, j) = hc[(std::size_t)i * nc + c] + hc[(std::size_t)(m_ + 1) * nc + (std::size_t)i * nc + c];
            h(j + 1, j) = std::sqrt(hn[c]);
            for (int i = 0; i < j; ++i) {
                const double t = cs[c][i] * h(i, j) + sn[c][i] * h(i + 1, j);
                h(i + 1, j) = -sn[c][i] * h(i, j) + cs[c][i] * h(i + 1, j);
                h(i, j) = t;
            }
            const double r = std::hypot(h(j, j), h(j + 1, j));
            if (!(r > 0) || !std::isfinite(r)) {
                done[c] = 1;
                continue;
            }
            cs[c][j] = h(j, j) / r;
            sn[c][j] = h(j + 1, j) / r;
            h(j, j) = r;
            h(j + 1, j) = 0.0;
            g[c][j + 1] = -sn[c][j] * g[c][j];
            g[c][j] = cs[c][j] * g[c][j];
            kcol[c] = j + 1;
            if (std::fabs(g[c][j + 1]) <= kInnerTol * beta[c]) done[c] = 1;
        }
    }
    // D = sum_i y_i V_i with H y = g per column (back substitution)
    std::vector<double> negy((std::size_t)m_ * nc, 0.0);
    int kmax = 0;
    for (int c = 0; c < nc; ++c) {
        const int k = kcol[c];
        kmax = k > kmax ? k : kmax;
        const double* Hc = H[c].data();
        std::vector<double> y(k);
        for (int i = k - 1; i >= 0; --i) {
            double s = g[c][i];
            for (int l = i + 1; l < k; ++l) s -= Hc[(std::size_t)l * (m_ + 1) + i] * y[l];
            y[i] = s / Hc[(std::size_t)i * (m_ + 1) + i];
        }
        for (int i = 0; i < k; ++i) negy[(std::size_t)i * nc + c] = -y[i];
    }
    detail::cuda_check(cudaMemsetAsync(D, 0, sizeof(double) * n * nc, st), "zero d");
    if (kmax > 0) {
        detail::cuda_check(cudaMemcpyAsync(c1, negy.data(), sizeof(double) * kmax * nc, cudaMemcpyHostToDevice, st),
                           "coefficients");
        ck(ddlak_multi_axpy(V_, vstride, kmax, c1, D, n, nc, st), "combine");
        detail::cuda_check(cudaStreamSynchronize(st), "stream synchronisation");
    }
    return steps;
}

}  // namespace ddla
