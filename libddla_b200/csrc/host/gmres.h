// GMRES preconditioned by the low-precision Cholesky factor, for the
// correction equations of GMRES-IR (Carson & Higham, SIAM J. Sci. Comput. 2018):
// solve A d = r with left preconditioning M^-1 A d = M^-1 r, M = L L^T the FP32
// factor, all vectors and the Arnoldi process in FP64.  The nrhs columns run
// as independent Krylov spaces in lockstep: every kernel works on all columns
// at once, classical Gram-Schmidt with one reorthogonalization (CGS2) keeps the
// coefficients on the device, and the host sees one small read-back per
// iteration to advance each column's Givens rotations.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include <ddla/ddla_handle_t.h>

namespace ddla {

// M^-1 = (L L^T)^-1 applied in place to an n x nrhs FP64 block, L the FP32
// factor: by inverted diagonal super-blocks when `blocked` (FP32 arithmetic
// with the FP32 inverses Dinv32 when `single`, else FP64 arithmetic), else by
// the fused chain solve (ddlak_potrs_mixed, Dinv = 64-row block inverses).
struct MixedPreconditioner {
    DdlaHandle_t h = nullptr;
    int n = 0;
    int nrhs = 0;
    const float* L = nullptr;
    long long ldl = 0;
    const double* Dinv = nullptr;
    const float* Dinv32 = nullptr;
    bool blocked = false;
    bool single = false;
    void* work = nullptr;
    std::size_t bytes = 0;
    void apply(double* B, long long ldb) const;
};

class GmresIR {
public:
    static constexpr int kRestart = 30;

    static std::size_t workspace_bytes(int n, int nrhs, int m);

    GmresIR(const DdlaHandle_t& h, int n, int nrhs, const double* A, long long lda, const MixedPreconditioner& M,
            void* work, int m);

    // D = approximately A^-1 R (both n x nrhs, ld = n).  Runs at most maxit
    // Arnoldi steps, stopping early when every column's preconditioned
    // residual has dropped by the inner tolerance.  Returns the steps taken.
    int solve(const double* R, double* D, int maxit);

private:
    DdlaHandle_t h_;
    int n_, nrhs_, m_;
    const double* A_;
    long long lda_;
    MixedPreconditioner M_;
    double* V_;      // (m+1) blocks of n x nrhs
    double* Wv_;     // n x nrhs
    double* Z_;      // zeros, n x nrhs (the B of A*v = -(0 - A v))
    double* coef_;   // 2 x (m+1) x nrhs: CGS pass 1 and 2
    double* nrm2_;   // nrhs
};

}  // namespace ddla
