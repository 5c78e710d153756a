// ddla::pposv_mixed -- FP64-accurate Hermitian positive-definite solve from a
// low-precision tensor-core Cholesky factor plus refinement (no reference
// counterpart; the LAPACK ?sposv contract).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <vector>

#include <ddla/ddla.h>
#include <ddla_kernels.h>

#include "ddla_stream.h"

namespace ddla {

void pposv_mixed(const DdlaHandle_t& h, char uplo, char precision, int n, int nrhs, double* A, const int* descA,
                 const double* B, const int* descB, double* X, const int* descX, int& info, MixedReport* report)
{
    detail::check_desc(descA, h);
    detail::check_desc(descB, h);
    detail::check_desc(descX, h);
    detail::require_gpu(h, "pposv_mixed");
    if (uplo != 'L' || (precision != 'B' && precision != 'T' && precision != 'D') || n < 0 || nrhs < 0 ||
        n > descA[DDLA_M_] || n > descA[DDLA_N_] || n > descB[DDLA_M_] || nrhs > descB[DDLA_N_] ||
        n > descX[DDLA_M_] || nrhs > descX[DDLA_N_])
        throw std::invalid_argument("pposv_mixed: invalid triangle, precision or dimensions");
    if (n && (!A || (nrhs && (!B || !X)))) throw std::invalid_argument("pposv_mixed: null matrix");
    MixedReport rep;
    info = 0;
    if (n == 0) {
        if (report) *report = rep;
        return;
    }
    if (precision != 'D') throw std::invalid_argument("pposv_mixed: low-precision factor not available");
    const long long ldb = descB[DDLA_LLD_], ldx = descX[DDLA_LLD_];
    if (nrhs)
        detail::cuda_check(cudaMemcpy2DAsync(X, ldx * sizeof(double), B, ldb * sizeof(double), n * sizeof(double),
                                             nrhs, cudaMemcpyDeviceToDevice, h->stream),
                           "copy B to X");
    pposv<double>(h, 'L', 'L', 'N', n, nrhs, A, 1, 1, descA, X, 1, 1, descX, info);
    if (report) *report = rep;
}

}  // namespace ddla
