"""ddla -- Python binding of the B200 Cholesky path (mirror of the reference's python/ddla).

    from libddla_b200 import ddla
    with ddla.Handle(ddla.Backend.GPU) as h:
        A = ddla.DistributedMatrix.from_global_matrix(h, a, mb=256, nb=256)
        B = ddla.DistributedMatrix.from_global_matrix(h, b, mb=256, nb=256)
        X, info = ddla.pposv(A, B, uplo="L")
"""
from ._c_api import (  # noqa: F401
    BACKEND_CPU, BACKEND_GPU, COMMUNICATION_CCL, COMMUNICATION_HOST_STAGED_MPI, COMMUNICATION_MPI, CSRC_, CTXT_,
    DLEN_, DTYPE_, LLD_, M_, MB_, N_, NB_, RSRC_, STATUS_ALLOC_FAILED, STATUS_BACKEND_UNAVAILABLE, STATUS_EXCEPTION,
    STATUS_INTERNAL_ERROR, STATUS_INVALID_HANDLE, STATUS_INVALID_VALUE, STATUS_SUCCESS, DdlaAllocFailedError,
    DdlaBackendUnavailableError, DdlaError, DdlaExceptionError, DdlaInternalError, DdlaInvalidHandleError,
    DdlaInvalidValueError, library_path,
)
from .backend import Backend, Communication, Handle  # noqa: F401
from .layout import ProcessorLayout  # noqa: F401
from .matrix import DistributedMatrix  # noqa: F401
from . import autograd, batched, grid  # noqa: F401
from .ops import (diag_logdet, gather, pdiag_logdet, pdiag_logdet_finish, pdiag_logdet_grid,  # noqa: F401
                  pdiag_logdet_local, phegst, potrf, potrf_bottom_right, pposv, pposv_mixed, pposv_mixed_host, ppotrf,
                  ppotrf_bottom_right, ppotrs, scatter)


def finalize():
    from ._c_api import ddla_c_finalize

    ddla_c_finalize()


__version__ = "0.1.0"
