"""ctypes binding of libddla_c.so -- the mirror of the reference's python/ddla/_c_api.py.

Same status constants, exception classes, descriptor offsets and library
search (DDLA_LIB_PATH, DDLA_DIR, LD_LIBRARY_PATH) as the reference
(python/ddla/_c_api.py:1-115); the in-tree build (libddla_b200/libddla_c.so)
is the final candidate.  Importing this module fails loudly when the native
library is missing: there is no Python fallback.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

STATUS_SUCCESS = 0
STATUS_INVALID_HANDLE = 1
STATUS_INVALID_VALUE = 2
STATUS_ALLOC_FAILED = 3
STATUS_BACKEND_UNAVAILABLE = 4
STATUS_INTERNAL_ERROR = 5
STATUS_EXCEPTION = 6

BACKEND_CPU = 0
BACKEND_GPU = 1

COMMUNICATION_MPI = 0
COMMUNICATION_HOST_STAGED_MPI = 1
COMMUNICATION_CCL = 2

DTYPE_ = 0
CTXT_ = 1
M_ = 2
N_ = 3
MB_ = 4
NB_ = 5
RSRC_ = 6
CSRC_ = 7
LLD_ = 8
DLEN_ = 9


class DdlaError(Exception):
    pass


class DdlaInvalidHandleError(DdlaError):
    pass


class DdlaInvalidValueError(DdlaError):
    pass


class DdlaAllocFailedError(DdlaError):
    pass


class DdlaBackendUnavailableError(DdlaError):
    pass


class DdlaInternalError(DdlaError):
    pass


class DdlaExceptionError(DdlaError):
    pass


_ERRORS = {
    STATUS_INVALID_HANDLE: DdlaInvalidHandleError,
    STATUS_INVALID_VALUE: DdlaInvalidValueError,
    STATUS_ALLOC_FAILED: DdlaAllocFailedError,
    STATUS_BACKEND_UNAVAILABLE: DdlaBackendUnavailableError,
    STATUS_INTERNAL_ERROR: DdlaInternalError,
    STATUS_EXCEPTION: DdlaExceptionError,
}

LIB_NAME = "libddla_c.so"


def library_path() -> Path:
    here = Path(__file__).resolve().parent
    candidates = []
    if os.environ.get("DDLA_LIB_PATH"):
        candidates.append(Path(os.environ["DDLA_LIB_PATH"]))
    if os.environ.get("DDLA_DIR"):
        d = Path(os.environ["DDLA_DIR"])
        candidates += [d / "lib" / LIB_NAME, d / "lib64" / LIB_NAME]
    for p in os.environ.get("LD_LIBRARY_PATH", "").split(":"):
        if p:
            candidates.append(Path(p) / LIB_NAME)
    candidates.append(here.parent / LIB_NAME)
    for c in candidates:
        if c.exists():
            return c
    raise OSError(f"{LIB_NAME} not found (build it with `python -m libddla_b200.build` or set DDLA_LIB_PATH)")


lib = ctypes.CDLL(str(library_path()), mode=ctypes.RTLD_GLOBAL)

_vp = ctypes.c_void_p
_i = ctypes.c_int
_c = ctypes.c_char
_ll = ctypes.c_longlong
_ip = ctypes.POINTER(ctypes.c_int)
_llp = ctypes.POINTER(ctypes.c_longlong)
_dp = ctypes.POINTER(ctypes.c_double)

_SIGS = {
    "ddla_c_error_string": (ctypes.c_char_p, [_i]),
    "ddla_c_init_backend": (_i, [ctypes.POINTER(_vp), _i]),
    "ddla_c_set": (_i, [_vp, _i, _i, _i, _c]),
    "ddla_c_local_group_create": (_i, [ctypes.POINTER(_vp), _i, ctypes.c_double]),
    "ddla_c_local_group_destroy": (_i, [_vp]),
    "ddla_c_set_local_group": (_i, [_vp, _vp, _i, _i, _i, _c]),
    "ddla_c_nccl_available": (_i, []),
    "ddla_c_nccl_unique_id": (_i, [_vp]),
    "ddla_c_set_nccl": (_i, [_vp, _vp, _i, _i, _i, _i, _c]),
    "ddla_c_set_communication": (_i, [_vp, _i]),
    "ddla_c_get_communication": (_i, [_vp, _ip]),
    "ddla_c_communication_available": (_i, [_vp, _i]),
    "ddla_c_destroy": (_i, [ctypes.POINTER(_vp)]),
    "ddla_c_backend_available": (_i, [_i]),
    "ddla_c_get_backend": (_i, [_vp]),
    "ddla_c_grid_dims": (_i, [_vp, _ip, _ip]),
    "ddla_c_grid_coords": (_i, [_vp, _ip, _ip]),
    "ddla_c_rank": (_i, [_vp]),
    "ddla_c_size": (_i, [_vp]),
    "ddla_c_descinit": (_i, [_vp, _vp, _i, _i, _i, _i, _i, _i, _i]),
    "ddla_c_numloc": (_i, [_i, _i, _i, _i, _i]),
    "ddla_c_malloc": (_i, [_vp, ctypes.POINTER(_vp), _ll]),
    "ddla_c_free": (_i, [_vp, _vp]),
    "ddla_c_memcpy": (_i, [_vp, _vp, _vp, _ll]),
    "ddla_c_memcpy2d": (_i, [_vp, _vp, _ll, _vp, _ll, _ll, _ll]),
    "ddla_c_memset": (_i, [_vp, _vp, _i, _ll]),
    "ddla_c_synchronize": (_i, [_vp]),
    "ddla_c_default_comm": (_i, []),
    "ddla_c_comm_rank": (_i, [_i]),
    "ddla_c_comm_size": (_i, [_i]),
    "ddla_c_finalize": (None, []),
    "ddla_c_bcast_dims": (_i, [_i, _ip, _ip, _ip, _i]),
    "ddla_d_pposv_mixed": (_i, [_vp, _c, _c, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _ip, _dp]),
    "ddla_d_pposv_mixed_host": (_i, [_vp, _c, _c, _i, _i, _vp, _i, _vp, _i, _vp, _i, _ip, _dp]),
    "ddla_c_get_stream": (_i, [_vp, ctypes.POINTER(_vp)]),
    "ddla_c_launch_count": (_ll, []),
    "ddla_c_pdiag_logdet_finish": (_i, [_vp, _i, _vp]),
    "ddla_c_fail_allocation": (_i, [_ll]),
    "ddla_c_live_workspaces": (_ll, []),
    "ddla_c_set_wait_budget": (_i, [_vp, _ll]),
    "ddla_c_profile_enable": (None, [_i]),
    "ddla_c_profile_read": (_i, [_i, _dp, _llp, _dp, _dp, _i]),
    "ddla_vbatched_plan_run": (_i, [_vp]),
    "ddla_vbatched_plan_info": (_i, [_vp, _ip, _dp]),
    "ddla_vbatched_plan_destroy": (_i, [_vp]),
    "ddla_vbatched_autotune": (_i, [_vp, _c, _i]),
    "ddla_vbatched_tuning": (_i, [_vp, _c, _i, _ip, _ip, ctypes.POINTER(ctypes.c_ubyte), _i, _ip]),
}
for _p in "sd":
    _SIGS.update({
        f"ddla_{_p}_posv_vbatched": (_i, [_vp, _c, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i]),
        f"ddla_{_p}_posv_vbatched_plan": (_i, [_vp, _c, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i, ctypes.POINTER(_vp)]),
        f"ddla_{_p}_chol_nll_batched": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
        f"ddla_{_p}_gp_nll_batched": (_i, [_vp, _i, _i, _i, _vp, _vp, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
        f"ddla_{_p}_chol_nll_grad_batched": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp]),
        f"ddla_{_p}_gp_nll_grad_batched": (_i, [_vp, _i, _i, _i, _vp, _vp, _i, _vp, _vp, _vp, _vp]),
    })
for _p in "sdcz":
    _SIGS.update({
        f"ddla_{_p}_gather": (_i, [_vp, _i, _i, _vp, _i, _i, _vp, _i, _vp, _i]),
        f"ddla_{_p}_scatter": (_i, [_vp, _i, _i, _vp, _i, _i, _vp, _i, _vp, _i]),
        f"ddla_{_p}_ppotrf": (_i, [_vp, _c, _i, _vp, _i, _i, _vp, _ip]),
        f"ddla_{_p}_ppotrs": (_i, [_vp, _c, _c, _c, _i, _i, _vp, _vp, _vp, _vp]),
        f"ddla_{_p}_pposv": (_i, [_vp, _c, _c, _c, _i, _i, _vp, _i, _i, _vp, _vp, _i, _i, _vp, _ip]),
        f"ddla_{_p}_potrf": (_i, [_vp, _c, _i, _vp, _i, _vp]),
        f"ddla_{_p}_diag_logdet": (_i, [_vp, _i, _vp, _i, _vp]),
        f"ddla_{_p}_pdiag_logdet": (_i, [_vp, _i, _vp, _vp, _vp]),
        f"ddla_{_p}_pdiag_logdet_local": (_i, [_vp, _i, _vp, _vp, _i, _i, _i, _i, _vp]),
        f"ddla_{_p}_potrf_bottom_right": (_i, [_vp, _c, _i, _vp, _i, _ip]),
        f"ddla_{_p}_ppotrf_bottom_right": (_i, [_vp, _c, _i, _vp, _vp, _ip]),
        f"ddla_{_p}_phegst": (_i, [_vp, _c, _i, _vp, _vp, _vp, _vp]),
        **({f"ddla_{_p}_gemm_vbatched_{v}": (_i, [_vp, _c, _c] + [_vp] * 11 + [_i]) for v in ("rc", "cr")}
           if _p in "cz" else {}),
        **({f"ddla_{_p}_gemm_vbatched2s_{v}": (_i, [_vp, _c, _c] + [_vp] * 11 + [_c, _c] + [_vp] * 10
                                               + [_i, _i, _vp, _i])
            for v in ("rzzr", "zrzr", "rzzz", "zrzz", "zzzr", "rrrz")} if _p in "cz" else {}),
        f"ddla_{_p}_gemm_vbatched": (_i, [_vp, _c, _c, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                          _i]),
        f"ddla_{_p}_gemm_vbatched2s": (_i, [_vp, _c, _c, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                            _c, _c, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _vp,
                                            _i]),
        f"ddla_{_p}_ppotrf_workspace_size": (_i, [_vp, _c, _i, _vp, _llp]),
        f"ddla_{_p}_ppotrf_run": (_i, [_vp, _c, _i, _vp, _vp, _ip, _vp, _ll]),
        f"ddla_{_p}_ppotrs_workspace_size": (_i, [_vp, _c, _i, _i, _vp, _vp, _llp]),
    })

for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args
    globals()[_name] = _f


def error_string(status: int) -> str:
    s = lib.ddla_c_error_string(int(status))
    return s.decode("utf-8", "replace") if s else ""


def check_status(status: int, where: str = "") -> None:
    if status == STATUS_SUCCESS:
        return
    cls = _ERRORS.get(status, DdlaError)
    raise cls(f"{where}: status {status}: {error_string(status)}")


class ddla_c_float_complex(ctypes.Structure):
    _fields_ = [("re", ctypes.c_float), ("im", ctypes.c_float)]


class ddla_c_double_complex(ctypes.Structure):
    _fields_ = [("re", ctypes.c_double), ("im", ctypes.c_double)]


def to_scalar(val, sfx: str):
    if sfx == "s":
        return ctypes.c_float(float(val))
    if sfx == "d":
        return ctypes.c_double(float(val))
    c = complex(val)
    if sfx == "c":
        return ddla_c_float_complex(c.real, c.imag)
    if sfx == "z":
        return ddla_c_double_complex(c.real, c.imag)
    raise ValueError(f"Unknown type suffix: {sfx}")
