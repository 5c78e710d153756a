"""The C-ABI library builds, loads and exports every declared symbol (CPU only, no compute calls)."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _declared(header: Path):
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    names = re.findall(r"\b(?:int|void|unsigned long long|const char\*)\s+\**\s*((?:ddla|ddlak)_\w+)\s*\(", text)
    return sorted(set(names))


def test_every_declared_symbol_is_exported(native_lib):
    lib = ctypes.CDLL(str(native_lib.library_path()))
    headers = sorted((ROOT / "include").glob("*.h"))
    assert headers, "no C-ABI headers"
    missing = []
    total = 0
    for h in headers:
        for name in _declared(h):
            total += 1
            if not hasattr(lib, name):
                missing.append(f"{h.name}:{name}")
    assert total > 60
    assert not missing, missing


def test_backend_queries_without_gpu(native_lib):
    C = native_lib
    # no CPU backend is built: there is no CPU fallback of the path
    assert C.ddla_c_backend_available(C.BACKEND_CPU) == 0
    h = ctypes.c_void_p()
    assert C.ddla_c_init_backend(ctypes.byref(h), C.BACKEND_CPU) == C.STATUS_BACKEND_UNAVAILABLE
    assert C.ddla_c_init_backend(ctypes.byref(h), 7) == C.STATUS_INVALID_VALUE
    assert C.ddla_c_numloc(10, 3, 0, 0, 1) == 10
    assert C.ddla_c_numloc(10, 3, 1, 0, 2) == 4  # blocks [3,6) and [9,10) on process 1 of 2
    assert C.ddla_c_comm_size(C.ddla_c_default_comm()) == 1
    assert C.error_string(C.STATUS_INVALID_VALUE) == "DDLA_STATUS_INVALID_VALUE"


def test_null_handle_statuses(native_lib):
    C = native_lib
    info = ctypes.c_int(-1)
    desc = (ctypes.c_int * 9)()
    assert C.ddla_d_ppotrf(None, b"L", 4, None, 1, 1, desc, ctypes.byref(info)) == C.STATUS_INVALID_HANDLE
    assert C.ddla_c_synchronize(None) == C.STATUS_INVALID_HANDLE
    h = ctypes.c_void_p()
    assert C.ddla_c_destroy(ctypes.byref(h)) == C.STATUS_SUCCESS


def test_oracle_is_not_linked_into_product():
    so = (ROOT / "libddla_b200" / "libddla_c.so").read_bytes()
    assert b"oracle_" not in so
    for src in (ROOT / "libddla_b200").rglob("*.py"):
        text = src.read_text()
        assert "import oracle" not in text and "from oracle" not in text, src
