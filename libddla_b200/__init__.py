"""libddla_b200 -- B200-native (sm_100a) drop-in for LibDDLA's Cholesky path.

The product is the native library libddla_c.so (hand-written CUDA kernels,
C++ ddla API and the reference's C ABI); `libddla_b200.ddla` is the ctypes
binding that mirrors the reference's python/ddla package.
"""
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
LIBRARY = PACKAGE_DIR / "libddla_c.so"
