import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests" / "golden"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the native kernels")


def _ensure_built():
    from libddla_b200.build import build

    build()


@pytest.fixture(scope="session")
def native_lib():
    _ensure_built()
    from libddla_b200.ddla import _c_api

    return _c_api


@pytest.fixture(scope="session")
def handle(native_lib):
    from libddla_b200 import ddla

    if not ddla.Handle.is_backend_available(ddla.Backend.GPU):
        pytest.fail("GPU test without a visible CUDA device")
    h = ddla.Handle(ddla.Backend.GPU)
    yield h
    h.destroy()


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    d = ROOT / "tests" / "golden"
    return {name: np.load(d / f"{name}.npz") for name in ("kat", "real_spd", "hpd", "logdet", "python")}
