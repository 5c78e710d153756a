"""Build the CPU oracle (test infrastructure, never part of the product).

    python oracle/build.py

Compiles oracle/ddla_oracle.c with gcc into oracle/liboracle_ddla.so.  The
reference's own sources are not compiled: its Cholesky path needs MPI, a BLAS
library and the generated src/public_dispatch.cpp, so oracle/_ref stays empty
and the restatement in ddla_oracle.c (plus the LAPACK arm in lapack_arm.py) is
the oracle.
"""
from __future__ import annotations

import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "ddla_oracle.c"
LIB = HERE / "liboracle_ddla.so"


def build(force: bool = False) -> Path:
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    cc = shutil.which("gcc") or "cc"
    cmd = [cc, "-std=c99", "-O2", "-fno-fast-math", "-ffp-contract=off", "-fPIC", "-shared", str(SRC), "-o",
           str(LIB), "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
