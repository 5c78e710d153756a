"""In-tree build of libddla_c.so (CUDA kernels + C++ host library + C ABI).

Every .cu under csrc/kernels and every .cpp under csrc/host is compiled with
nvcc for sm_100a only and linked into libddla_b200/libddla_c.so with the CUDA
runtime linked statically, so the library needs nothing at run time but the
driver.  Objects are rebuilt when a source or any header is newer.

    python -m libddla_b200.build [--force] [-j N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = ROOT / "_build" / "obj"
LIB = PKG / "libddla_c.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _sources() -> list[Path]:
    return sorted((CSRC / "kernels").glob("*.cu")) + sorted((CSRC / "host").glob("*.cpp"))


def _headers() -> list[Path]:
    hs = list((ROOT / "include").rglob("*.h"))
    for d in ("kernels", "host"):
        hs += list((CSRC / d).glob("*.h")) + list((CSRC / d).glob("*.cuh"))
    return hs


def _flags(src: Path) -> list[str]:
    common = ["-std=c++17", "-O3", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include"),
              "-I", str(CSRC / "kernels"), "-I", str(CSRC / "host")]
    if src.suffix == ".cu":
        return common + ARCH + ["-lineinfo", "--expt-relaxed-constexpr", "-Xptxas", "-O3"]
    return common + ["-x", "cu"] + ARCH  # host TUs also go through nvcc (same toolchain, cuda headers)


def _compile(src: Path, force: bool, verbose: bool) -> Path:
    obj = OBJ / (src.parent.name + "_" + src.stem + ".o")
    newest_dep = max([src.stat().st_mtime] + [h.stat().st_mtime for h in _headers()])
    if not force and obj.exists() and obj.stat().st_mtime >= newest_dep:
        return obj
    cmd = [nvcc(), *_flags(src), "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src}\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    OBJ.mkdir(parents=True, exist_ok=True)
    srcs = _sources()
    jobs = jobs or min(8, os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [nvcc(), "-shared", *ARCH, "-cudart", "static", "-o", str(LIB), *map(str, objs),
               "-Xlinker", "-soname=libddla_c.so", "-lpthread", "-ldl", "-lrt"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, jobs=a.j, verbose=a.v))


if __name__ == "__main__":
    sys.exit(main())
