"""In-tree build of the CUDA engine ``libcfdx_lbm.so`` for sm_100a.

Compiles every ``csrc/*.cu`` with nvcc (``-gencode arch=compute_100a,code=sm_100a``)
in parallel into ``_build/`` at the repository root and links the shared
library next to this file, where ``cfd_solvers_b200.bindings`` loads it.  The
C++ front end (``include/cfd/solvers/lbm/esoteric_pull_cuda.hpp``) and its two CLIs
(``cfd_solvers_b200/apps/cfd_bench.cpp``, ``cfd_solvers_b200/apps/cfd_solve.cpp``) link against the
same library.

Usage: ``python -m cfd_solvers_b200.build [--force] [--jobs N]``.
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
INCLUDE = ROOT / "include"
BUILD = ROOT / "_build"
LIB = PKG / "libcfdx_lbm.so"
APPS = PKG / "apps"
BENCH_BIN = PKG / "cfd-bench-cuda"
SOLVE_BIN = PKG / "cfd-solve-cuda"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden", "--expt-relaxed-constexpr",
              f"-I{INCLUDE}", f"-I{CSRC}"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found (CUDA toolkit required to build the sm_100a engine)")


def host_cxx() -> str:
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("g++ not found")


def _sources():
    return sorted(CSRC.glob("*.cu"))


def _headers():
    return sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h")))


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, verbose: bool) -> Path:
    obj = BUILD / (src.stem + ".o")
    if _stale(obj, [src] + _headers()):
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-ccbin", host_cxx(), "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return obj


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    """Builds libcfdx_lbm.so (and the cfd-bench-cuda and cfd-solve-cuda CLIs); returns the library path."""
    BUILD.mkdir(exist_ok=True)
    if force:
        for o in BUILD.glob("*.o"):
            o.unlink()
    srcs = _sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-ccbin", host_cxx(), "-Xcompiler", "-fPIC", "-o", str(LIB), *map(str, objs)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    headers = _headers() + list((INCLUDE / "cfd" / "solvers" / "lbm").glob("*.hpp"))
    for src, exe in ((APPS / "cfd_bench.cpp", BENCH_BIN), (APPS / "cfd_solve.cpp", SOLVE_BIN)):
        if src.exists() and (force or _stale(exe, [src, LIB] + headers)):
            cmd = [host_cxx(), "-std=c++20", "-O2", f"-I{INCLUDE}", str(src), "-o", str(exe),
                   f"-L{PKG}", "-lcfdx_lbm", "-Wl,-rpath,$ORIGIN"]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    return LIB


def main(argv=None) -> int:
    p = argparse.ArgumentParser(description=__doc__)
    p.add_argument("--force", action="store_true")
    p.add_argument("--jobs", type=int, default=None)
    p.add_argument("-v", "--verbose", action="store_true")
    a = p.parse_args(argv)
    print(build(a.force, a.jobs, a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
