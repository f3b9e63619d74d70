"""Build recipe for the native library and the CLI driver.

Compiles the sm_100a kernels and the C++ host layer in-tree:
    lpa_b200/liblpa_b200.so   -- the C-ABI library (include/lpa_capi.h)
    lpa_b200/bin/method       -- the ./method driver (reference CLI)
Run as ``python -m lpa_b200.build`` or through ``__graft_entry__.build()``.
Objects go to lpa_b200/_build/ and are rebuilt only when a source or header
is newer than the object.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
INC = ROOT / "include"
OUT = PKG / "_build"
LIB = PKG / "liblpa_b200.so"
BIN = PKG / "bin" / "method"

NVCC = os.environ.get("LPA_NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-ccbin", CXX, "-Xcompiler", "-fPIC",
                  "-Xcompiler", "-Wall", "--expt-relaxed-constexpr", f"-I{INC}", f"-I{PKG / 'csrc'}"]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-Wextra", "-pthread", f"-I{INC}", f"-I{PKG / 'cpp'}"]

CU_SOURCES = sorted((PKG / "csrc").glob("*.cu"))
CPP_SOURCES = sorted(p for p in (PKG / "cpp").glob("*.cpp") if p.name != "method.cpp")
HEADERS = sorted(list(INC.rglob("*.h")) + list((PKG / "csrc").glob("*.cuh")) +
                 list((PKG / "csrc").glob("*.h")) + list((PKG / "cpp").glob("*.h")))


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in HEADERS)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed ({r.returncode}):\n{' '.join(cmd)}\n{r.stdout}")
    if r.stdout.strip():
        sys.stderr.write(r.stdout)


def build(verbose: bool = False) -> Path:
    OUT.mkdir(exist_ok=True)
    jobs = []
    objs = []
    for src in CU_SOURCES:
        obj = OUT / (src.stem + ".cu.o")
        objs.append(obj)
        if _stale(obj, src):
            jobs.append([NVCC, *NVFLAGS, "-c", str(src), "-o", str(obj)])
    for src in CPP_SOURCES:
        obj = OUT / (src.stem + ".o")
        objs.append(obj)
        if _stale(obj, src):
            jobs.append([CXX, *CXXFLAGS, "-c", str(src), "-o", str(obj)])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        for f in [ex.submit(_run, j) for j in jobs]:
            f.result()
    if jobs or not LIB.exists():
        tmp = LIB.with_suffix(".so.tmp")
        _run([NVCC, *ARCH, "-shared", "-ccbin", CXX, "-cudart", "static", "-o", str(tmp),
              *map(str, objs), "-lpthread"])
        os.replace(tmp, LIB)
    # CLI driver
    method_src = PKG / "cpp" / "method.cpp"
    if method_src.exists() and (not BIN.exists() or BIN.stat().st_mtime < max(
            LIB.stat().st_mtime, method_src.stat().st_mtime, *(h.stat().st_mtime for h in HEADERS))):
        BIN.parent.mkdir(exist_ok=True)
        _run([CXX, *CXXFLAGS, str(method_src), "-o", str(BIN), f"-L{PKG}", "-llpa_b200",
              "-Wl,-rpath,$ORIGIN/.."])
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(verbose=True)
