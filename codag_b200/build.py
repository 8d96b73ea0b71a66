"""Build recipe for the in-tree native library and command-line tools.

Produces, next to the sources:
  codag_b200/libcodag_b200.so   CUDA decoders (sm_100a) and the C ABI of include/codag.h
  codag_b200/libcodag_fmt.so    host-only format producers and generators (include/codag_format.h)
  build/exe/src/<dir>/<tool>.cu.exe   CLIs with CODAG's command lines (rlev1, rlev2, zlib,
                                      util/base_deflate)

Run ``python -m codag_b200.build`` (or ``__graft_entry__.build()``).  nvcc cross-compiles
for sm_100a without a GPU.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
OBJ = REPO / "_build"
LIB = PKG / "libcodag_b200.so"
FMT_LIB = PKG / "libcodag_fmt.so"
EXE = REPO / "build" / "exe" / "src"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++20", "-Xcompiler", "-fPIC,-fopenmp", "-Xptxas", "-warn-spills"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-Wno-unused-function"]

HOST_SOURCES = sorted((CSRC / "host").glob("*.cpp"))
CUDA_SOURCES = [CSRC / "kernels" / name for name in ("codag_capi.cu", "encode_capi.cu", "transposed_capi.cu")]
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
HEADERS = (sorted(CSRC.rglob("*.cuh")) + sorted(CSRC.rglob("*.hpp")) + sorted(CSRC.glob("*.h")) +
           [REPO / "include" / "codag.h", REPO / "include" / "codag_format.h"])
CLI_SOURCES = {name: CSRC / "cli" / f"{name}_main.cpp" for name in ("rlev1", "rlev2", "zlib", "base_deflate")}
# where CODAG's Makefile puts each tool (build/exe/src/<dir>/<name>.cu.exe)
CLI_DIRS = {"rlev1": "rlev1", "rlev2": "rlev2", "zlib": "zlib", "base_deflate": "util"}


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    res = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"build step failed ({res.returncode}): {' '.join(map(str, cmd))}\n{res.stdout}\n{res.stderr}")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the libraries (and CLIs) if any source is newer than the outputs."""
    OBJ.mkdir(exist_ok=True)
    jobs = []
    host_objs, cuda_objs = [], []
    with cf.ThreadPoolExecutor(max_workers=max(2, os.cpu_count() or 2)) as pool:
        for src in HOST_SOURCES:
            obj = OBJ / (src.stem + ".host.o")
            host_objs.append(obj)
            if force or _stale(obj, [src] + HEADERS):
                jobs.append(pool.submit(_run, ["g++", *CXX_FLAGS, "-c", src, "-o", obj], verbose))
        for src in CUDA_SOURCES:
            obj = OBJ / (src.stem + ".cu.o")
            cuda_objs.append(obj)
            if force or _stale(obj, [src] + HEADERS):
                jobs.append(pool.submit(_run, ["nvcc", *NVCC_FLAGS, "-c", src, "-o", obj], verbose))
        for j in jobs:
            j.result()
    if force or _stale(FMT_LIB, host_objs):
        _run(["g++", "-shared", "-o", FMT_LIB, *host_objs, "-lz", "-fopenmp"], verbose)
    if force or _stale(LIB, cuda_objs):
        _run(["nvcc", *ARCH, "-shared", "-o", LIB, *cuda_objs], verbose)
    for name, src in CLI_SOURCES.items():
        if not src.exists():
            continue
        exe = EXE / CLI_DIRS[name] / f"{name}.cu.exe"
        exe.parent.mkdir(parents=True, exist_ok=True)
        if force or _stale(exe, [src, LIB, FMT_LIB, CSRC / "cli" / "cli_common.hpp"] + HEADERS):
            _run(["g++", "-O2", "-std=c++17", "-Wall", src, "-I", REPO / "include", "-I", CUDA / "include", "-o", exe,
                  "-L", PKG, "-lcodag_b200", "-lcodag_fmt", "-L", CUDA / "lib64", "-lcudart",
                  "-Wl,-rpath,$ORIGIN/../../../../codag_b200", f"-Wl,-rpath,{CUDA / 'lib64'}"], verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
