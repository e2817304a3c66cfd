"""Builds libbcgpu.so and the betc CLI in-tree (lib/), for sm_100a only.

    python centrality-gpu_b200/build.py          # or __graft_entry__.build()
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
SRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "lib"
INC = ROOT / "include"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOSTCXX = os.environ.get("BCGPU_HOSTCXX", "g++")  # the image's $CXX lacks the OpenMP spec
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp", "-I" + str(INC),
                   "-ccbin", HOSTCXX, "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-I" + str(INC), "-I/usr/local/cuda/include"]

CU_SOURCES = ["kernels_plain.cu", "kernels_batched.cu", "bcgpu.cu", "noalloc.cu"]
CXX_SOURCES = ["host_decomp.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    headers = list(SRC.glob("*.h")) + list(SRC.glob("*.cuh")) + list(INC.glob("*.h"))
    jobs = []
    objs = []
    for s in CU_SOURCES:
        o = OBJ / (s + ".o")
        objs.append(o)
        if force or _stale(o, [SRC / s] + headers):
            jobs.append([NVCC] + CU_FLAGS + ["-c", str(SRC / s), "-o", str(o)])
    for s in CXX_SOURCES:
        o = OBJ / (s + ".o")
        objs.append(o)
        if force or _stale(o, [SRC / s] + headers):
            jobs.append([HOSTCXX] + CXX_FLAGS + ["-c", str(SRC / s), "-o", str(o)])
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    lib = LIB / "libbcgpu.so"
    if force or _stale(lib, objs):
        _run([NVCC] + ARCH + ["-shared", "-ccbin", HOSTCXX, "-o", str(lib)] + [str(o) for o in objs] +
             ["-lgomp", "-Xlinker", "-soname=libbcgpu.so"])
    betc = LIB / "betc"
    main = SRC / "betc_main.cpp"
    if force or _stale(betc, [main, lib] + headers):
        _run([HOSTCXX] + CXX_FLAGS + [str(main), "-o", str(betc), "-L" + str(LIB), "-lbcgpu",
                                       "-Wl,-rpath,$ORIGIN"])
    return lib


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print("built", LIB / "libbcgpu.so", LIB / "betc")
