"""Builds libbcgpu.so and the betc CLI in-tree (lib/), for sm_100a only.

    python centrality-gpu_b200/build.py          # or __graft_entry__.build()
    python centrality-gpu_b200/build.py --variant phase -DBCGPU_PHASE_TIMERS
        # an instrumented copy in lib_phase/ (objects in _build_phase/); load it
        # with BCGPU_LIB_DIR=<package>/lib_phase. The default build is unaffected.
    python centrality-gpu_b200/build.py --variant ht -DBCGPU_HOST_TIMERS
        # the same for the host side of plan builds: each stage's wall time
        # ("[host] route", "[host] uploads", ...) printed to stderr.
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

CU_SOURCES = ["kernels_plain.cu", "kernels_batched.cu", "kernels_tile.cu", "bcgpu.cu", "noalloc.cu", "decomp_steps.cu"]
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


def build(verbose: bool = False, force: bool = False, variant: str = "", defines=()) -> Path:
    obj_dir = OBJ if not variant else PKG / f"_build_{variant}"
    lib_dir = LIB if not variant else PKG / f"lib_{variant}"
    obj_dir.mkdir(exist_ok=True)
    lib_dir.mkdir(exist_ok=True)
    extra = list(defines)
    headers = list(SRC.glob("*.h")) + list(SRC.glob("*.cuh")) + list(INC.glob("*.h"))
    jobs = []
    objs = []
    for s in CU_SOURCES:
        o = obj_dir / (s + ".o")
        objs.append(o)
        if force or _stale(o, [SRC / s] + headers):
            jobs.append([NVCC] + CU_FLAGS + extra + ["-c", str(SRC / s), "-o", str(o)])
    for s in CXX_SOURCES:
        o = obj_dir / (s + ".o")
        objs.append(o)
        if force or _stale(o, [SRC / s] + headers):
            jobs.append([HOSTCXX] + CXX_FLAGS + extra + ["-c", str(SRC / s), "-o", str(o)])
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    lib = lib_dir / "libbcgpu.so"
    if force or _stale(lib, objs):
        _run([NVCC] + ARCH + ["-shared", "-ccbin", HOSTCXX, "-o", str(lib)] + [str(o) for o in objs] +
             ["-lgomp", "-Xlinker", "-soname=libbcgpu.so"])
    betc = lib_dir / "betc"
    main = SRC / "betc_main.cpp"
    if force or _stale(betc, [main, lib] + headers):
        _run([HOSTCXX] + CXX_FLAGS + [str(main), "-o", str(betc), "-L" + str(LIB), "-lbcgpu",
                                       "-Wl,-rpath,$ORIGIN"])
    return lib


if __name__ == "__main__":
    argv = sys.argv[1:]
    var = argv[argv.index("--variant") + 1] if "--variant" in argv else ""
    lib_path = build(verbose="-v" in argv, force="-f" in argv, variant=var,
                     defines=[a for a in argv if a.startswith("-D")])
    print("built", lib_path, lib_path.parent / "betc")
