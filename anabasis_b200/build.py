"""Builds libanb.so (CUDA sm_100a + host front end) and the anabasis_simple executable in-tree.

Usage: python -m anabasis_b200.build [--force]

Objects go to anabasis_b200/_build/, products to anabasis_b200/_lib/.  Host C++ is compiled
without FMA contraction (-ffp-contract=off) so that mesh geometry reproduces the reference's
host arithmetic bit for bit.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "_lib"
INCLUDE = PKG.parent / "include"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

HOST_SOURCES = ["host_mesh.cpp", "host_case.cpp", "host_output.cpp", "host_api.cpp", "layout.cpp", "amg_setup.cpp"]
MMS_APPS = {1: "anabasis_poisson_mms", 2: "anabasis_poisson_mms_neumann", 3: "anabasis_poisson_mms_mixed",
            4: "anabasis_scalar_mms"}
CUDA_SOURCES = ["kernels_fv.cu", "kernels_krylov.cu", "kernels_scalar.cu", "kernels_adjoint.cu", "anb_api.cu", "adjoint_api.cu", "nalloc.cu",
                "setup_gpu.cu"]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off", "-Wall", "-Wno-unused-function"]
NVCCFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp", "--expt-relaxed-constexpr"]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} ... {cmd[-1]}")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.hpp")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles the library and the host program; returns the path of libanb.so."""
    BUILD.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    hdrs = _headers()
    objs: list[Path] = []
    jobs: list[list[str]] = []
    for src in HOST_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".o")
        if force or _stale(o, [s] + hdrs):
            if verbose:
                print("g++", src)
            jobs.append(["g++", *CXXFLAGS, f"-I{CUDA_HOME}/include", "-c", str(s), "-o", str(o)])
        objs.append(o)
    for src in CUDA_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".cu.o")
        if force or _stale(o, [s] + hdrs):
            if verbose:
                print("nvcc", src)
            jobs.append([NVCC, *NVCCFLAGS, "-c", str(s), "-o", str(o)])
        objs.append(o)
    # translation units are independent: compile them concurrently
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_run, j) for j in jobs]:
            f.result()
    lib = LIB / "libanb.so"
    if force or _stale(lib, objs):
        _run([NVCC, *ARCH, "-shared", "-o", str(lib), *map(str, objs), "-Xcompiler", "-fopenmp", "-lgomp"])
    app_src = CSRC / "app_main.cpp"
    app_obj = BUILD / "app_main.o"
    if force or _stale(app_obj, [app_src] + hdrs):
        _run(["g++", *CXXFLAGS, f"-I{CUDA_HOME}/include", "-c", str(app_src), "-o", str(app_obj)])
    app = LIB / "anabasis_simple"
    if force or _stale(app, [app_obj, lib]):
        _run(["g++", "-o", str(app), str(app_obj), f"-L{LIB}", "-lanb", f"-L{CUDA_HOME}/lib64", "-lcudart",
              "-Wl,-rpath,$ORIGIN", f"-Wl,-rpath,{CUDA_HOME}/lib64", "-fopenmp"])
    # the reference's manufactured-solution programs, one executable each from app_mms.cpp
    mms_src = CSRC / "app_mms.cpp"
    for idx, name in MMS_APPS.items():
        exe = LIB / name
        if force or _stale(exe, [mms_src, lib] + hdrs):
            _run(["g++", *CXXFLAGS, f"-DANB_MMS_APP={idx}", f"-I{CUDA_HOME}/include", "-o", str(exe), str(mms_src),
                  f"-L{LIB}", "-lanb", f"-L{CUDA_HOME}/lib64", "-lcudart", "-Wl,-rpath,$ORIGIN",
                  f"-Wl,-rpath,{CUDA_HOME}/lib64"])
    return lib


def clean() -> None:
    shutil.rmtree(BUILD, ignore_errors=True)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB / "libanb.so")
