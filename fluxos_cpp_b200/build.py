"""Build libfluxos_gpu.so (sm_100a) and the fluxos_gpu program in-tree.

    python -m fluxos_cpp_b200.build      (or fluxos_cpp_b200.build.build())

CUDA sources are compiled by nvcc for sm_100a only, with --fmad=false so no
multiply-add is contracted (the FP64 path reproduces the CPU reference's
roundings); the host C++ sources by g++. The CUDA runtime is linked
statically, so the library needs only the driver at run time.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
INC = os.path.join(ROOT, "include")
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "lib")
SO = os.path.join(LIB, "libfluxos_gpu.so")
EXE = os.path.join(LIB, "fluxos_gpu")

CU_SOURCES = ["fx_hydro.cu", "fx_ade.cu", "fx_capi.cu", "fx_batch.cu", "fx_noalloc.cu", "fx_results.cu"]
CPP_SOURCES = ["fluxos_io.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + INC]


def _cuda_home() -> str:
    for c in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if c and os.path.exists(os.path.join(c, "bin", "nvcc")):
            return c
    nv = shutil.which("nvcc")
    if nv:
        return os.path.dirname(os.path.dirname(nv))
    raise RuntimeError("nvcc not found: set CUDA_HOME")


def _cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _stale(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build(verbose: bool = False) -> str:
    cuda = _cuda_home()
    nvcc = os.path.join(cuda, "bin", "nvcc")
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(INC, "fluxos_gpu.h"))
    objs = []
    for f in CU_SOURCES:
        src, obj = os.path.join(CSRC, f), os.path.join(OBJ, f + ".o")
        if _stale(obj, [src] + headers):
            cmd = [nvcc] + ARCH + NVCC_FLAGS + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
        objs.append(obj)
    for f in CPP_SOURCES:
        src, obj = os.path.join(HOST, f), os.path.join(OBJ, f + ".o")
        if _stale(obj, [src] + headers):
            cmd = [_cxx(), "-std=c++17", "-O2", "-fPIC", "-I" + INC, "-I" + CSRC,
                   "-I" + os.path.join(cuda, "include"), "-c", src, "-o", obj]
            _run(cmd)
        objs.append(obj)
    if _stale(SO, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", SO] + objs)
    main_src = os.path.join(HOST, "fluxos_gpu_main.cpp")
    if _stale(EXE, [main_src, SO]):
        _run([_cxx(), "-std=c++17", "-O2", "-I" + INC, main_src, "-o", EXE, "-L" + LIB,
              "-lfluxos_gpu", "-Wl,-rpath,$ORIGIN"])
    return SO


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
