"""Builds libmikroptim_b200.so in-tree with nvcc for sm_100a (no GPU needed).

    python -m mikroptim_b200.build [--verbose]

Objects go to mikroptim_b200/_build/, the shared library next to this file, and the C++ host
layer (host/host.cpp) is linked against it as libmikroptim_b200_host.so. Every .cu file in
csrc/ is compiled with ``-gencode arch=compute_100a,code=sm_100a -O3 -lineinfo``; the CUDA
runtime is linked statically so the library does not depend on which libcudart the process
loaded first.
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmikroptim_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _flags(verbose: bool) -> list[str]:
    # host code in the .cu files is compiled without FP contraction, as the reference builds
    # its CPU code: the host-side sums and FD derivatives are bitwise equal to the reference's
    # only if the host compiler never fuses a multiply and an add (GCC does on aarch64)
    f = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-ffp-contract=off",
         "-I", os.path.join(ROOT, "include"), "-I", CSRC, "--expt-relaxed-constexpr"]
    if verbose:
        f += ["-Xptxas", "-v"]
    return f


def _compile(src: str, verbose: bool) -> tuple[str, str]:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        [os.path.join(ROOT, "include", "mikroptim_b200.h")]
    if (not verbose and os.path.exists(obj) and
            os.path.getmtime(obj) >= max(os.path.getmtime(p) for p in [src, *headers])):
        return obj, ""
    cmd = [nvcc(), *_flags(verbose), "-c", src, "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    return obj, res.stdout + res.stderr


HOST_DIR = os.path.join(HERE, "host")
HOST_LIB = os.path.join(HERE, "libmikroptim_b200_host.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build_host() -> str:
    """The C++ host layer (host/host.cpp, reference-shaped classes over the C ABI) as
    libmikroptim_b200_host.so next to the CUDA library, which it links (rpath $ORIGIN)."""
    srcs = [os.path.join(HOST_DIR, "host.cpp")]
    deps = srcs + glob.glob(os.path.join(HOST_DIR, "*.hpp")) + [LIB,
                                                              os.path.join(ROOT, "include",
                                                                           "mikroptim_b200.h")]
    if os.path.exists(HOST_LIB) and os.path.getmtime(HOST_LIB) >= max(
            os.path.getmtime(p) for p in deps):
        return HOST_LIB
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-std=c++20", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-Wall",
           "-Wextra", *srcs,
           "-I", os.path.join(ROOT, "include"), "-I", HOST_DIR,
           "-I", os.path.join(CUDA_HOME, "include"), "-o", HOST_LIB,
           "-L", HERE, "-lmikroptim_b200", "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart",
           "-Wl,-rpath,$ORIGIN", "-Wl,-rpath," + os.path.join(CUDA_HOME, "lib64")]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"host layer build failed:\n{res.stdout}\n{res.stderr}")
    return HOST_LIB


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose), sources))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                print(log)
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    build_host()
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true", help="print -Xptxas -v resource usage")
    a = ap.parse_args()
    print(build(a.verbose))
    sys.exit(0)
