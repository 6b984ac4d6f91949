"""Build recipe for the in-tree shared library fastapsp_b200/libfap_b200.so.

Every CUDA source is compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a); the host C++ (graph IO, METIS,
renumbering, fap::fapGraph) is compiled with the same nvcc driver.  The CUDA
runtime is linked statically so the library does not depend on which
libcudart another component of the process (e.g. torch) brings; METIS comes
from the CUDA toolkit's libmetis_static.a and its symbols stay hidden.

    python -m fastapsp_b200.build         # incremental
    python -m fastapsp_b200.build --force
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJDIR = os.path.join(HERE, "_objs")
LIB = os.path.join(HERE, "libfap_b200.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = shutil.which("nvcc") or os.path.join(CUDA_HOME, "bin", "nvcc")
CUDA_LIB = os.path.join(CUDA_HOME, "targets", "x86_64-linux", "lib")
METIS_A = os.path.join(CUDA_LIB, "libmetis_static.a")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
          "-I" + INCLUDE, "-I" + CSRC]
SOURCES = ["fap_device.cu", "fap_capi.cu", "fap_legacy.cu", "fap_noalloc.cu", "fap_host.cpp",
           "fap_serve.cpp"]
HEADERS = ["fap_common.cuh", "minplus_tile.cuh", "floyd.cuh", "sssp.cuh", "tma.cuh", "tma_tile.cuh",
           "fap_internal.h"]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(INCLUDE, "fap_b200.h"), os.path.join(INCLUDE, "fap_legacy_kernel.h"),
        os.path.join(INCLUDE, "fap_host.h"), os.path.join(INCLUDE, "fap_serve.h"),
        os.path.join(INCLUDE, "fap", "fap.h")]
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJDIR, os.path.splitext(src)[0] + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + hdrs + [__file__]):
            cmd = [NVCC] + ARCH + COMMON + ["-c", path, "-o", obj]
            if src.endswith(".cpp"):
                cmd = [NVCC, "-x", "cu"] + ARCH + COMMON + ["-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs + [
            METIS_A, "-Xlinker", "--exclude-libs,ALL", "-lm", "-lpthread"]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
