"""The drop-in claims for C++ callers, checked with the reference's own
sources where they lie in the reference checkout (never copied):
app/singleNodeExample.cpp compiles unchanged against include/fap/fap.h and
links against libfap_b200.so; and the reference's fap/fap.cpp built with
-DWITH_CUDA links against libfap_b200.so in place of its CUDA kernels.  Only
compiled and linked here: running either solves on a GPU.  Skipped where
the reference checkout is absent."""
import os
import shutil
import subprocess
import tempfile

import pytest

from conftest import ROOT
from fastapsp_b200 import _lib as L

REFERENCE = os.environ.get("FAP_REFERENCE_DIR", "/root/reference")
EXAMPLE = os.path.join(REFERENCE, "app", "singleNodeExample.cpp")


@pytest.mark.skipif(not os.path.exists(EXAMPLE) or shutil.which("g++") is None,
                    reason="reference example or g++ not available")
def test_reference_example_builds_against_the_drop_in():
    libdir = os.path.dirname(L.LIB_PATH)
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "single_node_example")
        r = subprocess.run(["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"), EXAMPLE,
                            "-o", exe, "-L" + libdir, "-lfap_b200", "-Wl,-rpath," + libdir],
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-3000:]
        assert os.path.getsize(exe) > 0


@pytest.mark.skipif(not os.path.exists(EXAMPLE) or shutil.which("g++") is None,
                    reason="reference example or g++ not available")
def test_reference_host_code_links_against_the_legacy_kernel_abi():
    """The reference's own fap/fap.cpp built with -DWITH_CUDA (its GPU
    build) links against libfap_b200.so in place of its CUDA kernels: every
    kernel entry point it calls is exported with the same C++ signature.
    METIS comes from the CUDA toolkit's static library, as for the oracle."""
    libdir = os.path.dirname(L.LIB_PATH)
    metis = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "targets", "x86_64-linux", "lib",
                         "libmetis_static.a")
    if not os.path.exists(metis):
        pytest.skip("no METIS static library")
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "single_node_example_cuda")
        r = subprocess.run(["g++", "-std=c++17", "-O1", "-fopenmp", "-w", "-DWITH_CUDA",
                            "-I" + os.path.join(ROOT, "oracle"), "-I" + REFERENCE,
                            os.path.join(REFERENCE, "fap", "fap.cpp"), EXAMPLE, "-o", exe,
                            "-L" + libdir, "-lfap_b200", "-Wl,-rpath," + libdir, metis, "-lm"],
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-3000:]
