"""The drop-in claims for C++ callers, checked with the reference's own
sources where they lie in the reference checkout (never copied):
app/singleNodeExample.cpp compiles unchanged against include/fap/fap.h and
links against libfap_b200.so; and the reference's fap/fap.cpp built with
-DWITH_CUDA links against libfap_b200.so in place of its CUDA kernels.  Only
compiled and linked here: running either solves on a GPU.  Skipped where
the reference checkout is absent.  A third test needs no checkout: every
public member of the reference's fapGraph, with its type, at compile time."""
import os
import shutil
import subprocess
import tempfile

import pytest

from conftest import ROOT
from fastapsp_b200 import _lib as L

# $FAP_REFERENCE_DIR, else a checkout named "reference" beside this repository
REFERENCE = os.environ.get("FAP_REFERENCE_DIR") or os.path.join(os.path.dirname(ROOT), "reference")
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


API_PROGRAM = r"""
#include <string>
#include <type_traits>
#include <vector>
#include "fap/fap.h"
using fap::fapGraph;
// Every public member of the reference's fap::fapGraph (fap/fap.h:70-124),
// with the reference's exact types.
static_assert(std::is_constructible<fapGraph, std::string, bool, bool, int32_t>::value, "file ctor");
static_assert(std::is_constructible<fapGraph, int32_t, int64_t, std::vector<int32_t>, std::vector<int32_t>,
                                    std::vector<float>, int32_t>::value, "metadata ctor");
void (fapGraph::*m01)() = &fapGraph::preCondition;
bool (fapGraph::*m02)() = &fapGraph::isSplit;
std::vector<int> (fapGraph::*m03)() = &fapGraph::getGraphId;
int32_t (fapGraph::*m04)(bool) = &fapGraph::solve;
int32_t (fapGraph::*m05)(int32_t, bool) = &fapGraph::solveSubGraph;
std::vector<int32_t> (fapGraph::*m06)() = &fapGraph::getMapping;
std::vector<float> (fapGraph::*m07)() = &fapGraph::getAllDistance;
std::vector<int32_t> (fapGraph::*m08)() = &fapGraph::getAllPath;
int32_t (fapGraph::*m09)() = &fapGraph::getCurrentSubGraphId;
std::vector<int32_t> (fapGraph::*m10)(int32_t) = &fapGraph::getSubGraphIndex;
std::vector<float> (fapGraph::*m11)(int32_t) = &fapGraph::getSubGraphDistance;
std::vector<int32_t> (fapGraph::*m12)(int32_t) = &fapGraph::getSubGraphPath;
std::vector<float> (fapGraph::*m13)(int32_t) = &fapGraph::getDistanceFromOnePoint;
std::vector<int32_t> (fapGraph::*m14)(int32_t) = &fapGraph::getPathFromOnePoint;
float (fapGraph::*m15)() = &fapGraph::getDistanceP2P;
std::vector<int32_t> (fapGraph::*m16)() = &fapGraph::getPathP2P;
bool (fapGraph::*m17)(float *, int *, int *, int, int, int *, int *, int *, float *, int *) =
    &fapGraph::check_result;
int32_t fapGraph::*d1 = &fapGraph::num_vertexs;
int32_t fapGraph::*d2 = &fapGraph::num_edges;
std::vector<int32_t> fapGraph::*d3 = &fapGraph::adj_size;
std::vector<int32_t> fapGraph::*d4 = &fapGraph::row_offset;
std::vector<int32_t> fapGraph::*d5 = &fapGraph::col_val;
std::vector<float> fapGraph::*d6 = &fapGraph::weight;
bool fapGraph::*d7 = &fapGraph::directed;
bool fapGraph::*d8 = &fapGraph::weighted;
// a derived class sees the reference's protected state
struct Derived : fapGraph {
  using fapGraph::fapGraph;
  int probe() { return K + current_subgraph_id + (int)C_BlockVer_num.size() + (int)isBoundry.size(); }
};
int main() { return 0; }
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_fapgraph_has_every_public_member_of_the_reference():
    """Compile-time check that include/fap/fap.h offers each public member of
    the reference's fapGraph with the same type (and its protected state to
    derived classes), so reference callers compile unchanged."""
    with tempfile.TemporaryDirectory() as tmp:
        src = os.path.join(tmp, "api.cpp")
        with open(src, "w") as f:
            f.write(API_PROGRAM)
        r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I" + os.path.join(ROOT, "include"), src],
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-3000:]
