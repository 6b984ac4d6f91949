"""The headers are plain C: a C99 program (gcc -std=c99 -pedantic -Werror)
includes include/fap_b200.h, fap_host.h and fap_serve.h, links
libfap_b200.so and drives the host side of fapGraph through the C ABI
(no GPU: CSR in, given partition, preCondition, binary save and load, error
codes).  This is the binding a C or cgo caller writes."""
import os
import shutil
import subprocess
import tempfile

import pytest

from conftest import ROOT
from fastapsp_b200 import _lib as L

PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "fap_b200.h"
#include "fap_host.h"
#include "fap_serve.h"

#define CHECK(x) do { int rc_ = (x); if (rc_ != FAP_OK) { \
  printf("FAIL %s -> %d: %s\n", #x, rc_, fap_host_last_error()); return 1; } } while (0)

int main(int argc, char **argv) {
  /* 4 x 4 grid, both directions of every edge, unit weights */
  int32_t ro[17], col[48];
  float w[48];
  int32_t n = 16, e = 0, v, r, c;
  for (v = 0; v < n; v++) {
    r = v / 4; c = v % 4; ro[v] = e;
    if (c > 0) { col[e] = v - 1; w[e++] = 1.0f; }
    if (c < 3) { col[e] = v + 1; w[e++] = 1.0f; }
    if (r > 0) { col[e] = v - 4; w[e++] = 1.0f; }
    if (r < 3) { col[e] = v + 4; w[e++] = 1.0f; }
  }
  ro[n] = e;
  fap_host_graph *g = NULL, *h = NULL;
  int32_t gid[16], vn[3], vo[3], bn[3], vn2[3], vo2[3], bn2[3], map[16], map2[16];
  int64_t sz[4];
  int d = -1, wt = -1;
  if (argc != 2) return 2;
  CHECK(fap_host_from_csr(n, e, ro, col, w, 2, 0, &g));
  for (v = 0; v < n; v++) gid[v] = (v % 4) < 2 ? 1 : 2;   /* columns 0-1 | 2-3 */
  CHECK(fap_host_set_partition(g, gid));
  CHECK(fap_host_precondition(g));
  CHECK(fap_host_parts(g, vn, vo, bn));
  if (vn[1] != 8 || vn[2] != 8 || bn[1] != 4 || bn[2] != 4 || vo[2] != 8) {
    printf("FAIL parts %d %d %d %d %d\n", vn[1], vn[2], bn[1], bn[2], vo[2]);
    return 1;
  }
  CHECK(fap_host_mapping(g, map));
  CHECK(fap_host_save(g, argv[1]));
  CHECK(fap_host_load(argv[1], &h));
  CHECK(fap_host_flags(h, &d, &wt));
  CHECK(fap_host_sizes(h, sz));
  CHECK(fap_host_precondition(h));
  CHECK(fap_host_parts(h, vn2, vo2, bn2));
  CHECK(fap_host_mapping(h, map2));
  if (d != 0 || sz[0] != 16 || sz[2] != 2 || sz[3] != 48 || memcmp(map, map2, sizeof(map)) != 0 ||
      memcmp(bn, bn2, sizeof(bn)) != 0) {
    printf("FAIL round trip\n");
    return 1;
  }
  CHECK(fap_host_destroy(h));
  h = NULL;
  /* errors come back as codes with a message, never as an abort */
  if (fap_host_load("no/such/file.fapb", &h) != FAP_ERR_IO || !strlen(fap_host_last_error())) {
    printf("FAIL missing file\n");
    return 1;
  }
  for (v = 0; v < n; v++) gid[v] = 3;
  if (fap_host_set_partition(g, gid) != FAP_ERR_PARTITION) {
    printf("FAIL bad partition\n");
    return 1;
  }
  CHECK(fap_host_destroy(g));
  printf("ok %d\n", fap_version());
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not installed")
def test_c99_program_drives_the_host_api():
    with tempfile.TemporaryDirectory() as tmp:
        src = os.path.join(tmp, "prog.c")
        exe = os.path.join(tmp, "prog")
        with open(src, "w") as f:
            f.write(PROGRAM)
        libdir = os.path.dirname(L.LIB_PATH)
        cc = subprocess.run(["gcc", "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror",
                             "-I" + os.path.join(ROOT, "include"), src, "-o", exe, "-L" + libdir,
                             "-lfap_b200", "-Wl,-rpath," + libdir], capture_output=True, text=True)
        assert cc.returncode == 0, cc.stderr
        run = subprocess.run([exe, os.path.join(tmp, "g.fapb")], capture_output=True, text=True,
                             timeout=120)
        assert run.returncode == 0 and run.stdout.startswith("ok "), run.stdout + run.stderr
