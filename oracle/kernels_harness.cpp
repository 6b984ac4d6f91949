// Harness around the reference's own CPU kernels with predecessors
// (fap/kernel/floyd.h, fap/kernel/minplus.h), compiled unmodified from the
// reference sources.  TEST INFRASTRUCTURE ONLY: it pins the oracle's
// restatement of these kernels (oracle/fap_oracle.c) to the reference.
//
// Usage: fap_kernels_ref OP IN OUT
//   IN holds int32 sizes then the arrays, OUT receives the outputs, all raw
//   little-endian:
//   floyd_path     in: s, mat[s*s] f32, path[s*s] i32          out: mat, path
//   minplus_path   in: M N K, mat1[M*K], mat2[K*N], mat2_path[K*N]
//                  out: res[M*N], path[M*N]     (min_plus_path_CPU_advanced)
//   floyd_min_plus in: M N K, mat1, mat2, mat2_path, res[M*N], path[M*N]
//                  out: res, path               (floyd_min_plus_CPU)
//   path_A         in: row col, A[row*col], A_path, diag[col*col], diag_path
//                  out: A, A_path               (floyd_path_A_CPU)
//   path_B         in: row col, B[row*col], B_path, diag[row*row], diag_path
//                  out: B, B_path               (floyd_path_B_CPU)
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "fap/kernel/floyd.h"
#include "fap/kernel/minplus.h"

namespace {

FILE *g_in = nullptr;

template <typename T>
std::vector<T> take(size_t n) {
  std::vector<T> v(n);
  if (n && fread(v.data(), sizeof(T), n, g_in) != n) {
    fprintf(stderr, "short input\n");
    exit(2);
  }
  return v;
}

int32_t take1() { return take<int32_t>(1)[0]; }

template <typename T>
void put(FILE *f, const std::vector<T> &v) {
  if (!v.empty() && fwrite(v.data(), sizeof(T), v.size(), f) != v.size()) {
    fprintf(stderr, "short write\n");
    exit(3);
  }
}

}  // namespace

int main(int argc, char **argv) {
  if (argc != 4) {
    fprintf(stderr, "usage: %s OP IN OUT\n", argv[0]);
    return 2;
  }
  const std::string op = argv[1];
  g_in = fopen(argv[2], "rb");
  FILE *out = fopen(argv[3], "wb");
  if (!g_in || !out) {
    perror("open");
    return 2;
  }
  if (op == "floyd_path") {
    const int s = take1();
    auto mat = take<float>((size_t)s * s);
    auto path = take<int32_t>((size_t)s * s);
    fap::floyd_CPU_path(s, mat.data(), path.data());
    put(out, mat);
    put(out, path);
  } else if (op == "minplus_path" || op == "floyd_min_plus") {
    const int M = take1(), N = take1(), K = take1();
    auto a = take<float>((size_t)M * K);
    auto b = take<float>((size_t)K * N);
    auto bp = take<int32_t>((size_t)K * N);
    std::vector<float> res((size_t)M * N);
    std::vector<int32_t> path((size_t)M * N);
    if (op == "minplus_path") {
      fap::min_plus_path_CPU_advanced(a.data(), b.data(), bp.data(), res.data(), path.data(), M, N, K);
    } else {
      res = take<float>((size_t)M * N);
      path = take<int32_t>((size_t)M * N);
      fap::floyd_min_plus_CPU(a.data(), b.data(), bp.data(), res.data(), path.data(), M, N, K);
    }
    put(out, res);
    put(out, path);
  } else if (op == "path_A" || op == "path_B") {
    const int row = take1(), col = take1();
    auto x = take<float>((size_t)row * col);
    auto xp = take<int32_t>((size_t)row * col);
    const size_t d = op == "path_A" ? (size_t)col * col : (size_t)row * row;
    auto diag = take<float>(d);
    auto diag_path = take<int32_t>(d);
    if (op == "path_A")
      fap::floyd_path_A_CPU(x.data(), xp.data(), row, col, diag.data(), diag_path.data());
    else
      fap::floyd_path_B_CPU(x.data(), xp.data(), row, col, diag.data(), diag_path.data());
    put(out, x);
    put(out, xp);
  } else {
    fprintf(stderr, "unknown op %s\n", op.c_str());
    return 2;
  }
  fclose(g_in);
  fclose(out);
  return 0;
}
