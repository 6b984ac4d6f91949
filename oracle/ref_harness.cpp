// Oracle harness around the reference's own CPU implementation of the
// per-subgraph solve path.  TEST INFRASTRUCTURE ONLY: it is the checker and
// the timed CPU baseline, never part of the product.
//
// The reference's fap/fap.cpp is compiled unmodified, as one translation unit
// (its headers define non-inline functions and fap/fap.h has no include
// guard).  Its private members are opened by redefining the access keywords
// after every standard header has been included, so that the harness can call
// fapGraph::run(dist, path, part) exactly the way fapGraph::solveSubGraph does
// (fap/fap.cpp:197-207).  solve()/solveSubGraph() themselves are not called:
// they fall off the end of a non-void function (fap/fap.cpp:194,207), which
// g++ 13 turns into a trap.
//
// Build: oracle/Makefile (reads the reference sources where they lie).
//
// Usage:
//   fap_ref --dir D -f NAME -k K -direct 0|1 -weight 0|1
//           [--parts all|1,5,9] [--meta FILE] [--dist FILE] [--path FILE]
//           [--rowsum FILE] [--quiet]
//   The graph is read from D/graph/<kind>/NAME.mtx (the reference resolves the
//   path relative to the working directory, fap/utils/readMatFile.h:43-51).
//   --meta  writes the CSR, partition and renumbering (binary, see dump_meta).
//   --dist  writes each solved part's s x n float block, in part order.
//   --path  writes each solved part's s x n int32 predecessor block (the
//           reference's run() always computes it), in part order.
//   --rowsum writes, per solved part and row, the uint64 checksum
//           sum_j uint32(int32(d[r][j])) * (2j + 1) mod 2^64 of the row's
//           distances cast to int32 (exact for integer weights while the
//           finite distances stay below 2^24; the sentinel 1e8 becomes
//           100000000): s values per part, in part order.
//   One JSON line per solved part goes to stdout with its wall time.
//   FAP_PARTITION_FILE=<file of n int32 part ids, 0-based> replaces the METIS
//   call by that partition (link-time wrap of METIS_PartGraphKway), so the
//   oracle and the product can be pinned to one shared partition.
#include <bits/stdc++.h>
#include <omp.h>
#include <sys/time.h>
#include <unistd.h>
#include "metis.h"

#define private public
#define protected public
#include "fap/fap.cpp"
#undef private
#undef protected

extern "C" int __real_METIS_PartGraphKway(idx_t *, idx_t *, idx_t *, idx_t *,
                                          idx_t *, idx_t *, idx_t *, idx_t *,
                                          real_t *, real_t *, idx_t *, idx_t *,
                                          idx_t *);

extern "C" int __wrap_METIS_PartGraphKway(
    idx_t *nvtxs, idx_t *ncon, idx_t *xadj, idx_t *adjncy, idx_t *vwgt,
    idx_t *vsize, idx_t *adjwgt, idx_t *nparts, real_t *tpwgts, real_t *ubvec,
    idx_t *options, idx_t *edgecut, idx_t *part) {
  const char *f = getenv("FAP_PARTITION_FILE");
  if (f == nullptr || f[0] == 0) {
    return __real_METIS_PartGraphKway(nvtxs, ncon, xadj, adjncy, vwgt, vsize,
                                      adjwgt, nparts, tpwgts, ubvec, options,
                                      edgecut, part);
  }
  FILE *fp = fopen(f, "rb");
  if (!fp) return METIS_ERROR_INPUT;
  std::vector<int32_t> p(*nvtxs);
  size_t got = fread(p.data(), sizeof(int32_t), p.size(), fp);
  fclose(fp);
  if (got != p.size()) return METIS_ERROR_INPUT;
  for (idx_t i = 0; i < *nvtxs; i++) part[i] = p[i];
  *edgecut = 0;
  return METIS_OK;
}

namespace {

double now_s() {
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return tv.tv_sec + tv.tv_usec * 1e-6;
}

template <typename T>
void put(FILE *f, const T *p, size_t n) {
  if (n && fwrite(p, sizeof(T), n, f) != n) {
    fprintf(stderr, "short write\n");
    exit(3);
  }
}

// Binary layout: int32 n, int32 m, int32 K, then row_offset[n+1],
// col_val[m], weight[m] (float32), graph_id[n] (1-based), st2ed[n],
// ed2st[n], C_BlockVer_num[K+1], C_BlockVer_offset[K+1], C_BlockBdy_num[K+1].
void dump_meta(fap::fapGraph &g, const char *path) {
  FILE *f = fopen(path, "wb");
  if (!f) { perror(path); exit(2); }
  int32_t hdr[3] = {g.num_vertexs, g.num_edges, g.K};
  put(f, hdr, 3);
  put(f, g.row_offset.data(), g.row_offset.size());
  put(f, g.col_val.data(), g.col_val.size());
  put(f, g.weight.data(), g.weight.size());
  put(f, g.graph_id.data(), g.graph_id.size());
  put(f, g.st2ed.data(), g.st2ed.size());
  put(f, g.ed2st.data(), g.ed2st.size());
  put(f, g.C_BlockVer_num.data(), g.C_BlockVer_num.size());
  put(f, g.C_BlockVer_offset.data(), g.C_BlockVer_offset.size());
  put(f, g.C_BlockBdy_num.data(), g.C_BlockBdy_num.size());
  fclose(f);
}

// Per-row checksums of an s x n block, int32 view of the float distances.
void put_rowsums(FILE *f, const float *d, int64_t s, int64_t n) {
  std::vector<uint64_t> sums((size_t)s);
  for (int64_t r = 0; r < s; r++) {
    uint64_t acc = 0;
    const float *row = d + r * n;
    for (int64_t j = 0; j < n; j++) {
      const uint32_t v = (uint32_t)(int32_t)(int64_t)row[j];
      acc += (uint64_t)v * (uint64_t)(2 * j + 1);
    }
    sums[(size_t)r] = acc;
  }
  put(f, sums.data(), sums.size());
}

}  // namespace

int main(int argc, char **argv) {
  std::string dir = ".", name, parts = "all", meta, distf, pathf, sumf;
  int K = 0, directed = 0, weighted = 0;
  bool quiet = false;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    auto nxt = [&]() -> std::string {
      if (i + 1 >= argc) { fprintf(stderr, "missing value for %s\n", a.c_str()); exit(2); }
      return argv[++i];
    };
    if (a == "--dir") dir = nxt();
    else if (a == "-f") name = nxt();
    else if (a == "-k") K = std::stoi(nxt());
    else if (a == "-direct") directed = std::stoi(nxt());
    else if (a == "-weight") weighted = std::stoi(nxt());
    else if (a == "--parts") parts = nxt();
    else if (a == "--meta") meta = nxt();
    else if (a == "--dist") distf = nxt();
    else if (a == "--path") pathf = nxt();
    else if (a == "--rowsum") sumf = nxt();
    else if (a == "--quiet") quiet = true;
    else { fprintf(stderr, "unknown arg %s\n", a.c_str()); return 2; }
  }
  if (name.empty() || K <= 0) {
    fprintf(stderr, "need -f NAME and -k K\n");
    return 2;
  }
  if (!meta.empty() && meta[0] != '/') meta = std::string(getcwd(nullptr, 0)) + "/" + meta;
  if (!distf.empty() && distf[0] != '/') distf = std::string(getcwd(nullptr, 0)) + "/" + distf;
  if (!pathf.empty() && pathf[0] != '/') pathf = std::string(getcwd(nullptr, 0)) + "/" + pathf;
  if (!sumf.empty() && sumf[0] != '/') sumf = std::string(getcwd(nullptr, 0)) + "/" + sumf;
  if (chdir(dir.c_str()) != 0) { perror(dir.c_str()); return 2; }

  // The reference prints a debug line on every min-plus call
  // (fap/kernel/minplus.h:81,86); keep stdout for the JSON lines.
  std::ofstream devnull("/dev/null");
  std::streambuf *saved = std::cout.rdbuf(devnull.rdbuf());

  double t0 = now_s();
  fap::fapGraph g(name, directed != 0, weighted != 0, K);
  g.preCondition();
  double t1 = now_s();
  if (!quiet)
    printf("{\"event\": \"prep\", \"n\": %d, \"m\": %d, \"K\": %d, \"seconds\": %.6f, \"threads\": %d}\n",
           g.num_vertexs, g.num_edges, K, t1 - t0, omp_get_max_threads());
  if (!meta.empty()) dump_meta(g, meta.c_str());

  std::vector<int> todo;
  if (parts == "all") {
    for (int p = 1; p <= K; p++) todo.push_back(p);
  } else if (parts != "none") {
    std::stringstream ss(parts);
    std::string tok;
    while (std::getline(ss, tok, ',')) todo.push_back(std::stoi(tok));
  }
  FILE *df = nullptr, *pf = nullptr, *sf = nullptr;
  if (!distf.empty()) {
    df = fopen(distf.c_str(), "wb");
    if (!df) { perror(distf.c_str()); return 2; }
  }
  if (!pathf.empty()) {
    pf = fopen(pathf.c_str(), "wb");
    if (!pf) { perror(pathf.c_str()); return 2; }
  }
  if (!sumf.empty()) {
    sf = fopen(sumf.c_str(), "wb");
    if (!sf) { perror(sumf.c_str()); return 2; }
  }
  const int64_t n = g.num_vertexs;
  for (int p : todo) {
    if (p < 1 || p > K) { fprintf(stderr, "bad part %d\n", p); return 2; }
    const int64_t s = g.C_BlockVer_num[p];
    std::vector<float> dist((size_t)(s * n));
    std::vector<int32_t> path((size_t)(s * n));
    double a = now_s();
    g.run(dist.data(), path.data(), p);
    double b = now_s();
    if (df) put(df, dist.data(), dist.size());
    if (pf) put(pf, path.data(), path.size());
    if (sf) put_rowsums(sf, dist.data(), s, n);
    printf("{\"event\": \"part\", \"part\": %d, \"rows\": %lld, \"bdy\": %d, \"entries\": %lld, \"seconds\": %.6f}\n",
           p, (long long)s, g.C_BlockBdy_num[p], (long long)(s * n), b - a);
    fflush(stdout);
  }
  if (df) fclose(df);
  if (pf) fclose(pf);
  if (sf) fclose(sf);
  std::cout.rdbuf(saved);
  return 0;
}
