// Host side of the drop-in fap::fapGraph (include/fap/fap.h): graph IO,
// METIS partitioning, boundary detection and renumbering stay on the host,
// exactly as the reference does them, and stages 1-3 go to the GPU through
// the C ABI (include/fap_b200.h).
//
// Reference behaviour reproduced here (Liu-xiandong/FastAPSP):
//   readVerEdges / readMatFile   fap/utils/readMatFile.h:36-173
//   Graph_decomposition          fap/utils/readIdFile.h:71-132
//   findBoundry                  fap/utils/util_preprocess.h:32-58
//   sort_and_encode              fap/utils/util_preprocess.h:73-106
//   fapGraph                     fap/fap.cpp:27-277
#include "fap/fap.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <map>
#include <string>
#include <unordered_set>
#include <vector>

#include "fap_b200.h"
#include "fap_host.h"

// METIS 5 k-way partitioner.  The CUDA toolkit's libmetis_static.a is linked
// into this library; it uses 64-bit idx_t.
extern "C" int METIS_PartGraphKway(int64_t *nvtxs, int64_t *ncon, int64_t *xadj, int64_t *adjncy,
                                   int64_t *vwgt, int64_t *vsize, int64_t *adjwgt, int64_t *nparts,
                                   float *tpwgts, float *ubvec, int64_t *options, int64_t *edgecut,
                                   int64_t *part);

namespace fap {

namespace {

constexpr int kMetisOk = 1;

[[noreturn]] void raise(int code, const std::string &msg) { throw fapError(code, msg); }

void check(int rc, const char *what) {
  if (rc != FAP_OK) raise(rc, std::string(what) + ": " + fap_last_error());
}

std::string mtx_path(const std::string &name, bool directed, bool weighted) {
  const char *kind = !directed ? (weighted ? "weight-undirected" : "unweight-undirected")
                               : (weighted ? "weight-directed" : "unweight-directed");
  return std::string("graph/") + kind + "/" + name + ".mtx";
}

// MatrixMarket reader with the reference's CSR layout: every input line a b
// [w] inserts a->b (and b->a when undirected); a vertex's adjacency lists its
// insertions newest first (the reference prepends to a linked list per
// vertex, readMatFile.h:30-34,150-162).  Ids are 1-based in the file.
// Weights are |w| as float32, or 1 when unweighted.
struct MtxGraph {
  int32_t n = 0;
  int64_t m_decl = 0;  // declared arcs (2x lines when undirected)
  std::vector<int32_t> adj_size, row_offset, col_val;
  std::vector<float> weight;
};

MtxGraph read_mtx(const std::string &path, bool directed, bool weighted) {
  std::ifstream in(path);
  if (!in) raise(FAP_ERR_IO, "cannot open graph file " + path);
  while (in.peek() == '%') in.ignore(2048, '\n');
  long long n = 0, t = 0, m = 0;
  if (!(in >> n >> t >> m) || n <= 0 || m < 0 || n > INT32_MAX)
    raise(FAP_ERR_IO, "malformed MatrixMarket header in " + path);
  MtxGraph g;
  g.n = (int32_t)n;
  g.m_decl = directed ? m : 2 * m;
  if (g.m_decl > INT32_MAX) raise(FAP_ERR_IO, "too many edges in " + path);
  std::vector<int32_t> src, dst;
  std::vector<float> w;
  src.reserve(g.m_decl);
  dst.reserve(g.m_decl);
  w.reserve(g.m_decl);
  long long a, b;
  double c;
  auto push = [&](long long x, long long y, float wt) {
    if ((int64_t)src.size() >= g.m_decl) raise(FAP_ERR_IO, "more edge lines than declared in " + path);
    src.push_back((int32_t)x);
    dst.push_back((int32_t)y);
    w.push_back(wt);
  };
  for (;;) {
    if (!(in >> a >> b)) break;
    float wt = 1.0f;
    if (weighted) {
      if (!(in >> c)) raise(FAP_ERR_IO, "missing weight in " + path);
      wt = static_cast<float>(std::fabs(c));
    }
    if (a < 1 || a > n || b < 1 || b > n) raise(FAP_ERR_IO, "vertex id out of range in " + path);
    a--;
    b--;
    push(a, b, wt);
    if (!directed) push(b, a, wt);
  }
  const int64_t used = (int64_t)src.size();
  g.adj_size.assign(n, 0);
  g.row_offset.assign(n + 1, 0);
  g.col_val.assign(g.m_decl, 0);
  g.weight.assign(g.m_decl, 0.0f);
  for (int64_t i = 0; i < used; i++) g.adj_size[src[i]]++;
  for (int32_t v = 0; v < n; v++) g.row_offset[v + 1] = g.row_offset[v] + g.adj_size[v];
  // newest insertion first within each vertex
  std::vector<int32_t> fill(g.row_offset.begin(), g.row_offset.end() - 1);
  for (int64_t i = used - 1; i >= 0; i--) {
    const int32_t u = src[i];
    g.col_val[fill[u]] = dst[i];
    g.weight[fill[u]] = w[i];
    fill[u]++;
  }
  return g;
}

// METIS k-way partition with default options; returns 1-based part ids.
// Directed graphs are symmetrised first (self-loops dropped), with the
// reference's containers so that the adjacency order METIS sees is the same
// (readIdFile.h:78-104).  The reference lists only vertices that have an
// edge, which misaligns xadj when some vertex has none; here such vertices
// get an empty adjacency instead.
std::vector<int> metis_partition(int32_t n, int64_t edges, const std::vector<int32_t> &adj_size,
                                 const std::vector<int32_t> &row_offset,
                                 const std::vector<int32_t> &col_val, bool directed, int32_t K) {
  std::vector<int> id(n, 1);
  if (K == 1) return id;
  std::vector<int64_t> xadj(1, 0), adjncy;
  if (directed) {
    std::map<int, std::unordered_set<int>> sym;
    for (int v = 0; v < n; v++) {
      for (int i = 0; i < adj_size[v]; i++) {
        const int u = col_val[row_offset[v] + i];
        if (u == v) continue;
        sym[v].insert(u);
        sym[u].insert(v);
      }
    }
    for (int v = 0; v < n; v++) {
      auto it = sym.find(v);
      if (it != sym.end())
        for (int u : it->second) adjncy.push_back(u);
      xadj.push_back((int64_t)adjncy.size());
    }
  } else {
    xadj.assign(row_offset.begin(), row_offset.end());
    adjncy.assign(col_val.begin(), col_val.begin() + std::max<int64_t>(edges, row_offset[n]));
  }
  if (adjncy.empty()) adjncy.push_back(0);
  int64_t nv = n, ncon = 1, np = K, objval = 0;
  std::vector<int64_t> part(n, 0);
  const int ret = METIS_PartGraphKway(&nv, &ncon, xadj.data(), adjncy.data(), nullptr, nullptr,
                                      nullptr, &np, nullptr, nullptr, nullptr, &objval, part.data());
  if (ret != kMetisOk) raise(FAP_ERR_PARTITION, "METIS_PartGraphKway failed");
  for (int32_t i = 0; i < n; i++) {
    if (part[i] < 0 || part[i] >= K) raise(FAP_ERR_PARTITION, "METIS returned an invalid part id");
    id[i] = (int)part[i] + 1;
  }
  return id;
}

struct DenseNode {
  int v;
  int GraphId;
  int isBound;
};

// Part ascending, boundary vertices first within a part (util_preprocess.h:66-71).
bool node_order(const DenseNode &a, const DenseNode &b) {
  if (a.GraphId == b.GraphId) return a.isBound > b.isBound;
  return a.GraphId < b.GraphId;
}

}  // namespace

// ---------------------------------------------------------------------------
// construction
// ---------------------------------------------------------------------------
void fapGraph::init_storage() {
  graph_id.assign(num_vertexs, 0);
  st2ed.assign(num_vertexs, 0);
  ed2st.assign(num_vertexs, 0);
  C_BlockVer_num.assign(K + 1, 0);
  C_BlockVer_offset.assign(K + 1, 0);
  C_BlockBdy_num.assign(K + 1, 0);
  C_BlockBdy_offset.assign(K + 1, 0);
}

fapGraph::fapGraph(std::string input_graph, bool directed, bool weight, int32_t K) {
  if (K < 1) raise(FAP_ERR_INVALID, "K must be >= 1");
  this->input_graph = input_graph;
  this->directed = directed;
  this->weighted = weight;
  MtxGraph g = read_mtx(mtx_path(input_graph, directed, weight), directed, weight);
  if (K > g.n) raise(FAP_ERR_INVALID, "K exceeds the number of vertices");
  num_vertexs = g.n;
  num_edges = (int32_t)g.m_decl;
  this->K = K;
  adj_size = std::move(g.adj_size);
  row_offset = std::move(g.row_offset);
  col_val = std::move(g.col_val);
  this->weight = std::move(g.weight);
  init_storage();
  graph_id = metis_partition(num_vertexs, num_edges, adj_size, row_offset, col_val, directed, K);
  for (int i = 0; i < num_vertexs; i++) BlockVer[graph_id[i]].push_back(i);
}

fapGraph::fapGraph(int32_t n, int64_t m, std::vector<int32_t> ro, std::vector<int32_t> cv,
                   std::vector<float> w, int32_t K)
    : fapGraph(n, m, std::move(ro), std::move(cv), std::move(w), K, false) {}

fapGraph::fapGraph(int32_t n, int64_t m, std::vector<int32_t> ro, std::vector<int32_t> cv,
                   std::vector<float> w, int32_t K, bool directed) {
  if (n <= 0 || K < 1 || K > n) raise(FAP_ERR_INVALID, "need n > 0 and 1 <= K <= n");
  if ((int64_t)ro.size() != (int64_t)n + 1 || ro[0] != 0 || ro[n] > m || (int64_t)cv.size() < ro[n] ||
      (int64_t)w.size() < ro[n])
    raise(FAP_ERR_INVALID, "inconsistent CSR");
  num_vertexs = n;
  num_edges = (int32_t)m;
  this->K = K;
  this->directed = directed;
  weighted = true;
  row_offset = std::move(ro);
  col_val = std::move(cv);
  weight = std::move(w);
  col_val.resize(std::max<int64_t>(m, row_offset[n]), 0);
  weight.resize(std::max<int64_t>(m, row_offset[n]), 0.0f);
  adj_size.assign(n, 0);
  for (int32_t v = 0; v < n; v++) {
    if (row_offset[v + 1] < row_offset[v]) raise(FAP_ERR_INVALID, "row_offset not monotone");
    adj_size[v] = row_offset[v + 1] - row_offset[v];
  }
  for (int64_t e = 0; e < row_offset[n]; e++)
    if (col_val[e] < 0 || col_val[e] >= n) raise(FAP_ERR_INVALID, "col_val out of range");
  init_storage();
  graph_id = metis_partition(num_vertexs, num_edges, adj_size, row_offset, col_val, directed, K);
  for (int i = 0; i < num_vertexs; i++) BlockVer[graph_id[i]].push_back(i);
}

fapGraph::~fapGraph() {
  if (dg_) fap_graph_destroy(dg_);
  if (ctx_) fap_ctx_destroy(ctx_);
}

void fapGraph::setPartition(const std::vector<int32_t> &gid) {
  if ((int32_t)gid.size() != num_vertexs) raise(FAP_ERR_PARTITION, "partition size != n");
  for (int32_t v : gid)
    if (v < 1 || v > K) raise(FAP_ERR_PARTITION, "partition id outside 1..K");
  graph_id.assign(gid.begin(), gid.end());
  BlockVer.clear();
  for (int i = 0; i < num_vertexs; i++) BlockVer[graph_id[i]].push_back(i);
  partition_injected_ = true;
  prepared_ = false;
}

// ---------------------------------------------------------------------------
// Binary graph file: magic, sizes, CSR, partition, FNV-1a 64 checksum of
// everything before it.  Little-endian, as written by this library.
// ---------------------------------------------------------------------------
namespace {
constexpr char kBinMagic[8] = {'F', 'A', 'P', 'C', 'S', 'R', '0', '1'};

struct BinHeader {
  char magic[8];
  int32_t n;
  int32_t K;
  int64_t m_decl;  // the declared edge count (num_edges)
  int64_t nnz;     // row_offset[n]
  int32_t directed;
  int32_t weighted;
};

uint64_t fnv1a(uint64_t h, const void *p, size_t len) {
  const unsigned char *b = static_cast<const unsigned char *>(p);
  for (size_t i = 0; i < len; i++) {
    h ^= b[i];
    h *= 1099511628211ull;
  }
  return h;
}
}  // namespace

void fapGraph::saveBinary(const std::string &path) const {
  BinHeader h{};
  std::memcpy(h.magic, kBinMagic, 8);
  h.n = num_vertexs;
  h.K = K;
  h.m_decl = num_edges;
  h.nnz = row_offset.empty() ? 0 : row_offset[num_vertexs];
  h.directed = directed ? 1 : 0;
  h.weighted = weighted ? 1 : 0;
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) raise(FAP_ERR_IO, "cannot write " + path);
  uint64_t sum = 14695981039346656037ull;
  auto put = [&](const void *p, size_t len) {
    f.write(static_cast<const char *>(p), (std::streamsize)len);
    sum = fnv1a(sum, p, len);
  };
  put(&h, sizeof(h));
  put(row_offset.data(), ((size_t)num_vertexs + 1) * 4);
  put(col_val.data(), (size_t)h.nnz * 4);
  put(weight.data(), (size_t)h.nnz * 4);
  put(graph_id.data(), (size_t)num_vertexs * 4);
  f.write(reinterpret_cast<const char *>(&sum), sizeof(sum));
  if (!f) raise(FAP_ERR_IO, "write failed: " + path);
}

std::unique_ptr<fapGraph> fapGraph::loadBinary(const std::string &path) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) raise(FAP_ERR_IO, "cannot read " + path);
  const int64_t size = (int64_t)f.tellg();
  f.seekg(0);
  BinHeader h{};
  if (size < (int64_t)sizeof(h) || !f.read(reinterpret_cast<char *>(&h), sizeof(h)) ||
      std::memcmp(h.magic, kBinMagic, 8) != 0)
    raise(FAP_ERR_IO, path + ": not a binary graph file");
  if (h.n <= 0 || h.K < 1 || h.K > h.n || h.nnz < 0 || h.nnz > INT32_MAX || h.m_decl < h.nnz ||
      h.m_decl > INT32_MAX)
    raise(FAP_ERR_IO, path + ": bad sizes");
  const int64_t want = (int64_t)sizeof(h) + ((int64_t)h.n + 1) * 4 + 2 * h.nnz * 4 + (int64_t)h.n * 4 + 8;
  if (size != want) raise(FAP_ERR_IO, path + ": truncated or oversized");
  uint64_t sum = fnv1a(14695981039346656037ull, &h, sizeof(h));
  auto get = [&](void *p, size_t len) {
    if (!f.read(static_cast<char *>(p), (std::streamsize)len)) raise(FAP_ERR_IO, path + ": short read");
    sum = fnv1a(sum, p, len);
  };
  std::vector<int32_t> ro((size_t)h.n + 1), cv((size_t)h.nnz), gid((size_t)h.n);
  std::vector<float> w((size_t)h.nnz);
  get(ro.data(), ro.size() * 4);
  get(cv.data(), cv.size() * 4);
  get(w.data(), w.size() * 4);
  get(gid.data(), gid.size() * 4);
  uint64_t stored = 0;
  if (!f.read(reinterpret_cast<char *>(&stored), sizeof(stored)) || stored != sum)
    raise(FAP_ERR_IO, path + ": checksum mismatch");
  if (ro[0] != 0 || ro[h.n] != h.nnz) raise(FAP_ERR_IO, path + ": inconsistent CSR");
  for (int32_t v = 0; v < h.n; v++)
    if (ro[v + 1] < ro[v]) raise(FAP_ERR_IO, path + ": row_offset not monotone");
  for (int32_t c : cv)
    if (c < 0 || c >= h.n) raise(FAP_ERR_IO, path + ": col_val out of range");
  for (int32_t p : gid)
    if (p < 1 || p > h.K) raise(FAP_ERR_IO, path + ": part id outside 1..K");
  return std::unique_ptr<fapGraph>(new fapGraph(LoadedTag{}, h.n, h.m_decl, std::move(ro), std::move(cv),
                                                std::move(w), h.K, h.directed != 0, h.weighted != 0,
                                                std::move(gid)));
}

fapGraph::fapGraph(LoadedTag, int32_t n, int64_t m, std::vector<int32_t> ro, std::vector<int32_t> cv,
                   std::vector<float> w, int32_t K, bool directed, bool weighted, std::vector<int32_t> gid) {
  num_vertexs = n;
  num_edges = (int32_t)m;
  this->K = K;
  this->directed = directed;
  this->weighted = weighted;
  row_offset = std::move(ro);
  col_val = std::move(cv);
  weight = std::move(w);
  col_val.resize(std::max<int64_t>(m, row_offset[n]), 0);
  weight.resize(std::max<int64_t>(m, row_offset[n]), 0.0f);
  adj_size.assign(n, 0);
  for (int32_t v = 0; v < n; v++) adj_size[v] = row_offset[v + 1] - row_offset[v];
  init_storage();
  graph_id.assign(gid.begin(), gid.end());
  for (int i = 0; i < num_vertexs; i++) BlockVer[graph_id[i]].push_back(i);
}

void fapGraph::setDevice(int device) { device_ = device; }
void fapGraph::setDtype(int dtype) { dtype_ = dtype; }
void fapGraph::setMode(SolveMode mode) { mode_ = mode; }
void fapGraph::setMaxResidentRows(int64_t rows) {
  row_limit_ = std::max<int64_t>(rows, 0);
  if (dg_) check(fap_graph_set_param(dg_, "max_resident_rows", (double)row_limit_), "max_resident_rows");
}

int fapGraph::getDtype() {
  ensure_device();
  return fap_graph_dtype(dg_);
}

// ---------------------------------------------------------------------------
// preCondition: boundary flags + renumbering (util_preprocess.h:32-106)
// ---------------------------------------------------------------------------
void fapGraph::preCondition() {
  const int n = num_vertexs;
  isBoundry.clear();
  BlockBoundary.clear();
  std::vector<char> bdy(n, 0);
  for (int v = 0; v < n; v++) {
    for (int e = row_offset[v]; e < row_offset[v] + adj_size[v]; e++) {
      const int u = col_val[e];
      if (graph_id[u] != graph_id[v]) {
        bdy[v] = 1;
        bdy[u] = 1;
      }
    }
  }
  for (int v = 0; v < n; v++) {
    isBoundry[v] = bdy[v];
    if (bdy[v]) BlockBoundary[graph_id[v]].push_back(v);
  }
  std::vector<DenseNode> nodes(n);
  for (int v = 0; v < n; v++) nodes[v] = DenseNode{v, graph_id[v], (int)bdy[v]};
  std::sort(nodes.begin(), nodes.end(), node_order);
  for (int i = 0; i < n; i++) {
    st2ed[i] = nodes[i].v;
    ed2st[nodes[i].v] = i;
  }
  int cnt = 0;
  max_subgraph_vertexs = 0;
  for (int p = 1; p <= K; p++) {
    C_BlockVer_offset[p] = cnt;
    C_BlockVer_num[p] = (int)BlockVer[p].size();
    C_BlockBdy_offset[p] = cnt;
    C_BlockBdy_num[p] = (int)BlockBoundary[p].size();
    cnt += (int)BlockVer[p].size();
    max_subgraph_vertexs = std::max(max_subgraph_vertexs, C_BlockVer_num[p]);
  }
  is_split = (num_vertexs > max_vertexs_num_limit);
  prepared_ = true;
  cache_tried_ = false;
  if (dg_) {
    check(fap_graph_set_parts(dg_, K, graph_id.data(), st2ed.data(), C_BlockVer_num.data(),
                              C_BlockVer_offset.data(), C_BlockBdy_num.data()),
          "fap_graph_set_parts");
  }
}

bool fapGraph::isSplit() { return is_split; }
std::vector<int> fapGraph::getGraphId() { return graph_id; }

// ---------------------------------------------------------------------------
// GPU plumbing
// ---------------------------------------------------------------------------
void fapGraph::ensure_device() {
  if (!ctx_) check(fap_ctx_create(device_, &ctx_), "fap_ctx_create");
  if (!dg_) {
    check(fap_graph_create(ctx_, num_vertexs, row_offset[num_vertexs], row_offset.data(),
                           col_val.data(), weight.data(), dtype_, &dg_),
          "fap_graph_create");
    if (prepared_)
      check(fap_graph_set_parts(dg_, K, graph_id.data(), st2ed.data(), C_BlockVer_num.data(),
                                C_BlockVer_offset.data(), C_BlockBdy_num.data()),
            "fap_graph_set_parts");
    if (row_limit_ > 0)
      check(fap_graph_set_param(dg_, "max_resident_rows", (double)row_limit_), "max_resident_rows");
  }
}

void fapGraph::run_parts(const std::vector<int32_t> &ids) {
  check(fap_solve(dg_, ids.data(), (int32_t)ids.size(), static_cast<int>(mode_)), "fap_solve");
  check(fap_graph_check(dg_), "fap_graph_check");
}

// Output rows for solving the parts in groups, when the device holds fewer
// than n of them: as many as setMaxResidentRows allows, else room for
// `need` rows (the largest part to be solved; fewer allowed rows than that
// raise FAP_ERR_NOMEM).  In
// the batched form every part's stage-1 rows and local closure are also
// kept resident once, when they fit (fap_graph_cache_build), so that each
// group runs only its parts' min-plus merge; without room for them each
// group runs its own stage 1.
int64_t fapGraph::reserve_group_rows(int64_t need) {
  need = std::max<int64_t>(need, 1);
  int64_t rows = need;
  if (row_limit_ >= need && fap_graph_reserve(dg_, row_limit_) == FAP_OK) {
    rows = row_limit_;
  } else {
    check(fap_graph_reserve(dg_, need), "fap_graph_reserve");
  }
  if (mode_ == SolveMode::Batched && !cache_tried_) {
    cache_tried_ = true;
    (void)fap_graph_cache_build(dg_);  // FAP_ERR_NOMEM: groups run stage 1 themselves
  }
  return rows;
}

// Solves every part into all n output rows, reserving them again when an
// earlier grouped solve left fewer; FAP_ERR_NOMEM when they do not fit.
int fapGraph::solve_all(int mode) {
  std::vector<int32_t> all;
  for (int32_t p = 1; p <= K; p++) all.push_back(p);
  int rc = fap_solve(dg_, all.data(), K, mode);
  if (rc == FAP_ERR_NOMEM && fap_graph_reserve(dg_, 0) == FAP_OK) rc = fap_solve(dg_, all.data(), K, mode);
  return rc;
}

// Solves parts first, first + 1, ... while their rows fit in `rows`; returns
// the first part not solved.
int32_t fapGraph::run_group(int32_t first, int64_t rows) {
  std::vector<int32_t> ids;
  int64_t used = 0;
  for (int32_t p = first; p <= K; p++) {
    if (!ids.empty() && used + C_BlockVer_num[p] > rows) break;
    ids.push_back(p);
    used += C_BlockVer_num[p];
  }
  run_parts(ids);
  return first + (int32_t)ids.size();
}

void fapGraph::copy_block(int32_t id, float *dst) {
  check(fap_graph_copy_block(dg_, id, dst, FAP_DTYPE_F32), "fap_graph_copy_block");
}

void fapGraph::copy_path_block(int32_t id, int32_t *dst) {
  check(fap_graph_copy_path_block(dg_, id, dst), "fap_graph_copy_path_block");
}

void fapGraph::set_paths(bool on) {
  check(fap_graph_set_param(dg_, "paths", on ? 1.0 : 0.0), "paths");
}

int32_t fapGraph::solve(bool path_needed) {
  if (!prepared_) raise(FAP_ERR_STATE, "solve before preCondition");
  is_path_needed = path_needed;
  ensure_device();
  set_paths(path_needed);
  const int64_t n = num_vertexs;
  dist.assign((size_t)(n * n), 0.0f);
  path.assign((size_t)(n * n), -1);
  path_ready_ = false;
  const int rc = solve_all(static_cast<int>(mode_));
  if (rc == FAP_OK) {
    check(fap_graph_check(dg_), "fap_graph_check");
    for (int32_t p = 1; p <= K; p++) {
      copy_block(p, dist.data() + (size_t)C_BlockVer_offset[p] * n);
      if (path_needed) copy_path_block(p, path.data() + (size_t)C_BlockVer_offset[p] * n);
    }
  } else if (rc == FAP_ERR_NOMEM) {
    // Fewer than n rows fit on the device: solve and copy group by group.
    const int64_t rows = reserve_group_rows(max_subgraph_vertexs);
    for (int32_t p = 1; p <= K;) {
      const int32_t next = run_group(p, rows);
      for (; p < next; p++) {
        copy_block(p, dist.data() + (size_t)C_BlockVer_offset[p] * n);
        if (path_needed) copy_path_block(p, path.data() + (size_t)C_BlockVer_offset[p] * n);
      }
    }
  } else {
    check(rc, "fap_solve");
  }
  path_ready_ = path_needed;
  return 0;
}

int32_t fapGraph::solveSubGraph(int32_t id, bool path_needed) {
  if (!prepared_) raise(FAP_ERR_STATE, "solveSubGraph before preCondition");
  if (id < 1 || id > K) return -1;
  is_path_needed = path_needed;
  ensure_device();
  if (path_needed) set_paths(true);
  const int64_t n = num_vertexs;
  void *dp;
  int64_t rows, ld;
  if (mode_ == SolveMode::Plain) {
    // Plain form: every call solves its part with its own launch sequence.
    const int rc = fap_solve(dg_, &id, 1, FAP_MODE_PLAIN);
    if (rc == FAP_ERR_NOMEM) {
      reserve_group_rows(C_BlockVer_num[id]);
      run_parts({id});
    } else {
      check(rc, "fap_solve");
      check(fap_graph_check(dg_), "fap_graph_check");
    }
  } else if (fap_graph_block(dg_, id, &dp, &rows, &ld) != FAP_OK ||
             (path_needed && fap_graph_path_block(dg_, id, &dp, &rows, &ld) != FAP_OK)) {
    // Batched form: solve every part once (blocks stay resident in HBM);
    // later calls only copy.  Without room for every block, solve this part
    // and the ones after it that fit (the reference's callers visit the
    // parts in order), from the resident cache when it fits.
    const int rc = solve_all(FAP_MODE_BATCHED);
    if (rc == FAP_OK) {
      check(fap_graph_check(dg_), "fap_graph_check");
    } else if (rc == FAP_ERR_NOMEM) {
      run_group(id, reserve_group_rows(C_BlockVer_num[id]));
    } else {
      check(rc, "fap_solve");
    }
  }
  subgraph_dist.resize((size_t)C_BlockVer_num[id] * n);
  subgraph_path.assign((size_t)C_BlockVer_num[id] * n, -1);
  current_subgraph_id = id;
  copy_block(id, subgraph_dist.data());
  if (path_needed) copy_path_block(id, subgraph_path.data());
  return 0;
}

// ---------------------------------------------------------------------------
// getters
// ---------------------------------------------------------------------------
std::vector<int32_t> fapGraph::getMapping() { return st2ed; }

std::vector<float> fapGraph::getAllDistance() {
  if (is_split) raise(FAP_ERR_STATE, "getAllDistance on a split graph");
  return dist;
}

std::vector<int32_t> fapGraph::getAllPath() {
  if (is_split) raise(FAP_ERR_STATE, "getAllPath on a split graph");
  return path;
}

std::vector<int32_t> fapGraph::getSubGraphIndex(int32_t id) {
  if (id < 1 || id > K) raise(FAP_ERR_INVALID, "part id out of range");
  const int off = C_BlockVer_offset[id], size = C_BlockVer_num[id];
  return std::vector<int32_t>(st2ed.begin() + off, st2ed.begin() + off + size);
}

int32_t fapGraph::getCurrentSubGraphId() { return current_subgraph_id; }

std::vector<float> fapGraph::getSubGraphDistance(int32_t id) {
  if (id != current_subgraph_id) raise(FAP_ERR_STATE, "part is not the current one");
  return subgraph_dist;
}

std::vector<int32_t> fapGraph::getSubGraphPath(int32_t id) {
  if (id != current_subgraph_id) raise(FAP_ERR_STATE, "part is not the current one");
  return subgraph_path;
}

std::vector<float> fapGraph::getDistanceFromOnePoint(int32_t v) {
  if (v < 0 || v >= num_vertexs) raise(FAP_ERR_INVALID, "vertex out of range");
  if (graph_id[v] != current_subgraph_id) raise(FAP_ERR_STATE, "vertex is not in the current part");
  const int64_t n = num_vertexs;
  const int64_t row = ed2st[v] - C_BlockVer_offset[current_subgraph_id];
  return std::vector<float>(subgraph_dist.begin() + row * n, subgraph_dist.begin() + (row + 1) * n);
}

std::vector<int32_t> fapGraph::getPathFromOnePoint(int32_t v) {
  if (v < 0 || v >= num_vertexs) raise(FAP_ERR_INVALID, "vertex out of range");
  if (graph_id[v] != current_subgraph_id) raise(FAP_ERR_STATE, "vertex is not in the current part");
  const int64_t n = num_vertexs;
  const int64_t row = ed2st[v] - C_BlockVer_offset[current_subgraph_id];
  return std::vector<int32_t>(subgraph_path.begin() + row * n, subgraph_path.begin() + (row + 1) * n);
}

float fapGraph::getDistanceP2P(int32_t from, int32_t to) {
  if (from < 0 || from >= num_vertexs || to < 0 || to >= num_vertexs)
    raise(FAP_ERR_INVALID, "vertex out of range");
  const int64_t n = num_vertexs;
  if (!dist.empty()) return dist[(size_t)ed2st[from] * n + to];
  if (graph_id[from] != current_subgraph_id) solveSubGraph(graph_id[from]);
  const int64_t row = ed2st[from] - C_BlockVer_offset[current_subgraph_id];
  return subgraph_dist[(size_t)row * n + to];
}

float fapGraph::getDistanceP2P() {
  raise(FAP_ERR_INVALID, "getDistanceP2P needs its two endpoints: getDistanceP2P(from, to)");
}

std::vector<int32_t> fapGraph::getPathP2P() {
  raise(FAP_ERR_INVALID, "getPathP2P needs its two endpoints: getPathP2P(from, to)");
}

// The vertices of a shortest path from `from` to `to` (both included), read
// off the predecessor row of `from`; empty when `to` is unreachable.  The
// reference leaves this a TODO (fap/fap.cpp:263-269).
std::vector<int32_t> fapGraph::getPathP2P(int32_t from, int32_t to) {
  if (from < 0 || from >= num_vertexs || to < 0 || to >= num_vertexs)
    raise(FAP_ERR_INVALID, "vertex out of range");
  const int64_t n = num_vertexs;
  const int32_t *row = nullptr;
  if (path_ready_) {
    row = path.data() + (size_t)ed2st[from] * n;
  } else {
    if (graph_id[from] != current_subgraph_id || !is_path_needed) solveSubGraph(graph_id[from], true);
    row = subgraph_path.data() + (size_t)(ed2st[from] - C_BlockVer_offset[current_subgraph_id]) * n;
  }
  std::vector<int32_t> out;
  int32_t cur = to;
  out.push_back(cur);
  while (cur != from) {
    cur = row[cur];
    if (cur < 0) return {};
    out.push_back(cur);
    if ((int64_t)out.size() > n) raise(FAP_ERR_STATE, "predecessor chain does not end at the source");
  }
  std::reverse(out.begin(), out.end());
  return out;
}

bool fapGraph::check_result(float *d, int *p, int *source, int source_num, int vertexs, int *,
                            int *, int *, float *, int *) {
  (void)p;
  if (source_num <= 0 || vertexs != num_vertexs) return false;
  ensure_device();
  unsigned int seed = (unsigned int)time(nullptr);
  const int cases = 20, cols = 10;
  std::vector<int32_t> rows_idx(cases), srcs(cases);
  for (int c = 0; c < cases; c++) {
    rows_idx[c] = rand_r(&seed) % source_num;
    srcs[c] = source[rows_idx[c]];
  }
  std::vector<float> ref((size_t)cases * vertexs);
  check(fap_graph_sssp_rows(dg_, srcs.data(), cases, ref.data()), "fap_graph_sssp_rows");
  const float big = 1e8f / 10;
  for (int c = 0; c < cases; c++) {
    for (int k = 0; k < cols; k++) {
      const int des = rand_r(&seed) % vertexs;
      const float now = d[(size_t)rows_idx[c] * vertexs + des];
      const float want = ref[(size_t)c * vertexs + des];
      if (now > big && want > big) continue;
      if (std::fabs(now - want) > 1e-5f) return false;
    }
  }
  return true;
}

}  // namespace fap

// ---------------------------------------------------------------------------
// C wrappers of fap::fapGraph (for FFI callers, e.g. the Python mirror)
// ---------------------------------------------------------------------------
namespace {
thread_local std::string h_err;
int h_fail(const fap::fapError &e) {
  h_err = e.what();
  return e.code() < 0 ? e.code() : FAP_ERR_INVALID;
}
int h_fail_std(const std::exception &e) {
  h_err = e.what();
  return FAP_ERR_INVALID;
}
int h_invalid(const char *msg) {
  h_err = msg;
  return FAP_ERR_INVALID;
}
}  // namespace

// Every pointer argument of a wrapper is checked: NULL is FAP_ERR_INVALID.
#define FAPH_NEED(cond) \
  if (!(cond)) return h_invalid("NULL argument")

#define FAPH_BODY(...)                         \
  try {                                        \
    __VA_ARGS__;                               \
    return FAP_OK;                             \
  } catch (const fap::fapError &e) {           \
    return h_fail(e);                          \
  } catch (const std::bad_alloc &) {           \
    h_err = "host allocation failed";          \
    return FAP_ERR_NOMEM;                      \
  } catch (const std::exception &e) {          \
    return h_fail_std(e);                      \
  }

extern "C" {

const char *fap_host_last_error(void) { return h_err.c_str(); }

int fap_host_from_mtx(const char *name, int directed, int weighted, int K, fap::fapGraph **out) {
  FAPH_NEED(name && out);
  FAPH_BODY(*out = new fap::fapGraph(std::string(name), directed != 0, weighted != 0, K))
}

int fap_host_from_csr(int32_t n, int64_t m, const int32_t *ro, const int32_t *col, const float *w,
                      int K, int directed, fap::fapGraph **out) {
  FAPH_NEED(ro && out && (m <= 0 || (col && w)));
  if (n <= 0 || m < 0) return h_invalid("n must be positive and m non-negative");
  FAPH_BODY({
    std::vector<int32_t> r(ro, ro + n + 1), c(col, col + m);
    std::vector<float> ww(w, w + m);
    *out = new fap::fapGraph(n, m, std::move(r), std::move(c), std::move(ww), K, directed != 0);
  })
}

int fap_host_save(fap::fapGraph *g, const char *path) {
  FAPH_NEED(g && path);
  FAPH_BODY(g->saveBinary(path))
}

int fap_host_load(const char *path, fap::fapGraph **out) {
  FAPH_NEED(path && out);
  FAPH_BODY(*out = fap::fapGraph::loadBinary(path).release())
}

int fap_host_destroy(fap::fapGraph *g) {
  delete g;
  return FAP_OK;
}

int fap_host_set_partition(fap::fapGraph *g, const int32_t *gid) {
  FAPH_NEED(g && gid);
  FAPH_BODY(g->setPartition(std::vector<int32_t>(gid, gid + g->num_vertexs)))
}

int fap_host_set_options(fap::fapGraph *g, int device, int dtype, int mode) {
  FAPH_NEED(g);
  FAPH_BODY({
    g->setDevice(device);
    g->setDtype(dtype);
    g->setMode(mode == 0 ? fap::SolveMode::Plain : fap::SolveMode::Batched);
  })
}

int fap_host_set_max_resident_rows(fap::fapGraph *g, int64_t rows) {
  FAPH_NEED(g);
  FAPH_BODY(g->setMaxResidentRows(rows))
}

int fap_host_precondition(fap::fapGraph *g) {
  FAPH_NEED(g);
  FAPH_BODY(g->preCondition())
}

int fap_host_is_split(fap::fapGraph *g) {
  FAPH_NEED(g);
  return g->isSplit() ? 1 : 0;
}

int fap_host_dtype(fap::fapGraph *g) {
  FAPH_NEED(g);
  int dt = FAP_ERR_INVALID;
  try {
    dt = g->getDtype();
  } catch (const fap::fapError &e) {
    return h_fail(e);
  } catch (const std::bad_alloc &) {
    h_err = "host allocation failed";
    return FAP_ERR_NOMEM;
  } catch (const std::exception &e) {
    return h_fail_std(e);
  }
  return dt;
}

// sizes: [n, m_decl, K, stored arcs]
int fap_host_flags(fap::fapGraph *g, int *directed, int *weighted) {
  FAPH_NEED(g && directed && weighted);
  *directed = g->directed ? 1 : 0;
  *weighted = g->weighted ? 1 : 0;
  return FAP_OK;
}

int fap_host_sizes(fap::fapGraph *g, int64_t *out4) {
  FAPH_NEED(g && out4);
  out4[0] = g->num_vertexs;
  out4[1] = g->num_edges;
  out4[2] = g->getK();
  out4[3] = g->row_offset.empty() ? 0 : g->row_offset.back();
  return FAP_OK;
}

int fap_host_csr(fap::fapGraph *g, int32_t *ro, int32_t *col, float *w) {
  FAPH_NEED(g && ro && col && w);
  const int64_t used = g->row_offset.back();
  std::memcpy(ro, g->row_offset.data(), (g->num_vertexs + 1) * sizeof(int32_t));
  std::memcpy(col, g->col_val.data(), used * sizeof(int32_t));
  std::memcpy(w, g->weight.data(), used * sizeof(float));
  return FAP_OK;
}

int fap_host_graph_id(fap::fapGraph *g, int32_t *out) {
  FAPH_NEED(g && out);
  auto v = g->getGraphId();
  std::memcpy(out, v.data(), v.size() * sizeof(int32_t));
  return FAP_OK;
}

int fap_host_mapping(fap::fapGraph *g, int32_t *out) {
  FAPH_NEED(g && out);
  auto v = g->getMapping();
  std::memcpy(out, v.data(), v.size() * sizeof(int32_t));
  return FAP_OK;
}

// ver_num, ver_offset, bdy_num: K+1 entries each
int fap_host_parts(fap::fapGraph *g, int32_t *vnum, int32_t *voff, int32_t *bnum) {
  FAPH_NEED(g && vnum && voff && bnum);
  const int K = g->getK();
  std::memcpy(vnum, g->getBlockVerNum().data(), (K + 1) * sizeof(int32_t));
  std::memcpy(voff, g->getBlockVerOffset().data(), (K + 1) * sizeof(int32_t));
  std::memcpy(bnum, g->getBlockBdyNum().data(), (K + 1) * sizeof(int32_t));
  return FAP_OK;
}

int fap_host_solve(fap::fapGraph *g, int path_needed) {
  FAPH_NEED(g);
  FAPH_BODY(g->solve(path_needed != 0))
}

int fap_host_solve_subgraph(fap::fapGraph *g, int id, int path_needed) {
  FAPH_NEED(g);
  FAPH_BODY({
    if (g->solveSubGraph(id, path_needed != 0) != 0) throw fap::fapError(FAP_ERR_INVALID, "bad part id");
  })
}

int fap_host_current_subgraph(fap::fapGraph *g) {
  FAPH_NEED(g);
  return g->getCurrentSubGraphId();
}

int fap_host_subgraph_distance(fap::fapGraph *g, int id, float *out) {
  FAPH_NEED(g && out);
  FAPH_BODY({
    auto v = g->getSubGraphDistance(id);
    std::memcpy(out, v.data(), v.size() * sizeof(float));
  })
}

int fap_host_all_distance(fap::fapGraph *g, float *out) {
  FAPH_NEED(g && out);
  FAPH_BODY({
    auto v = g->getAllDistance();
    std::memcpy(out, v.data(), v.size() * sizeof(float));
  })
}

int fap_host_distance_from_one_point(fap::fapGraph *g, int v, float *out) {
  FAPH_NEED(g && out);
  FAPH_BODY({
    auto r = g->getDistanceFromOnePoint(v);
    std::memcpy(out, r.data(), r.size() * sizeof(float));
  })
}

int fap_host_distance_p2p(fap::fapGraph *g, int from, int to, float *out) {
  FAPH_NEED(g && out);
  FAPH_BODY(*out = g->getDistanceP2P(from, to))
}

int fap_host_subgraph_path(fap::fapGraph *g, int id, int32_t *out) {
  FAPH_NEED(g && out);
  FAPH_BODY({
    auto v = g->getSubGraphPath(id);
    std::memcpy(out, v.data(), v.size() * sizeof(int32_t));
  })
}

int fap_host_all_path(fap::fapGraph *g, int32_t *out) {
  FAPH_NEED(g && out);
  FAPH_BODY({
    auto v = g->getAllPath();
    std::memcpy(out, v.data(), v.size() * sizeof(int32_t));
  })
}

int fap_host_path_from_one_point(fap::fapGraph *g, int v, int32_t *out) {
  FAPH_NEED(g && out);
  FAPH_BODY({
    auto r = g->getPathFromOnePoint(v);
    std::memcpy(out, r.data(), r.size() * sizeof(int32_t));
  })
}

int fap_host_path_p2p(fap::fapGraph *g, int from, int to, int32_t *out, int32_t cap, int32_t *len) {
  FAPH_NEED(g && len && (out || cap <= 0));
  FAPH_BODY({
    auto r = g->getPathP2P(from, to);
    *len = (int32_t)r.size();
    if ((int32_t)r.size() > cap) throw fap::fapError(FAP_ERR_INVALID, "output buffer too small");
    std::memcpy(out, r.data(), r.size() * sizeof(int32_t));
  })
}

int fap_host_check_result(fap::fapGraph *g, int id, int *ok) {
  FAPH_NEED(g && ok);
  FAPH_BODY({
    auto d = g->getSubGraphDistance(id);
    auto src = g->getSubGraphIndex(id);
    *ok = g->check_result(d.data(), nullptr, src.data(), (int)src.size(), g->num_vertexs, nullptr,
                          nullptr, nullptr, nullptr, nullptr)
              ? 1
              : 0;
  })
}

fap_dgraph *fap_host_device_graph(fap::fapGraph *g) { return g ? g->deviceGraph() : nullptr; }

}  // extern "C"
