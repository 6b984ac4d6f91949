// fap/fap.h -- drop-in replacement for the reference's fap::fapGraph
// (fap/fap.h:22-125 of Liu-xiandong/FastAPSP), backed by the B200 solve path.
//
// Same constructor, preCondition, isSplit, solve, solveSubGraph and getters.
// Host code keeps the reference's IO, METIS call, boundary detection and
// renumbering; stages 1-3 run on the GPU through the C ABI in fap_b200.h.
//
// Differences from the reference, all fixes of reference defects:
//   - solve / solveSubGraph / check_result return their documented value
//     (the reference falls off the end of these non-void functions,
//     fap/fap.cpp:194,207,277);
//   - the metadata constructor builds the graph (fap/fap.cpp:61-65 is empty);
//   - getDistanceFromOnePoint / getPathFromOnePoint index the requested row
//     (fap/fap.cpp:245-258 forget the row length);
//   - getDistanceP2P / getPathP2P take the two endpoints (TODO in the
//     reference, fap/fap.cpp:263-269; the argument-free forms throw);
//   - errors throw fap::fapError instead of exit().
#ifndef FAP_B200_FAP_H_
#define FAP_B200_FAP_H_

#include <stdint.h>

#include <sstream>
#include <stdexcept>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

struct fap_ctx;
struct fap_dgraph;

namespace fap {

class __attribute__((visibility("default"))) fapError : public std::runtime_error {
 public:
  fapError(int code, const std::string &msg) : std::runtime_error(msg), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

// Solve forms of the GPU path.
enum class SolveMode { Plain = 0, Batched = 1 };

class __attribute__((visibility("default"))) fapGraph {
 protected:
  std::string input_graph;
  std::stringstream input_file;

  const int32_t max_vertexs_num_limit = 20000;
  bool is_split = false;
  bool is_path_needed = false;
  std::string output_file;
  std::vector<float> dist;
  std::vector<int32_t> path;
  int32_t current_subgraph_id = 0;
  std::vector<float> subgraph_dist;
  std::vector<int32_t> subgraph_path;

  int32_t K = 0;
  std::vector<int> graph_id;
  std::unordered_map<int, std::vector<int>> BlockVer;
  std::unordered_map<int, std::vector<int>> BlockBoundary;
  std::unordered_map<int, int> isBoundry;
  std::vector<int> st2ed;
  std::vector<int> ed2st;
  std::vector<int> C_BlockVer_num;
  std::vector<int> C_BlockVer_offset;
  std::vector<int> C_BlockBdy_num;
  std::vector<int> C_BlockBdy_offset;
  int32_t max_subgraph_vertexs = 0;

 private:
  struct LoadedTag {};
  fapGraph(LoadedTag, int32_t n, int64_t m, std::vector<int32_t> ro, std::vector<int32_t> cv,
           std::vector<float> w, int32_t K, bool directed, bool weighted, std::vector<int32_t> gid);
  // GPU state
  fap_ctx *ctx_ = nullptr;
  fap_dgraph *dg_ = nullptr;
  int device_ = 0;
  int dtype_ = -1;  // FAP_DTYPE_AUTO
  SolveMode mode_ = SolveMode::Batched;
  bool prepared_ = false;
  bool partition_injected_ = false;

  void init_storage();
  void ensure_device();
  bool path_ready_ = false;  // `path` holds every part's predecessors

  int64_t row_limit_ = 0;     // setMaxResidentRows
  bool cache_tried_ = false;  // the resident cache was attempted for grouped solves

  void run_parts(const std::vector<int32_t> &ids);
  int solve_all(int mode);
  int64_t reserve_group_rows(int64_t need);
  int32_t run_group(int32_t first, int64_t rows);
  void copy_block(int32_t id, float *dst);
  void copy_path_block(int32_t id, int32_t *dst);
  void set_paths(bool on);

 public:
  int32_t num_vertexs = 0;
  int32_t num_edges = 0;
  std::vector<int32_t> adj_size;
  std::vector<int32_t> row_offset;
  std::vector<int32_t> col_val;
  std::vector<float> weight;
  bool directed = false;
  bool weighted = false;

  // Reads graph/<kind>/<input_graph>.mtx relative to the working directory
  // and partitions it into K parts with METIS (fap/fap.cpp:27-59).
  fapGraph(std::string input_graph, bool directed, bool weight, int32_t K);
  // Builds the graph from a CSR (row_offset[n+1], col_val[m], weight[m]) and
  // partitions it with METIS as an undirected graph.
  fapGraph(int32_t num_vertexs, int64_t num_edges, std::vector<int32_t> row_offset,
           std::vector<int32_t> col_val, std::vector<float> weight, int32_t K);
  // Same, for a directed CSR.
  fapGraph(int32_t num_vertexs, int64_t num_edges, std::vector<int32_t> row_offset,
           std::vector<int32_t> col_val, std::vector<float> weight, int32_t K, bool directed);
  ~fapGraph();
  // Binary graph file (CSR + partition): saveBinary writes what the
  // constructor built (the graph and its METIS or injected partition);
  // loadBinary rebuilds the graph without parsing text or running METIS,
  // ready for preCondition.  A checksum guards the file; a bad file raises
  // fapError (FAP_ERR_IO).
  void saveBinary(const std::string &path) const;
  static std::unique_ptr<fapGraph> loadBinary(const std::string &path);
  fapGraph(const fapGraph &) = delete;
  fapGraph &operator=(const fapGraph &) = delete;

  // Replaces the METIS partition by a given one (1-based part per vertex),
  // before preCondition.  Lets two implementations share one partition.
  void setPartition(const std::vector<int32_t> &graph_id_1based);
  // GPU options: device ordinal, distance type (FAP_DTYPE_*), solve form.
  void setDevice(int device);
  void setDtype(int dtype);
  void setMode(SolveMode mode);
  SolveMode getMode() const { return mode_; }
  // Bounds the output rows held on the device (0 = no bound): solve and
  // solveSubGraph then run the parts in groups whose rows fit, as they do
  // when HBM cannot hold all n rows.
  void setMaxResidentRows(int64_t rows);
  int getDtype();

  void preCondition();
  bool isSplit();
  std::vector<int> getGraphId();

  // Solves every part into getAllDistance(); 0 on success.
  int32_t solve(bool is_path_needed = false);
  // Solves one part (1-based) into getSubGraphDistance(); 0 on success.
  int32_t solveSubGraph(int32_t sub_garph_id, bool is_path_needed = false);

  std::vector<int32_t> getMapping();
  std::vector<float> getAllDistance();
  std::vector<int32_t> getAllPath();
  int32_t getCurrentSubGraphId();
  std::vector<int32_t> getSubGraphIndex(int32_t sub_garph_id);
  std::vector<float> getSubGraphDistance(int32_t sub_garph_id);
  std::vector<int32_t> getSubGraphPath(int32_t sub_garph_id);
  std::vector<float> getDistanceFromOnePoint(int32_t vectex_id);
  std::vector<int32_t> getPathFromOnePoint(int32_t vectex_id);
  float getDistanceP2P(int32_t from, int32_t to);
  std::vector<int32_t> getPathP2P(int32_t from, int32_t to);
  // The reference's argument-free declarations (fap/fap.h:116-119), kept so
  // that its callers compile; with no endpoints there is nothing to answer,
  // so they throw fapError(FAP_ERR_INVALID) (the reference's bodies are
  // empty TODOs that return nothing, fap/fap.cpp:263-269).
  float getDistanceP2P();
  std::vector<int32_t> getPathP2P();

  // Per-part counts after preCondition (index 1..K).
  const std::vector<int> &getBlockVerNum() const { return C_BlockVer_num; }
  const std::vector<int> &getBlockVerOffset() const { return C_BlockVer_offset; }
  const std::vector<int> &getBlockBdyNum() const { return C_BlockBdy_num; }
  int32_t getK() const { return K; }
  fap_dgraph *deviceGraph() { return dg_; }

  // Sampled self-check (fap/utils/checkResult.h:38-82): 20 random rows x 10
  // random columns of `dist` (rows = source[]) against shortest-path rows
  // recomputed by the GPU SSSP stage; |diff| <= 1e-5 or both unreachable.
  bool check_result(float *dist, int *path, int *source, int source_num, int vertexs,
                    int *adj_size, int *row_offset, int *col_val, float *weight, int *graph_id);
};

}  // namespace fap

#endif  // FAP_B200_FAP_H_
