// C ABI of the per-subgraph solve path: device-resident graph state and the
// per-part pipeline (reference fapGraph::run, fap/fap.cpp:92-181), in a plain
// (one launch sequence per part) and a batched (one launch per stage for all
// requested parts) form.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <exception>
#include <new>
#include <string>
#include <vector>

#include "fap_b200.h"
#include "fap_common.cuh"
#include "fap_internal.h"

using namespace fapb;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

// No C++ exception leaves an entry point of the C ABI: the host-side
// std::vector / std::string allocations turn into FAP_ERR_NOMEM.
int fail_exception() {
  try {
    throw;
  } catch (const std::bad_alloc &) {
    return fail(FAP_ERR_NOMEM, "host allocation failed");
  } catch (const std::exception &e) {
    return fail(FAP_ERR_INVALID, "%s", e.what());
  } catch (...) {
    return fail(FAP_ERR_INVALID, "unknown C++ exception");
  }
}

#define FAP_CK(call)                                                                     \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      if (e_ == cudaErrorMemoryAllocation) {                                             \
        cudaGetLastError();                                                              \
        return fail(FAP_ERR_NOMEM, "%s: %s", #call, cudaGetErrorString(e_));             \
      }                                                                                  \
      return fail(FAP_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));                \
    }                                                                                    \
  } while (0)

#define FAP_TRY(expr)         \
  do {                        \
    int r_ = (expr);          \
    if (r_ != FAP_OK) return r_; \
  } while (0)

// Records ev on st; inside a stream capture the record becomes an event node
// of the graph, so the host can still time the replayed stages.
cudaError_t record_event(cudaEvent_t ev, cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) cs = cudaStreamCaptureStatusNone;
  return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal)
                                             : cudaEventRecord(ev, st);
}

// Bytes a DevBuf allocates for `want`: small buffers (descriptors, source
// lists) grow to the next power of two, so that batches of changing
// composition rarely reallocate (each cudaFree synchronises the device).
size_t alloc_size(size_t want) {
  if (want == 0 || want > (size_t(64) << 20)) return want;
  size_t r = 4096;
  while (r < want) r <<= 1;
  return r;
}

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  int ensure(size_t want) {
    if (want <= bytes) return FAP_OK;
    want = alloc_size(want);
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    if (want == 0) return FAP_OK;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      return fail(FAP_ERR_NOMEM, "cudaMalloc(%zu bytes): %s", want, cudaGetErrorString(e));
    }
    bytes = want;
    return FAP_OK;
  }
  // Stream-ordered growth for buffers used on one stream only: the old
  // buffer is freed after the stream's earlier work, and nothing waits for
  // the rest of the device (cudaFree would).  release() works on either kind.
  int ensure_async(size_t want, cudaStream_t st) {
    if (want <= bytes) return FAP_OK;
    want = alloc_size(want);
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    bytes = 0;
    if (want == 0) return FAP_OK;
    cudaError_t e = cudaMallocAsync(&p, want, st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      return fail(FAP_ERR_NOMEM, "cudaMallocAsync(%zu bytes): %s", want, cudaGetErrorString(e));
    }
    bytes = want;
    return FAP_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <typename T>
  T *as() const { return reinterpret_cast<T *>(p); }
};

// RAII: make the context's device current for the duration of a call.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace

struct fap_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t own = nullptr;
  cudaEvent_t ev[6] = {};
  DevBuf scratch;     // fap_op_floyd padding copy
  DevBuf status;      // int device status for device-pointer ops
  DevBuf sink;        // microbenchmark sink
  int64_t launches = 0;
  int graphs = 0;             // live fap_dgraph objects created on this context
  bool destroy_pending = false;  // fap_ctx_destroy called while graphs were live
};

// Device copy of a FloydQueue item list (see fap_internal.h) and its
// counters.  Items: for every pivot block kb, the Floyd-1 items of all parts
// that have block kb, then their Floyd-2 items, then their Floyd-3 items;
// after all Floyd items the boundary-row scatter items of every part
// (nfloyd Floyd items, nitems in all).
struct QueueBuf {
  DevBuf items, cnt;
  int32_t nfloyd = 0, nitems = 0, stride = 2, nparts = 0;
  bool sym = false;
};

namespace {
// Items of the Floyd work queue.  sym: the matrices are symmetric; the panel
// items are the row panel's tiles only (each also stores its transpose into
// the column panel) and the remainder items the tiles (i, j) with i <= j
// (each off-diagonal one also stores its transpose into (j, i)); t holds
// i << 16 | j for those.  Per pivot block: every part's diagonal item, then
// every part's panel items, then every part's remainder items, so every
// dependency of an item (per part: Floyd-1 of block kb after every Floyd-3
// item of block kb - 1, Floyd-2 after Floyd-1, Floyd-3 after every Floyd-2
// of the block) comes earlier in the list.  The boundary-row scatter items
// follow all Floyd items.
std::vector<QItem> floyd_queue_items(const std::vector<PartDesc> &parts, bool sym, int32_t *nfloyd,
                                     int32_t *max_nb) {
  std::vector<QItem> it;
  int mnb = 0;
  for (const PartDesc &d : parts) mnb = std::max<int>(mnb, (int)ceil_div(std::max(d.s, 1), kFloydTile));
  for (int kb = 0; kb < mnb; kb++) {
    for (size_t p = 0; p < parts.size(); p++) {
      const int nb = (int)ceil_div(parts[p].s, kFloydTile);
      if (kb < nb) it.push_back(QItem{kQFloyd1, (int32_t)p, kb, 0});
    }
    for (size_t p = 0; p < parts.size(); p++) {
      const int nb = (int)ceil_div(parts[p].s, kFloydTile);
      if (kb >= nb) continue;
      if (sym) {
        for (int j = 0; j < nb; j++)
          if (j != kb) it.push_back(QItem{kQFloyd2S, (int32_t)p, kb, (kb << 16) | j});
      } else {
        for (int t = 0; t < 2 * (nb - 1); t++) it.push_back(QItem{kQFloyd2, (int32_t)p, kb, t});
      }
    }
    for (size_t p = 0; p < parts.size(); p++) {
      const int nb = (int)ceil_div(parts[p].s, kFloydTile);
      if (kb >= nb) continue;
      if (sym) {
        for (int i = 0; i < nb; i++)
          for (int j = i; j < nb; j++)
            if (i != kb && j != kb) it.push_back(QItem{kQFloyd3S, (int32_t)p, kb, (i << 16) | j});
      } else {
        for (int t = 0; t < (nb - 1) * (nb - 1); t++) it.push_back(QItem{kQFloyd3, (int32_t)p, kb, t});
      }
    }
  }
  *nfloyd = (int32_t)it.size();
  for (size_t p = 0; p < parts.size(); p++)
    for (int r = 0; r < parts[p].b; r += kQScatterRows) it.push_back(QItem{kQScatter, (int32_t)p, r, 0});
  *max_nb = mnb;
  return it;
}

// Whether every item's dependencies come before it in `it` and every Floyd
// item of the parts appears exactly once (the queue's waits end only then).
bool queue_order_ok(const std::vector<PartDesc> &parts, bool sym, const std::vector<QItem> &it, int32_t nfloyd) {
  const int np = (int)parts.size();
  std::vector<std::vector<int>> c1(np), c2(np), c3(np);
  std::vector<int> nbs(np);
  size_t want = 0;
  for (int p = 0; p < np; p++) {
    const int nb = parts[p].s > 0 ? (int)ceil_div(parts[p].s, kFloydTile) : 0;
    nbs[p] = nb;
    c1[p].assign(nb, 0);
    c2[p].assign(nb, 0);
    c3[p].assign(nb, 0);
    want += nb * (1 + (sym ? nb - 1 : 2 * (nb - 1)) + (sym ? (size_t)(nb - 1) * nb / 2 : (size_t)(nb - 1) * (nb - 1)));
  }
  if ((size_t)nfloyd != want) return false;
  std::vector<uint64_t> keys;
  keys.reserve(nfloyd);
  for (int32_t x = 0; x < nfloyd; x++) {
    const QItem &q = it[x];
    if (q.pidx < 0 || q.pidx >= np || q.kb < 0 || q.kb >= nbs[q.pidx]) return false;
    const int p = q.pidx, nb = nbs[p], kb = q.kb;
    const int n2 = sym ? nb - 1 : 2 * (nb - 1), n3 = sym ? (nb - 1) * nb / 2 : (nb - 1) * (nb - 1);
    int ph;
    if (q.kind == kQFloyd1) {
      if (kb > 0 && c3[p][kb - 1] != n3) return false;
      ph = 0;
      c1[p][kb]++;
    } else if (q.kind == (sym ? kQFloyd2S : kQFloyd2)) {
      if (c1[p][kb] != 1) return false;
      ph = 1;
      c2[p][kb]++;
    } else if (q.kind == (sym ? kQFloyd3S : kQFloyd3)) {
      if (c2[p][kb] != n2) return false;
      ph = 2;
      c3[p][kb]++;
    } else {
      return false;
    }
    if (q.t < 0) return false;
    keys.push_back(((((uint64_t)p << 8 | (uint64_t)kb) * 3 + ph) << 32) | (uint32_t)q.t);
  }
  std::sort(keys.begin(), keys.end());
  return std::adjacent_find(keys.begin(), keys.end()) == keys.end();
}

}  // namespace

struct fap_dgraph {
  fap_ctx *ctx = nullptr;
  int32_t n = 0;
  int64_t m = 0;
  int dtype = FAP_DTYPE_F32;
  DevBuf ro, col, w;
  std::vector<int32_t> h_ro, h_col;
  std::vector<uint32_t> h_w;      // weight bits as uploaded (int32 or float)
  double mean_w = 1.0;
  // CSR relabelled into sorted-position order (SSSP work space)
  DevBuf ro_s, col_s, w_s, sssp_scratch;
  // partition
  int32_t K = 0;
  std::vector<int32_t> gid, st2ed, ed2st, vnum, voff, bnum;
  DevBuf d_gid, d_st2ed, d_ed2st;
  // output
  int64_t ldD = 0;
  int64_t max_rows = 0;
  int64_t row_limit = 0;  // "max_resident_rows": bound on max_rows, 0 = none
  DevBuf D;
  std::vector<int64_t> row_base;  // per part (1..K), -1 = not resident
  // batch state
  DevBuf F, d_parts, d_work, d_src, d_srcrows, d_status, d_checks, staging;
  // Asynchronous block copies (fap_graph_copy_block_async): per slot a
  // float32 staging buffer, the stream its device-to-host copy runs on and
  // the events that order it (conversion done on the context stream, copy
  // done), so that the next block's conversion overlaps this one's copy.
  struct CopySlot {
    DevBuf staging;
    cudaStream_t stream = nullptr;
    cudaEvent_t converted = nullptr, done = nullptr;
    bool busy = false;
  };
  CopySlot cslot[FAP_COPY_SLOTS];
  std::vector<PartDesc> parts;
  std::vector<MPWork> work;
  std::vector<int32_t> src;
  std::vector<int64_t> srcrows;
  std::vector<int32_t> part_src_off;                 // per batch index, size nparts+1
  std::vector<int32_t> part_work_begin, part_work_end;  // per batch index, into work (thick parts)
  std::vector<int32_t> thin;      // batch indices of thin-boundary parts
  std::vector<int32_t> thin_pos;  // per batch index: position in thin, or -1
  DevBuf d_thin;
  std::vector<int32_t> last_ids;
  bool last_cached = false;  // last_ids' descriptors point into the resident cache
  int64_t f_elems = 0;
  int max_ldf = 0, max_b = 0, max_s = 0;
  // tuning
  double sssp_delta = -1.0;  // <0: automatic
  int64_t sssp_max_rounds = -1;  // <0: 8n + 1024
  bool floyd_per_cta = false;     // batched Floyd: one CTA per part instead of per-tile launches
  int sssp_chain = 0;             // SSSP chain-following budget (hops per thread per round)
  int sssp_precheck = 1;          // SSSP: plain read of dist[v] before the atomicMin
  // Min-plus tiles in the packed 16-bit form where the distances provably
  // fit (int32 graphs; Pack16): bounds buffers of the prepared batch.
  bool pack16 = true;
  DevBuf d_pk_off, d_pk_range, d_pk_maxa, d_pk_tiles;
  // ... with the operands packed beforehand (Pack16::s16 / at) when they fit
  // in kPrepackBytes and a quarter of the free device memory (parameter
  // "minplus_prepack"); pk_krow: their first row per batch part
  bool prepack = true;
  DevBuf d_pk_s16, d_pk_at, d_pk_krow;
  std::vector<int32_t> pk_krow;
  // the same for the tiled expansion of the boundary graph (Expand16), sized
  // for the launch's part list
  DevBuf d_xk_off, d_xk_range, d_xk_maxb, d_xk_tiles, d_xk_ap, d_xk_bd;
  // Work queue of the batched Floyd (FloydQueue): the batch's items and
  // counters, and the resident cache build's (its parts are all parts).
  // Parts with at most this many boundary vertices (<= kThinBoundary) take
  // the store-shaped thin min-plus kernel, the others the register-tiled
  // one (parameter "thin_max_b", tuned with the solve form).
  int thin_max_b = kThinBoundary;
  bool floyd_queue = true;
  bool floyd_sym = true;  // use sym_local in the queue (parameter "floyd_symmetric")
  QueueBuf q, cq;
  Pack16 pk{};
  // CUDA graph of the batched launch sequence (replayed while nothing that
  // it captured changes: batch, buffers, parameters, stream)
  bool use_graph = true;
  uint64_t epoch = 1;
  uint64_t direct_epoch = 0;  // epoch of the last batched solve launched directly (0: none)
  cudaGraphExec_t gexec = nullptr;
  uint64_t gexec_epoch = 0;
  cudaStream_t gexec_stream = nullptr;
  int64_t gexec_launches = 0;
  // Resident cache: the boundary rows of every part (cBd, rows in part order,
  // cb_off[p] = first row of part p) and every part's closed Floyd matrix
  // (cF, equal padded squares of side cache_ldf, part p at (p - 1)).
  bool cache_ready = false;
  bool use_cache = true;
  // Sharded boundary-graph form (fap_graph_shard_*): the rank's own parts
  // (ascending) and which cache slots hold finished parts (empty: all).
  std::vector<int32_t> shard_own;
  bool shard_begun = false;
  std::vector<char> cache_valid;
  DevBuf d_cown;
  // Boundary-graph form of stage 1 (see launch_bgraph): applicable when no
  // two arcs join the same ordered pair inside a part (the reference's
  // matrix build keeps the last of such duplicates, which the local closure
  // would not reproduce); boff = prefix sums of the boundary counts.
  int stage1 = 0;  // 0 auto, 1 SSSP, 2 boundary graph whenever applicable
  bool bnd_dupfree = false;
  // Every arc inside a part has its reverse with the same weight (and no
  // duplicates): each part's local closure is a symmetric matrix, so the
  // Floyd work queue computes only the tiles on and above the diagonal and
  // stores each one's transpose (floyd_queue_items, sym).
  bool sym_local = false;
  int64_t total_b = 0;
  std::vector<int32_t> boff;
  std::vector<int32_t> bpcol;  // boundary columns of dB padded per part to multiples of 4 (prefix sums)
  bool last_bmethod = false;   // the prepared batch uses it
  bool cache_bmethod = false;  // the resident cache was built with it
  int64_t ldB = 0;
  DevBuf d_dB, d_bpart, d_brows, d_FB;
  // Column table of the staged expansion (launch_bdy_expand): max_b x ldD
  // values for a prepared batch of all parts, when that is at most
  // kColTableBytes (resident-cache builds and larger tables: the expansion
  // gathers from F, so that a server's resident graphs hold no table).
  DevBuf d_bTc;
  int bTc_maxb = 0;
  // Large boundary sets: dB closed by Bellman-Ford in alternating local
  // (min-plus with the parts' local closures) and cross steps (the in-arc
  // CSR of the cross-part arcs over boundary indices, built once per
  // partition; gpart: part of every boundary index) and the boundary rows
  // written by the tiled expansion (grow: boundary index -> D row).
  std::string stage1_name, cache_stage1_name;  // fap_graph_stage1_name
  int bgraph_form = 0;        // 0 by size, 1 Floyd + staged expansion, 2 Bellman-Ford + tiled expansion
  int64_t bgraph_edges = 0;  // sum_p b_p (b_p - 1) + cross-part arcs
  int64_t bgraph_cross = 0;  // cross-part arcs
  bool bg_csr_ready = false;
  DevBuf d_bitro, d_bitcol, d_botro, d_botcol, d_bitw;     // cross-arc CSRs (in with weights, out)
  DevBuf d_bitems, d_bDt, d_bact, d_bpact, d_bgpart, d_bpcolmap, d_grow;  // d_bitems: the two work lists
  // Tiled form of stage 1's SSSP (launch_msbf): 0 automatic (graphs with at
  // least 6 arcs per vertex, where few Bellman-Ford iterations suffice), 1
  // frontier kernel, 2 tiled.  Work items over the in-edge CSR.
  int sssp_form = 0;
  // memory for tiles side by side (tiled SSSP, Bellman-Ford closure): more
  // than L2 holds, since an iteration touches only its changed rows, and
  // fewer groups of tiles mean fewer launches and convergence read-backs
  int64_t tile_bytes = int64_t(384) << 20;
  DevBuf d_msbf_items, d_msbf_act, d_msbf_changed;
  int msbf_nitems = 0;
  int *h_changed = nullptr;  // pinned, 4 ints
  // Predecessor matrices: P has D's shape; the in-edge CSR (tro/tcol/tw)
  // is built when paths are switched on; path_ok[p]: p's resident block has
  // its predecessor rows.
  bool paths = false;
  DevBuf P, d_tro, d_tcol, d_tw;
  std::vector<char> path_ok;
  DevBuf cBd, cF, d_cparts, d_rowgroups, d_rowloc, d_rowout, d_rowidx;
  std::vector<int64_t> cb_off;
  std::vector<PartDesc> cparts;
  cudaEvent_t cev[5] = {};                  // phases of the last cache build
  float cache_ms[4] = {-1, -1, -1, -1};     // fap_graph_cache_timing
  int cache_ldf = 0, cache_max_b = 0, cache_max_s = 0;
  // last solve
  int last_mode = -1;
  float timing[5] = {-1, -1, -1, -1, -1};
  int64_t launches = 0;
};

// ---------------------------------------------------------------------------
// misc
// ---------------------------------------------------------------------------
extern "C" const char *fap_last_error(void) { return g_err.c_str(); }
extern "C" int fap_version(void) { return 0x000100; }

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
extern "C" int fap_ctx_create(int device, fap_ctx **out) try {
  if (!out) return fail(FAP_ERR_INVALID, "fap_ctx_create: out is NULL");
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(FAP_ERR_CUDA, "no CUDA device available (%s)", cudaGetErrorString(e));
  }
  if (device < 0 || device >= count) return fail(FAP_ERR_INVALID, "device %d out of range", device);
  DeviceGuard g(device);
  fap_ctx *c = new fap_ctx();
  c->device = device;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
    delete c;
    return fail(FAP_ERR_CUDA, "cudaGetDeviceProperties failed");
  }
  if (prop.major < 10) {
    delete c;
    return fail(FAP_ERR_CUDA, "device %d is sm_%d%d; this library is built for sm_100a", device,
                prop.major, prop.minor);
  }
  c->sm_count = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return fail(FAP_ERR_CUDA, "cudaStreamCreate failed");
  }
  c->stream = c->own;
  for (auto &ev : c->ev) cudaEventCreate(&ev);
  if (c->status.ensure(sizeof(int)) != FAP_OK) {
    fap_ctx_destroy(c);
    return FAP_ERR_NOMEM;
  }
  *out = c;
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

namespace {
void ctx_release(fap_ctx *c) {
  DeviceGuard g(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  c->scratch.release();
  c->status.release();
  c->sink.release();
  for (auto &ev : c->ev)
    if (ev) cudaEventDestroy(ev);
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
}
}  // namespace

// A context outlives its graphs: with graphs still alive the release is
// deferred until the last of them is destroyed, so callers (and garbage
// collectors) may destroy the two in either order.
extern "C" int fap_ctx_destroy(fap_ctx *c) try {
  if (!c) return FAP_OK;
  if (c->graphs > 0) {
    c->destroy_pending = true;
    return FAP_OK;
  }
  ctx_release(c);
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_ctx_set_stream(fap_ctx *c, void *stream) try {
  if (!c) return fail(FAP_ERR_INVALID, "ctx is NULL");
  c->stream = stream ? reinterpret_cast<cudaStream_t>(stream) : c->own;
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_ctx_get_stream(fap_ctx *c, void **stream) try {
  if (!c || !stream) return fail(FAP_ERR_INVALID, "NULL argument");
  *stream = reinterpret_cast<void *>(c->stream);
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_ctx_sync(fap_ctx *c) try {
  if (!c) return fail(FAP_ERR_INVALID, "ctx is NULL");
  DeviceGuard g(c->device);
  FAP_CK(cudaStreamSynchronize(c->stream));
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

// ---------------------------------------------------------------------------
// graph
// ---------------------------------------------------------------------------
extern "C" int fap_graph_create(fap_ctx *ctx, int32_t n, int64_t m, const int32_t *row_offset,
                                const int32_t *col_val, const float *weight, int dtype,
                                fap_dgraph **out) try {
  if (!ctx || !out) return fail(FAP_ERR_INVALID, "NULL argument");
  *out = nullptr;
  if (n <= 0) return fail(FAP_ERR_INVALID, "n must be positive (got %d)", n);
  if (m < 0 || (m > 0 && (!col_val || !weight)) || !row_offset)
    return fail(FAP_ERR_INVALID, "bad CSR arguments");
  if (m > INT32_MAX) return fail(FAP_ERR_INVALID, "m exceeds int32 edge indexing");
  if (row_offset[0] != 0) return fail(FAP_ERR_INVALID, "row_offset[0] must be 0");
  for (int32_t v = 0; v < n; v++)
    if (row_offset[v + 1] < row_offset[v]) return fail(FAP_ERR_INVALID, "row_offset not monotone at %d", v);
  const int64_t used = row_offset[n];
  if (used > m) return fail(FAP_ERR_INVALID, "row_offset[n]=%lld exceeds m=%lld", (long long)used, (long long)m);
  bool integral = true;
  for (int64_t e = 0; e < used; e++) {
    if (col_val[e] < 0 || col_val[e] >= n)
      return fail(FAP_ERR_INVALID, "col_val[%lld]=%d out of range", (long long)e, col_val[e]);
    const float x = weight[e];
    if (!(x >= 0.0f) || !std::isfinite(x))
      return fail(FAP_ERR_INVALID, "weight[%lld] must be finite and non-negative", (long long)e);
    if (x != std::floor(x) || x > (float)FAP_MAX_INT_WEIGHT) integral = false;
  }
  int dt = dtype;
  if (dt == FAP_DTYPE_AUTO) dt = integral ? FAP_DTYPE_I32 : FAP_DTYPE_F32;
  if (dt == FAP_DTYPE_I32 && !integral)
    return fail(FAP_ERR_RANGE, "int32 distances need integral weights <= %d", FAP_MAX_INT_WEIGHT);
  if (dt != FAP_DTYPE_I32 && dt != FAP_DTYPE_F32) return fail(FAP_ERR_INVALID, "bad dtype %d", dtype);

  DeviceGuard g(ctx->device);
  fap_dgraph *G = new fap_dgraph();
  G->ctx = ctx;
  ctx->graphs++;
  G->n = n;
  G->m = used;
  G->dtype = dt;
  G->ldD = round_up(n, kLdAlign);
  auto cleanup = [&](int rc) {
    fap_graph_destroy(G);
    return rc;
  };
  int rc;
  if ((rc = G->ro.ensure((size_t)(n + 1) * 4)) != FAP_OK) return cleanup(rc);
  if ((rc = G->col.ensure((size_t)std::max<int64_t>(used, 1) * 4)) != FAP_OK) return cleanup(rc);
  if ((rc = G->w.ensure((size_t)std::max<int64_t>(used, 1) * 4)) != FAP_OK) return cleanup(rc);
  cudaError_t e = cudaMemcpy(G->ro.p, row_offset, (size_t)(n + 1) * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && used > 0)
    e = cudaMemcpy(G->col.p, col_val, (size_t)used * 4, cudaMemcpyHostToDevice);
  G->h_ro.assign(row_offset, row_offset + n + 1);
  G->h_col.assign(col_val, col_val + used);
  G->h_w.resize((size_t)used);
  double wsum = 0.0;
  for (int64_t i = 0; i < used; i++) {
    wsum += weight[i];
    if (dt == FAP_DTYPE_I32) {
      const int32_t wi = (int32_t)weight[i];
      std::memcpy(&G->h_w[i], &wi, 4);
    } else {
      std::memcpy(&G->h_w[i], &weight[i], 4);
    }
  }
  G->mean_w = used > 0 ? std::max(wsum / (double)used, 1e-30) : 1.0;
  if (e == cudaSuccess && used > 0)
    e = cudaMemcpy(G->w.p, G->h_w.data(), (size_t)used * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cleanup(fail(FAP_ERR_CUDA, "CSR upload: %s", cudaGetErrorString(e)));
  if ((rc = G->d_status.ensure(sizeof(int))) != FAP_OK) return cleanup(rc);
  cudaMemset(G->d_status.p, 0, sizeof(int));
  *out = G;
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

namespace {
void cache_drop(fap_dgraph *G) {
  for (DevBuf *b : {&G->cBd, &G->cF, &G->d_cparts, &G->d_rowgroups, &G->d_rowloc, &G->d_rowout,
                    &G->d_rowidx})
    b->release();
  G->cache_ready = false;
  G->cache_valid.clear();
  G->shard_begun = false;
  G->cb_off.clear();
  G->cparts.clear();
  G->last_ids.clear();
  G->epoch++;
}
}  // namespace

extern "C" int fap_graph_destroy(fap_dgraph *G) try {
  if (!G) return FAP_OK;
  fap_ctx *c = G->ctx;
  {
    DeviceGuard g(c->device);
    cudaStreamSynchronize(c->stream);
    if (G->gexec) cudaGraphExecDestroy(G->gexec);
    for (DevBuf *b : {&G->ro, &G->col, &G->w, &G->ro_s, &G->col_s, &G->w_s, &G->sssp_scratch, &G->d_thin,
                      &G->d_gid, &G->d_st2ed, &G->d_ed2st, &G->D, &G->F, &G->d_parts, &G->d_work,
                      &G->d_src, &G->d_srcrows, &G->d_status, &G->d_checks, &G->staging, &G->P,
                      &G->d_tro, &G->d_tcol, &G->d_tw, &G->d_dB, &G->d_bpart, &G->d_brows, &G->d_FB,
                      &G->d_msbf_items, &G->d_msbf_act, &G->d_msbf_changed, &G->d_bitro, &G->d_bitcol,
                      &G->d_botro, &G->d_botcol, &G->d_bitw, &G->d_bitems, &G->d_bDt, &G->d_bact, &G->d_bpact,
                      &G->d_bgpart, &G->d_bpcolmap, &G->d_grow, &G->d_pk_off, &G->d_pk_range,
                      &G->d_pk_s16, &G->d_pk_at, &G->d_pk_krow, &G->d_pk_maxa, &G->d_pk_tiles, &G->q.items, &G->q.cnt, &G->cq.items, &G->cq.cnt,
                      &G->d_xk_off, &G->d_xk_range, &G->d_xk_maxb, &G->d_xk_tiles, &G->d_bTc,
                      &G->d_xk_ap, &G->d_xk_bd})
      b->release();
    if (G->h_changed) cudaFreeHost(G->h_changed);
    for (auto &cs : G->cslot) {
      if (cs.stream) cudaStreamSynchronize(cs.stream);
      cs.staging.release();
      if (cs.converted) cudaEventDestroy(cs.converted);
      if (cs.done) cudaEventDestroy(cs.done);
      if (cs.stream) cudaStreamDestroy(cs.stream);
    }
    for (cudaEvent_t &ev : G->cev)
      if (ev) cudaEventDestroy(ev);
    cache_drop(G);
  }
  delete G;
  c->graphs--;
  if (c->destroy_pending && c->graphs == 0) ctx_release(c);
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_dtype(const fap_dgraph *G) { return G ? G->dtype : FAP_ERR_INVALID; }

extern "C" int fap_graph_set_parts(fap_dgraph *G, int32_t K, const int32_t *graph_id,
                                   const int32_t *st2ed, const int32_t *ver_num,
                                   const int32_t *ver_offset, const int32_t *bdy_num) try {
  if (!G || !graph_id || !st2ed || !ver_num || !ver_offset || !bdy_num)
    return fail(FAP_ERR_INVALID, "NULL argument");
  const int32_t n = G->n;
  if (K < 1 || K > n) return fail(FAP_ERR_PARTITION, "K=%d must be in [1, n=%d]", K, n);
  std::vector<int32_t> ed2st(n, -1);
  for (int32_t i = 0; i < n; i++) {
    const int32_t v = st2ed[i];
    if (v < 0 || v >= n || ed2st[v] != -1) return fail(FAP_ERR_PARTITION, "st2ed is not a permutation");
    ed2st[v] = i;
    if (graph_id[v] < 1 || graph_id[v] > K)
      return fail(FAP_ERR_PARTITION, "graph_id[%d]=%d outside 1..K", v, graph_id[v]);
  }
  int64_t off = 0;
  for (int32_t p = 1; p <= K; p++) {
    if (ver_offset[p] != off) return fail(FAP_ERR_PARTITION, "ver_offset[%d] inconsistent", p);
    if (ver_num[p] < 0 || bdy_num[p] < 0 || bdy_num[p] > ver_num[p])
      return fail(FAP_ERR_PARTITION, "part %d counts inconsistent", p);
    for (int32_t i = 0; i < ver_num[p]; i++)
      if (graph_id[st2ed[off + i]] != p) return fail(FAP_ERR_PARTITION, "part %d block holds a foreign vertex", p);
    off += ver_num[p];
  }
  if (off != n) return fail(FAP_ERR_PARTITION, "part sizes sum to %lld, not n", (long long)off);
  // Both ends of every cross-part arc are boundary vertices
  // (fap/utils/util_preprocess.h:32-59), i.e. sit in the first bdy_num[p]
  // places of their part's block; every stage relies on it.
  for (int32_t u = 0; u < n; u++)
    for (int32_t e = G->h_ro[u]; e < G->h_ro[u + 1]; e++) {
      const int32_t v = G->h_col[e];
      const int32_t pu = graph_id[u], pv = graph_id[v];
      if (pu == pv) continue;
      if (ed2st[u] - ver_offset[pu] >= bdy_num[pu] || ed2st[v] - ver_offset[pv] >= bdy_num[pv])
        return fail(FAP_ERR_PARTITION, "arc %d->%d crosses parts but an end is not in its part's boundary block",
                    u, v);
    }
  DeviceGuard g(G->ctx->device);
  // The graph has no parts until every step below has succeeded: a failure
  // part-way (an allocation, a copy) leaves K = 0, so a later solve is
  // refused instead of reading half-updated tables.
  G->K = 0;
  G->gid.assign(graph_id, graph_id + n);
  G->st2ed.assign(st2ed, st2ed + n);
  G->ed2st = std::move(ed2st);
  G->vnum.assign(ver_num, ver_num + K + 1);
  G->voff.assign(ver_offset, ver_offset + K + 1);
  G->bnum.assign(bdy_num, bdy_num + K + 1);
  G->boff.assign(K + 2, 0);
  for (int32_t p = 1; p <= K; p++) G->boff[p + 1] = G->boff[p] + bdy_num[p];
  G->total_b = G->boff[K + 1];
  G->bpcol.assign(K + 2, 0);
  for (int32_t p = 1; p <= K; p++) G->bpcol[p + 1] = G->bpcol[p] + (int32_t)round_up(bdy_num[p], 4);
  {
    // duplicate arcs inside a part?
    G->bnd_dupfree = true;
    std::vector<int32_t> seen((size_t)n, -1);
    for (int32_t u = 0; u < n && G->bnd_dupfree; u++)
      for (int32_t e = G->h_ro[u]; e < G->h_ro[u + 1]; e++) {
        const int32_t v = G->h_col[e];
        if (graph_id[v] != graph_id[u]) continue;
        if (seen[v] == u) {
          G->bnd_dupfree = false;
          break;
        }
        seen[v] = u;
      }
  }
  {
    // symmetric parts: the intra-part arcs of every row sorted by head, and
    // each arc's reverse looked up in its head's row (no two intra-part arcs
    // join the same ordered pair, so the reverse is unique)
    G->sym_local = false;
    if (G->bnd_dupfree) {
      std::vector<int64_t> sro((size_t)n + 1, 0);
      for (int32_t u = 0; u < n; u++) {
        int64_t c = 0;
        for (int32_t e = G->h_ro[u]; e < G->h_ro[u + 1]; e++) {
          const int32_t v = G->h_col[e];
          c += graph_id[v] == graph_id[u] && v != u;
        }
        sro[u + 1] = sro[u] + c;
      }
      std::vector<std::pair<int32_t, uint32_t>> arcs((size_t)sro[n]);
      for (int32_t u = 0; u < n; u++) {
        int64_t pos = sro[u];
        for (int32_t e = G->h_ro[u]; e < G->h_ro[u + 1]; e++) {
          const int32_t v = G->h_col[e];
          if (graph_id[v] == graph_id[u] && v != u) arcs[(size_t)pos++] = {v, G->h_w[e]};
        }
        std::sort(arcs.begin() + sro[u], arcs.begin() + sro[u + 1]);
      }
      bool sym = true;
      for (int32_t u = 0; u < n && sym; u++)
        for (int64_t i = sro[u]; i < sro[u + 1] && sym; i++) {
          const int32_t v = arcs[(size_t)i].first;
          const auto b = arcs.begin() + sro[v], e = arcs.begin() + sro[v + 1];
          const auto it = std::lower_bound(b, e, std::make_pair(u, (uint32_t)0));
          sym = it != e && it->first == u && it->second == arcs[(size_t)i].second;
        }
      G->sym_local = sym;
    }
  }
  {
    // edges of the boundary graph
    int64_t cross = 0;
    for (int32_t u = 0; u < n; u++)
      for (int32_t e = G->h_ro[u]; e < G->h_ro[u + 1]; e++) cross += graph_id[G->h_col[e]] != graph_id[u];
    G->bgraph_cross = cross;
    G->bgraph_edges = cross;
    for (int32_t p = 1; p <= K; p++) G->bgraph_edges += (int64_t)bdy_num[p] * std::max(bdy_num[p] - 1, 0);
    G->bg_csr_ready = false;
  }
  G->row_base.assign(K + 1, -1);
  G->last_ids.clear();
  cache_drop(G);
  FAP_TRY(G->d_gid.ensure((size_t)n * 4));
  FAP_TRY(G->d_st2ed.ensure((size_t)n * 4));
  FAP_TRY(G->d_ed2st.ensure((size_t)n * 4));
  FAP_CK(cudaMemcpy(G->d_gid.p, G->gid.data(), (size_t)n * 4, cudaMemcpyHostToDevice));
  FAP_CK(cudaMemcpy(G->d_st2ed.p, G->st2ed.data(), (size_t)n * 4, cudaMemcpyHostToDevice));
  FAP_CK(cudaMemcpy(G->d_ed2st.p, G->ed2st.data(), (size_t)n * 4, cudaMemcpyHostToDevice));
  // SSSP work space: the CSR relabelled into sorted positions, so that
  // vertices of one part (geometrically compact) sit next to each other.
  const int64_t m = G->m;
  std::vector<int32_t> ro_s((size_t)n + 1, 0), col_s((size_t)std::max<int64_t>(m, 1));
  std::vector<uint32_t> w_s((size_t)std::max<int64_t>(m, 1));
  for (int32_t i = 0; i < n; i++) {
    const int32_t v = G->st2ed[i];
    ro_s[i + 1] = ro_s[i] + (G->h_ro[v + 1] - G->h_ro[v]);
    int32_t pos = ro_s[i];
    for (int32_t e = G->h_ro[v]; e < G->h_ro[v + 1]; e++, pos++) {
      col_s[pos] = G->ed2st[G->h_col[e]];
      w_s[pos] = G->h_w[e];
    }
  }
  FAP_TRY(G->ro_s.ensure((size_t)(n + 1) * 4));
  FAP_TRY(G->col_s.ensure(col_s.size() * 4));
  FAP_TRY(G->w_s.ensure(w_s.size() * 4));
  FAP_CK(cudaMemcpy(G->ro_s.p, ro_s.data(), (size_t)(n + 1) * 4, cudaMemcpyHostToDevice));
  FAP_CK(cudaMemcpy(G->col_s.p, col_s.data(), col_s.size() * 4, cudaMemcpyHostToDevice));
  FAP_CK(cudaMemcpy(G->w_s.p, w_s.data(), w_s.size() * 4, cudaMemcpyHostToDevice));
  G->K = K;
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_reserve(fap_dgraph *G, int64_t max_rows) try {
  if (!G) return fail(FAP_ERR_INVALID, "NULL graph");
  if (G->row_limit > 0 && max_rows > G->row_limit)
    return fail(FAP_ERR_NOMEM, "%lld rows asked, at most %lld may be resident (\"max_resident_rows\")",
                (long long)max_rows, (long long)G->row_limit);
  if (max_rows <= 0 || max_rows > G->n) max_rows = G->n;
  if (G->row_limit > 0) max_rows = std::min(max_rows, G->row_limit);
  DeviceGuard g(G->ctx->device);
  cudaStreamSynchronize(G->ctx->stream);
  const size_t bytes = (size_t)max_rows * (size_t)G->ldD * 4;
  // No block is resident while the buffers change: a failed allocation
  // below leaves max_rows = 0 and no part placed, so the next solve
  // reserves again instead of writing through a released buffer.
  G->max_rows = 0;
  std::fill(G->row_base.begin(), G->row_base.end(), -1);
  G->last_ids.clear();
  G->epoch++;
  if (G->D.bytes < bytes) {
    G->D.release();
    FAP_TRY(G->D.ensure(bytes));
  }
  if (G->paths && G->P.bytes < bytes) {
    G->P.release();
    FAP_TRY(G->P.ensure(bytes));
  }
  G->max_rows = max_rows;
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

namespace {

// Boundary sets up to this size close dB by Floyd; larger ones by the tiled
// Bellman-Ford over the boundary graph (Floyd's cube grows too fast).
constexpr int64_t kBgraphFloydMax = 8192;
// The staged expansion keeps kExpandRows rows of dB in shared memory.
constexpr int64_t kBgraphStagedMax = 4096;
// Largest column table of the staged expansion (max_b x ldD values).
constexpr size_t kColTableBytes = size_t(256) << 20;
constexpr size_t kPrepackBytes = size_t(8) << 30;
// Automatic Bellman-Ford closure only while the boundary graph has at most
// this many edges per edge of the graph (its cliques grow as b_p^2) and dB
// stays within 64 Ki boundary vertices (17 GB).
constexpr int64_t kBgraphEdgeRatio = 8;
constexpr int64_t kBgraphAutoMaxB = 65536;

bool bgraph_bf(const fap_dgraph *G) {
  return G->bgraph_form == 2 || (G->bgraph_form == 0 && G->total_b > kBgraphFloydMax);
}
const char *stage1_form_name(const fap_dgraph *G, bool bmethod);

bool bgraph_tiled_expand(const fap_dgraph *G) { return G->bgraph_form == 2 || G->total_b > kBgraphStagedMax; }

// Whether the boundary-graph form of stage 1 applies to g.
// Automatic choice: int32 distances only (there both forms give the exact
// shortest distances bit for bit; float32 sums would round in a different
// order, a few ulps); up to 8192 boundary vertices with Floyd on the boundary
// graph, beyond that with the tiled Bellman-Ford while the boundary graph
// stays sparse (grid-like graphs with many parts).
bool bmethod_ok(const fap_dgraph *G) {
  if (G->stage1 == 1 || !G->bnd_dupfree || G->total_b <= 0) return false;
  if (bgraph_bf(G) && (G->bgraph_cross >= INT32_MAX || G->total_b >= INT32_MAX / kMsbfS)) return false;
  if (G->stage1 == 2) return true;
  if (G->dtype != FAP_DTYPE_I32) return false;
  return !bgraph_bf(G) ||
         (G->bgraph_edges <= kBgraphEdgeRatio * G->m && G->total_b <= kBgraphAutoMaxB);
}

// Tiles of the Bellman-Ford closure run side by side: as many as fit in
// tile_bytes, at most 16.
int bgraph_ztiles(const fap_dgraph *G) {
  const int64_t per = std::max<int64_t>(G->total_b, 1) * kMsbfS * 4;
  const int64_t tiles = ceil_div(std::max<int64_t>(G->total_b, 1), kMsbfS);
  return (int)std::max<int64_t>(1, std::min<int64_t>({G->tile_bytes / per, 16, tiles}));
}

// Cross-part arcs between boundary vertices (g = boff[p] + c for the c-th
// boundary vertex of part p) as two CSRs over boundary indices, in-arcs with
// their weights and out-arcs, and the part of every boundary index.
int build_bgraph_csr(fap_dgraph *G) {
  if (G->bg_csr_ready) return FAP_OK;
  const int64_t nb = G->total_b;
  auto bidx = [&](int32_t v) -> int64_t {
    const int32_t p = G->gid[v];
    const int32_t l = G->ed2st[v] - G->voff[p];
    return l < G->bnum[p] ? G->boff[p] + l : -1;
  };
  std::vector<int32_t> gpart((size_t)nb);
  for (int32_t p = 1; p <= G->K; p++)
    for (int32_t c = 0; c < G->bnum[p]; c++) gpart[G->boff[p] + c] = p;
  std::vector<int64_t> au, av;  // arcs (boundary indices) in CSR order
  std::vector<uint32_t> aw;
  for (int32_t u = 0; u < G->n; u++)
    for (int32_t e = G->h_ro[u]; e < G->h_ro[u + 1]; e++) {
      const int32_t v = G->h_col[e];
      if (G->gid[v] == G->gid[u]) continue;
      const int64_t gu = bidx(u), gv = bidx(v);
      if (gu < 0 || gv < 0) continue;
      au.push_back(gu);
      av.push_back(gv);
      aw.push_back(G->h_w[e]);
    }
  const size_t ne = au.size();
  std::vector<int32_t> itro((size_t)nb + 1, 0), otro((size_t)nb + 1, 0);
  for (size_t a = 0; a < ne; a++) {
    itro[av[a] + 1]++;
    otro[au[a] + 1]++;
  }
  for (int64_t g = 0; g < nb; g++) {
    itro[g + 1] += itro[g];
    otro[g + 1] += otro[g];
  }
  std::vector<int32_t> itcol(std::max<size_t>(ne, 1)), otcol(std::max<size_t>(ne, 1));
  std::vector<uint32_t> itw(std::max<size_t>(ne, 1), 0);
  std::vector<int32_t> ifill(itro.begin(), itro.end() - 1), ofill(otro.begin(), otro.end() - 1);
  for (size_t a = 0; a < ne; a++) {
    itcol[ifill[av[a]]] = (int32_t)au[a];
    itw[ifill[av[a]]++] = aw[a];
    otcol[ofill[au[a]]++] = (int32_t)av[a];
  }
  const int z = bgraph_ztiles(G);
  FAP_TRY(G->d_bitro.ensure(itro.size() * 4));
  FAP_TRY(G->d_bitcol.ensure(itcol.size() * 4));
  FAP_TRY(G->d_bitw.ensure(itw.size() * 4));
  FAP_TRY(G->d_botro.ensure(otro.size() * 4));
  FAP_TRY(G->d_botcol.ensure(otcol.size() * 4));
  FAP_TRY(G->d_bgpart.ensure((size_t)nb * 4));
  FAP_TRY(G->d_bpcolmap.ensure((size_t)nb * 4));
  FAP_TRY(G->d_bDt.ensure((size_t)z * nb * kMsbfS * 4));
  FAP_TRY(G->d_bact.ensure((size_t)3 * z * nb * 4));
  FAP_TRY(G->d_bpact.ensure((size_t)z * (G->K + 1) * 4));
  FAP_TRY(G->d_bitems.ensure((size_t)2 * z * nb * 4 + 4 * sizeof(int)));  // two work lists + counts
  FAP_TRY(G->d_msbf_changed.ensure(4 * sizeof(int)));
  if (!G->h_changed) FAP_CK(cudaHostAlloc(reinterpret_cast<void **>(&G->h_changed), 4 * sizeof(int), 0));
  FAP_CK(cudaMemcpy(G->d_bitro.p, itro.data(), itro.size() * 4, cudaMemcpyHostToDevice));
  FAP_CK(cudaMemcpy(G->d_bitcol.p, itcol.data(), itcol.size() * 4, cudaMemcpyHostToDevice));
  FAP_CK(cudaMemcpy(G->d_bitw.p, itw.data(), itw.size() * 4, cudaMemcpyHostToDevice));
  FAP_CK(cudaMemcpy(G->d_botro.p, otro.data(), otro.size() * 4, cudaMemcpyHostToDevice));
  FAP_CK(cudaMemcpy(G->d_botcol.p, otcol.data(), otcol.size() * 4, cudaMemcpyHostToDevice));
  FAP_CK(cudaMemcpy(G->d_bgpart.p, gpart.data(), gpart.size() * 4, cudaMemcpyHostToDevice));
  std::vector<int32_t> pcol((size_t)nb);
  for (int64_t g = 0; g < nb; g++) pcol[g] = G->bpcol[gpart[g]] + (int32_t)(g - G->boff[gpart[g]]);
  FAP_CK(cudaMemcpy(G->d_bpcolmap.p, pcol.data(), pcol.size() * 4, cudaMemcpyHostToDevice));
  G->bg_csr_ready = true;
  return FAP_OK;
}

// Per-part table, output-row list and dB for a batch of all parts in the
// boundary-graph form (descriptors built, F offsets final).
int prepare_bgraph(fap_dgraph *G, const std::vector<PartDesc> &parts, bool col_table = false) {
  const int32_t K = G->K;
  std::vector<BPart> bp((size_t)K + 1);
  std::vector<int64_t> rows;
  for (const PartDesc &d : parts) {
    BPart &b = bp[d.part];
    b.voff = d.start;
    b.b = d.b;
    b.boff = G->boff[d.part];
    b.ldf = d.ldf;
    b.f_off = d.f_off;
    for (int32_t k = 0; k < d.b; k++) {
      rows.push_back(G->boff[d.part] + k);
      rows.push_back(d.row_base + k);
    }
  }
  // (the Bellman-Ford closure writes dB's columns padded per part, so that
  // the expansion's TMA boxes start on 16-byte boundaries)
  G->ldB = round_up(std::max<int64_t>(bgraph_bf(G) ? G->bpcol[G->K + 1] : G->total_b, 1), kFloydTile);
  FAP_TRY(G->d_dB.ensure((size_t)G->ldB * G->ldB * 4));
  const int64_t ldFB = parts.empty() ? kFloydTile : parts[0].ldf;
  FAP_TRY(G->d_FB.ensure((size_t)std::max<int64_t>(G->total_b, 1) * ldFB * 4));
  FAP_TRY(G->d_bpart.ensure(bp.size() * sizeof(BPart)));
  FAP_TRY(G->d_brows.ensure(std::max<size_t>(rows.size(), 2) * 8));
  FAP_CK(cudaMemcpy(G->d_bpart.p, bp.data(), bp.size() * sizeof(BPart), cudaMemcpyHostToDevice));
  if (!rows.empty())
    FAP_CK(cudaMemcpy(G->d_brows.p, rows.data(), rows.size() * 8, cudaMemcpyHostToDevice));
  if (bgraph_tiled_expand(G)) {
    std::vector<int64_t> grow((size_t)G->total_b, 0);
    for (size_t i = 0; i + 1 < rows.size(); i += 2) grow[rows[i]] = rows[i + 1];
    FAP_TRY(G->d_grow.ensure(grow.size() * 8));
    FAP_CK(cudaMemcpy(G->d_grow.p, grow.data(), grow.size() * 8, cudaMemcpyHostToDevice));
  }
  if (bgraph_bf(G)) FAP_TRY(build_bgraph_csr(G));
  G->bTc_maxb = 0;
  if (col_table && !bgraph_bf(G) && !bgraph_tiled_expand(G)) {
    int maxb = 0;
    for (const PartDesc &d : parts) maxb = std::max(maxb, d.b);
    const size_t bytes = (size_t)maxb * G->ldD * 4;
    if (maxb > 0 && bytes <= kColTableBytes) {
      FAP_TRY(G->d_bTc.ensure(bytes));
      G->bTc_maxb = maxb;
    }
  }
  return FAP_OK;
}

// dB (total_b x total_b, ld ldB) = the closed boundary graph of the local
// closures F of all parts: Floyd for small boundary sets, the tiled
// Bellman-Ford (host-polled convergence) for large ones.
template <typename T>
int close_bgraph(fap_dgraph *G, const PartDesc *dp, int np, int max_b, const T *F, int *status,
                 int64_t max_rounds, int64_t *L) {
  cudaStream_t st = G->ctx->stream;
  T *dB = G->d_dB.as<T>();
  if (!bgraph_bf(G)) {
    FAP_CK(launch_bgraph<T>(dp, np, max_b, F, dB, G->ldB, G->ro.as<const int32_t>(), G->col.as<const int32_t>(),
                            G->w.as<const T>(), G->n, G->d_gid.as<const int32_t>(),
                            G->d_ed2st.as<const int32_t>(), G->d_bpart.as<const BPart>(), st, L));
    FAP_CK(launch_floyd_matrix<T>(dB, G->ldB, (int)ceil_div(G->total_b, kFloydTile), status, st, L,
                                  (int)G->total_b));
    return FAP_OK;
  }
  const int z = bgraph_ztiles(G);
  int *wl = G->d_bitems.as<int>();
  FAP_CK(launch_bgraph_bf<T>(dp, np, max_b, F, G->d_bitro.as<const int32_t>(), G->d_bitcol.as<const int32_t>(),
                             G->d_bitw.as<const T>(), G->d_botro.as<const int32_t>(), G->d_botcol.as<const int32_t>(),
                             G->d_bgpart.as<const int32_t>(), G->d_bpcolmap.as<const int32_t>(), (int)G->total_b,
                             G->K, z, dB,
                             G->ldB, G->d_bDt.as<T>(), G->d_bact.as<int>(), G->d_bpact.as<int>(), wl,
                             wl + (int64_t)2 * z * G->total_b, G->d_msbf_changed.as<int>(), G->h_changed,
                             max_rounds, status, st, L));
  return FAP_OK;
}

// Boundary rows of D (or of the cache) from the closed dB: the staged
// expansion for small boundary sets, the tiled one otherwise.  Also FB.
template <typename T>
int expand_bgraph(fap_dgraph *G, const PartDesc *dp, int np, int max_s, const T *F, T *Dout, int64_t ldFB,
                  int *status, int64_t *L, int64_t nrows = -1) {
  cudaStream_t st = G->ctx->stream;
  if (bgraph_bf(G)) {  // padded dB columns: TMA-fed tiles (F: np squares of side ldFB)
    // packed 16-bit tiles where they provably fit (int32, "minplus_pack16")
    Expand16 xk{};
    const bool pack = G->pack16 && G->dtype == FAP_DTYPE_I32;
    if (pack) {
      const int64_t nrt = ceil_div(G->total_b, 128);
      FAP_TRY(G->d_xk_off.ensure_async((size_t)np * G->total_b * 4, st));
      FAP_TRY(G->d_xk_range.ensure_async((size_t)np * nrt * 4, st));
      FAP_TRY(G->d_xk_maxb.ensure_async((size_t)np * 4, st));
      if (!G->d_xk_tiles.p) {
        FAP_TRY(G->d_xk_tiles.ensure_async(2 * sizeof(unsigned long long), st));
        FAP_CK(cudaMemsetAsync(G->d_xk_tiles.p, 0, 2 * sizeof(unsigned long long), st));
      }
      xk.off = G->d_xk_off.as<int32_t>();
      xk.range = G->d_xk_range.as<int32_t>();
      xk.maxB = G->d_xk_maxb.as<int32_t>();
      xk.nrt = (int32_t)nrt;
      xk.tiles = G->d_xk_tiles.as<unsigned long long>();
      // operands packed beforehand ("minplus_prepack"), when they fit
      int32_t max_b = 0;
      for (int32_t q = 1; q <= G->K; q++) max_b = std::max(max_b, G->bnum[q]);
      const int64_t ap_ld = round_up(ceil_div(G->total_b, 2), 4);
      const size_t ap_bytes = (size_t)G->total_b * ap_ld * 4, bd_bytes = (size_t)G->total_b * ldFB * 4;
      const bool grow = G->d_xk_ap.bytes < ap_bytes || G->d_xk_bd.bytes < bd_bytes;
      size_t free_b = 0, total_mem = 0;
      if (G->prepack && max_b > 0 && ldFB % 4 == 0 && ap_bytes + bd_bytes <= kPrepackBytes &&
          (!grow || (cudaMemGetInfo(&free_b, &total_mem) == cudaSuccess && ap_bytes + bd_bytes <= free_b / 4)) &&
          G->d_xk_ap.ensure_async(ap_bytes, st) == FAP_OK && G->d_xk_bd.ensure_async(bd_bytes, st) == FAP_OK) {
        xk.ap = G->d_xk_ap.as<uint32_t>();
        xk.bd = G->d_xk_bd.as<uint32_t>();
        xk.ap_ld = (int32_t)ap_ld;
        xk.bd_ld = (int32_t)ldFB;
        xk.max_b = max_b;
        xk.rows = G->total_b;
      } else {
        cudaGetLastError();  // (a failed cudaMemGetInfo or allocation: tiles convert their stages)
      }
    }
    FAP_CK(launch_bdy_expand_tma<T>(dp, np, max_s, (int)G->total_b, G->d_grow.as<const int64_t>(),
                                    G->d_st2ed.as<const int32_t>(), G->d_dB.as<const T>(), G->ldB, F, ldFB, np,
                                    Dout, G->ldD, G->d_FB.as<T>(), ldFB, status, st, L, pack ? &xk : nullptr));
    return FAP_OK;
  }
  if (!bgraph_tiled_expand(G)) {
    // (rows: the first nrows (boundary index, output row) pairs of d_brows)
    FAP_CK(launch_bdy_expand<T>(G->d_brows.as<const int64_t>(), nrows >= 0 ? (int)nrows : (int)G->total_b,
                                G->d_bpart.as<const BPart>(),
                                G->d_gid.as<const int32_t>(), G->d_ed2st.as<const int32_t>(), G->n,
                                G->d_dB.as<const T>(), G->ldB, (int)G->total_b, F, Dout, G->ldD, G->d_FB.as<T>(),
                                ldFB, G->bTc_maxb > 0 ? G->d_bTc.as<T>() : nullptr, G->bTc_maxb, st, L));
  } else {
    FAP_CK(launch_bdy_expand_tiled<T>(dp, np, max_s, (int)G->total_b, G->d_grow.as<const int64_t>(),
                                      G->d_st2ed.as<const int32_t>(), G->d_dB.as<const T>(), G->ldB, F, Dout,
                                      G->ldD, G->d_FB.as<T>(), ldFB, st, L));
  }
  return FAP_OK;
}

// Builds (or reuses) the batch descriptors for the requested parts.
int prepare_batch(fap_dgraph *G, const std::vector<int32_t> &ids, bool cached, bool bmethod) {
  const bool same = (ids == G->last_ids) && (cached == G->last_cached) && (bmethod == G->last_bmethod);
  if (same) return FAP_OK;
  // The descriptors change from here on: until they are complete no batch
  // counts as prepared, so a failure below forces a full rebuild next time.
  G->last_ids.clear();
  const int64_t n = G->n;
  const bool full = (G->max_rows == n);
  // rows
  std::vector<int64_t> base(ids.size());
  int64_t next = 0;
  for (size_t i = 0; i < ids.size(); i++) {
    const int32_t p = ids[i];
    if (full) {
      base[i] = G->voff[p];
    } else {
      base[i] = next;
      next += G->vnum[p];
    }
  }
  if (!full && next > G->max_rows)
    return fail(FAP_ERR_NOMEM, "requested parts need %lld rows, %lld reserved", (long long)next,
                (long long)G->max_rows);
  G->parts.clear();
  G->work.clear();
  G->src.clear();
  G->srcrows.clear();
  G->part_src_off.assign(1, 0);
  G->part_work_begin.clear();
  G->part_work_end.clear();
  G->thin.clear();
  G->thin_pos.clear();
  // Floyd arena: equal padded squares (one tensor map describes all parts);
  // with the resident cache, the parts' closed matrices in the cache.
  int32_t ldf = kFloydTile;
  for (int32_t p : ids) ldf = std::max<int32_t>(ldf, (int32_t)round_up(std::max(G->vnum[p], 1), kFloydTile));
  if (cached) ldf = G->cache_ldf;
  int64_t foff = 0;
  G->max_ldf = ldf;
  G->max_b = 0;
  G->max_s = 0;
  for (size_t i = 0; i < ids.size(); i++) {
    const int32_t p = ids[i];
    PartDesc d{};
    d.part = p;
    d.start = G->voff[p];
    d.s = G->vnum[p];
    d.b = G->bnum[p];
    d.row_base = base[i];
    d.ldf = ldf;
    d.f_off = cached ? (int64_t)(p - 1) * ldf * ldf : foff;
    d.bd_row = cached ? (int32_t)G->cb_off[p] : bmethod ? G->boff[p] : 0;
    d.flags = bmethod ? kPartLocal : 0;
    d.bd_col = G->bpcol[p];
    foff += (int64_t)d.ldf * d.ldf;
    G->max_b = std::max(G->max_b, d.b);
    G->max_s = std::max(G->max_s, d.s);
    G->parts.push_back(d);
    for (int32_t k = 0; k < d.b; k++) {
      G->src.push_back(d.start + k);  // sorted position = SSSP work-space id
      G->srcrows.push_back(d.row_base + k);
    }
    G->part_src_off.push_back((int32_t)G->src.size());
    G->part_work_begin.push_back((int32_t)G->work.size());
    if (d.b <= G->thin_max_b) {
      G->thin_pos.push_back((int32_t)G->thin.size());
      G->thin.push_back((int32_t)i);
    } else {
      G->thin_pos.push_back(-1);
      for (int32_t m0 = 0; m0 < d.s - d.b; m0 += kMinplusBM) G->work.push_back(MPWork{(int32_t)i, m0});
    }
    G->part_work_end.push_back((int32_t)G->work.size());
  }
  G->f_elems = foff;
  // These buffers are used on the context's stream only, so they grow in
  // stream order: a cudaFree would wait for the whole device (every other
  // graph's stream of a server included).  The synchronisation below makes
  // the new buffers ready for the host copies that fill them.
  cudaStream_t st = G->ctx->stream;
  if (!cached) FAP_TRY(G->F.ensure_async((size_t)std::max<int64_t>(foff, 1) * 4, st));
  FAP_TRY(G->d_parts.ensure_async(std::max<size_t>(G->parts.size(), 1) * sizeof(PartDesc), st));
  FAP_TRY(G->d_work.ensure_async(std::max<size_t>(G->work.size(), 1) * sizeof(MPWork), st));
  FAP_TRY(G->d_thin.ensure_async(std::max<size_t>(G->thin.size(), 1) * 4, st));
  FAP_TRY(G->d_src.ensure_async(std::max<size_t>(G->src.size(), 1) * 4, st));
  FAP_TRY(G->d_srcrows.ensure_async(std::max<size_t>(G->srcrows.size(), 1) * 8, st));
  if (!cached && !bmethod)  // (the plain form runs the frontier SSSP per part whatever the form)
    FAP_TRY(G->sssp_scratch.ensure_async(
        (size_t)std::max(sssp_scratch_rows(G->n, (int)G->src.size()), 1) * (size_t)G->n * 4, st));
  G->pk = Pack16{};
  if (G->pack16 && G->dtype == FAP_DTYPE_I32 && !G->work.empty()) {
    const size_t np = G->parts.size();
    const int64_t ntiles = G->ldD / kMinplusBN;
    FAP_TRY(G->d_pk_off.ensure_async(np * (size_t)G->ldD * 4, st));
    FAP_TRY(G->d_pk_range.ensure_async(np * (size_t)ntiles * 4, st));
    FAP_TRY(G->d_pk_maxa.ensure_async(np * 4, st));
    if (!G->d_pk_tiles.p) {
      FAP_TRY(G->d_pk_tiles.ensure_async(2 * sizeof(unsigned long long), st));
      FAP_CK(cudaMemsetAsync(G->d_pk_tiles.p, 0, 2 * sizeof(unsigned long long), st));
    }
    G->pk = Pack16{};
    G->pk.off = G->d_pk_off.as<int32_t>();
    G->pk.range = G->d_pk_range.as<int32_t>();
    G->pk.maxA = G->d_pk_maxa.as<int32_t>();
    G->pk.ntiles = (int32_t)ntiles;
    G->pk.tiles = G->d_pk_tiles.as<unsigned long long>();
    // Operands packed beforehand for the parts with tile work: rows of the
    // parts' boundary vertices in batch order.
    G->pk_krow.assign(np, -1);
    int64_t prows = 0;
    int32_t at_ld = 0, max_b = 0;
    for (const MPWork &w : G->work) {
      const PartDesc &d = G->parts[w.pidx];
      if (G->pk_krow[w.pidx] >= 0) continue;
      G->pk_krow[w.pidx] = (int32_t)prows;
      prows += d.b;
      at_ld = std::max(at_ld, d.s - d.b);
      max_b = std::max(max_b, d.b);
    }
    at_ld = (int32_t)round_up((int64_t)std::max(at_ld, 1), 4);
    const size_t pbytes = (size_t)prows * ((size_t)G->ldD * 2 + (size_t)at_ld * 4);
    // (the free memory is asked for only when the buffers have to grow)
    const bool grow = G->d_pk_s16.bytes < (size_t)prows * G->ldD * 2 || G->d_pk_at.bytes < (size_t)prows * at_ld * 4;
    size_t free_b = 0, total_b = 0;
    if (G->prepack && prows > 0 && prows < INT32_MAX && pbytes <= kPrepackBytes &&
        (!grow || (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && pbytes <= free_b / 4)) &&
        G->d_pk_s16.ensure_async((size_t)prows * G->ldD * 2, st) == FAP_OK &&
        G->d_pk_at.ensure_async((size_t)prows * at_ld * 4, st) == FAP_OK &&
        G->d_pk_krow.ensure_async(np * 4, st) == FAP_OK) {
      G->pk.s16 = G->d_pk_s16.as<uint16_t>();
      G->pk.at = G->d_pk_at.as<uint32_t>();
      G->pk.krow = G->d_pk_krow.as<const int32_t>();
      G->pk.at_ld = at_ld;
      G->pk.max_b = max_b;
      G->pk.prows = prows;
    } else {
      cudaGetLastError();  // (a failed cudaMemGetInfo or allocation: tiles convert their stages)
      G->pk_krow.clear();
    }
  }
  std::vector<QItem> qitems;
  if (!cached) {
    int32_t mnb = 0;
    // (the local closures of the boundary-graph form are symmetric when the
    // parts are; the SSSP form's matrices hold boundary rows and are not)
    G->q.sym = bmethod && G->sym_local && G->floyd_sym;
    qitems = floyd_queue_items(G->parts, G->q.sym, &G->q.nfloyd, &mnb);
    G->q.nitems = (int32_t)qitems.size();
    G->q.stride = 2 + 2 * mnb;
    G->q.nparts = (int32_t)G->parts.size();
    FAP_TRY(G->q.items.ensure_async(std::max<size_t>(qitems.size(), 1) * sizeof(QItem), st));
    FAP_TRY(G->q.cnt.ensure_async(((size_t)G->q.nparts * G->q.stride + 2) * 4, st));
  }
  FAP_CK(cudaStreamSynchronize(st));
  if (!qitems.empty())
    FAP_CK(cudaMemcpy(G->q.items.p, qitems.data(), qitems.size() * sizeof(QItem), cudaMemcpyHostToDevice));
  if (bmethod) FAP_TRY(prepare_bgraph(G, G->parts, true));
  FAP_CK(cudaMemcpy(G->d_parts.p, G->parts.data(), G->parts.size() * sizeof(PartDesc), cudaMemcpyHostToDevice));
  if (!G->work.empty())
    FAP_CK(cudaMemcpy(G->d_work.p, G->work.data(), G->work.size() * sizeof(MPWork), cudaMemcpyHostToDevice));
  if (!G->thin.empty())
    FAP_CK(cudaMemcpy(G->d_thin.p, G->thin.data(), G->thin.size() * 4, cudaMemcpyHostToDevice));
  if (G->pk.s16 != nullptr)
    FAP_CK(cudaMemcpy(G->d_pk_krow.p, G->pk_krow.data(), G->pk_krow.size() * 4, cudaMemcpyHostToDevice));
  if (!G->src.empty()) {
    FAP_CK(cudaMemcpy(G->d_src.p, G->src.data(), G->src.size() * 4, cudaMemcpyHostToDevice));
    FAP_CK(cudaMemcpy(G->d_srcrows.p, G->srcrows.data(), G->srcrows.size() * 8, cudaMemcpyHostToDevice));
  }
  // Rows of other parts may have been overwritten by this batch.
  std::fill(G->row_base.begin(), G->row_base.end(), -1);
  G->last_ids = ids;
  G->last_cached = cached;
  G->last_bmethod = bmethod;
  G->epoch++;
  return FAP_OK;
}

// Bucket width of the near/far SSSP: the tuned value when set, else 64 mean
// edge weights (wide enough that a bucket is finished in a few rounds, narrow
// enough to keep re-relaxations near Dijkstra's count on road-like graphs).
template <typename T>
T sssp_delta_for(const fap_dgraph *G) {
  if (G->sssp_delta == -2.0) return Dist<T>::inf();  // tuned: plain Bellman-Ford
  double d = G->sssp_delta > 0 ? G->sssp_delta : 64.0 * G->mean_w;
  d = std::min<double>(d, (double)Dist<T>::inf());
  if (Dist<T>::kDtype == FAP_DTYPE_I32) d = std::max(1.0, std::floor(d));
  return (T)d;
}

// Predecessor rows of the batch's parts (after their distances).
template <typename T>
int launch_paths(fap_dgraph *G, const PartDesc *dp, int np, int max_s, const T *F, int64_t *L) {
  FAP_CK(launch_pred<T>(dp, np, max_s, G->D.as<const T>(), G->P.as<int32_t>(), G->ldD, G->n,
                        G->d_tro.as<const int32_t>(), G->d_tcol.as<const int32_t>(), G->d_tw.as<const T>(),
                        G->d_st2ed.as<const int32_t>(), F, G->ctx->stream, L));
  return FAP_OK;
}

int ensure_in_edges(fap_dgraph *G);

// Runs a FloydQueue: the Floyd items (and with `scatter` the boundary-row
// scatter into D, and with mp_work > 0 that many min-plus work items' tiles).
template <typename T>
cudaError_t run_floyd_queue(fap_dgraph *G, QueueBuf &qb, const PartDesc *dp, T *F, int64_t ldf, bool scatter,
                            const MPWork *dw, int mp_work, T *D, int64_t drows, int *status, int64_t *L,
                            int arena_parts = -1) {
  cudaStream_t st = G->ctx->stream;
  cudaError_t e = cudaMemsetAsync(qb.cnt.p, 0, ((size_t)qb.nparts * qb.stride + 2) * 4, st);
  if (e != cudaSuccess) return e;
  FloydQueue q{qb.items.as<const QItem>(), scatter ? qb.nitems : qb.nfloyd, mp_work, qb.cnt.as<int32_t>(),
               qb.stride, qb.nparts, qb.sym ? 1 : 0};
  return launch_floyd_queue<T>(dp, arena_parts > 0 ? arena_parts : qb.nparts, F, ldf, q, dw, G->n, D, G->ldD,
                               drows, G->d_st2ed.as<const int32_t>(),
                               G->d_gid.as<const int32_t>(), G->d_ed2st.as<const int32_t>(), status, st, L,
                               nullptr);
}

// Bounds buffers of the packed min-plus for the prepared batch, or null.
const Pack16 *pack16_of(const fap_dgraph *G) { return G->pk.off != nullptr ? &G->pk : nullptr; }

// Whether stage 1's SSSP runs in the tiled form.
bool use_msbf(const fap_dgraph *G) {
  if (G->sssp_form == 1) return false;
  if (G->sssp_form == 2) return true;
  return G->n > 0 && G->m >= 6 * (int64_t)G->n;
}

const char *stage1_form_name(const fap_dgraph *G, bool bmethod) {
  if (bmethod) return bgraph_bf(G) ? "boundary graph, Bellman-Ford closure" : "boundary graph, Floyd closure";
  return use_msbf(G) ? "SSSP, tiled Bellman-Ford" : "SSSP, frontier";
}

// Tiles of the tiled SSSP form run side by side: as many as fit in
// tile_bytes, at most 16.
int msbf_ztiles(const fap_dgraph *G, int count) {
  const int64_t per = std::max<int64_t>(G->n, 1) * kMsbfS * 4;
  return (int)std::max<int64_t>(1, std::min<int64_t>({G->tile_bytes / per, 16, ceil_div(count, kMsbfS)}));
}

// Work items, bitmaps and the pinned convergence flags of the tiled form,
// for `count` sources.
int prepare_msbf(fap_dgraph *G, int count) {
  FAP_TRY(ensure_in_edges(G));
  if (G->msbf_nitems == 0) {
    std::vector<int32_t> tro((size_t)G->n + 1);
    FAP_CK(cudaMemcpy(tro.data(), G->d_tro.p, tro.size() * 4, cudaMemcpyDeviceToHost));
    std::vector<MsbfItem> items;
    for (int32_t v = 0; v < G->n; v++)
      for (int32_t e = tro[v]; e < tro[v + 1]; e += 32) items.push_back(MsbfItem{v, e});
    FAP_TRY(G->d_msbf_items.ensure(std::max<size_t>(items.size(), 1) * sizeof(MsbfItem)));
    if (!items.empty())
      FAP_CK(cudaMemcpy(G->d_msbf_items.p, items.data(), items.size() * sizeof(MsbfItem), cudaMemcpyHostToDevice));
    G->msbf_nitems = (int)items.size();
  }
  const int z = msbf_ztiles(G, count);
  FAP_TRY(G->d_msbf_act.ensure((size_t)2 * z * ceil_div(G->n, 32) * 4));
  FAP_TRY(G->d_msbf_changed.ensure(4 * sizeof(int)));
  if (!G->h_changed) FAP_CK(cudaHostAlloc(reinterpret_cast<void **>(&G->h_changed), 4 * sizeof(int), 0));
  FAP_TRY(G->sssp_scratch.ensure((size_t)z * G->n * kMsbfS * 4));
  return FAP_OK;
}

// Stage 1's SSSP from `count` sources (sorted positions) into rows srow of
// D (ld ldD, all ldD columns): the tiled form or the frontier kernel.
template <typename T>
int run_stage1_sssp(fap_dgraph *G, const int32_t *src, const int64_t *srow, int count, T *D, int *status,
                    int64_t max_rounds, int64_t *L) {
  cudaStream_t st = G->ctx->stream;
  if (use_msbf(G)) {
    FAP_TRY(prepare_msbf(G, count));
    FAP_CK(launch_msbf<T>(G->d_msbf_items.as<const MsbfItem>(), G->msbf_nitems, G->d_tro.as<const int32_t>(),
                          G->d_tcol.as<const int32_t>(), G->d_tw.as<const T>(), G->n,
                          G->d_st2ed.as<const int32_t>(), src, srow, count, D, G->ldD, G->ldD,
                          msbf_ztiles(G, count), G->sssp_scratch.as<T>(), G->d_msbf_act.as<uint32_t>(), G->d_msbf_changed.as<int>(),
                          G->h_changed, max_rounds, status, st, L));
    return FAP_OK;
  }
  FAP_CK(launch_sssp<T>(G->ro_s.as<const int32_t>(), G->col_s.as<const int32_t>(), G->w_s.as<const T>(), G->n,
                        src, srow, count, D, G->ldD, G->ldD, G->d_ed2st.as<const int32_t>(),
                        G->sssp_scratch.as<T>(), sssp_delta_for<T>(G), G->sssp_chain, G->sssp_precheck,
                        max_rounds, status, st, L));
  return FAP_OK;
}

template <typename T>
int run_solve(fap_dgraph *G, int mode) {
  fap_ctx *c = G->ctx;
  cudaStream_t st = c->stream;
  const int np = (int)G->parts.size();
  const T *w = G->w.as<const T>();
  T *D = G->D.as<T>();
  T *F = G->F.as<T>();
  const int32_t *ro = G->ro.as<const int32_t>(), *col = G->col.as<const int32_t>();
  const int32_t *ro_s = G->ro_s.as<const int32_t>(), *col_s = G->col_s.as<const int32_t>();
  const T *w_s = G->w_s.as<const T>();
  T *scratch = G->sssp_scratch.as<T>();
  const PartDesc *dp = G->d_parts.as<const PartDesc>();
  const MPWork *dw = G->d_work.as<const MPWork>();
  const int32_t *src = G->d_src.as<const int32_t>();
  const int64_t *srow = G->d_srcrows.as<const int64_t>();
  const int32_t *gid = G->d_gid.as<const int32_t>(), *st2ed = G->d_st2ed.as<const int32_t>(),
                *ed2st = G->d_ed2st.as<const int32_t>();
  int *status = G->d_status.as<int>();
  const T delta = sssp_delta_for<T>(G);
  const int64_t max_rounds = G->sssp_max_rounds > 0 ? G->sssp_max_rounds : 8 * (int64_t)G->n + 1024;
  int64_t L = 0;
  FAP_CK(cudaMemsetAsync(status, 0, sizeof(int), st));
  for (int i = 0; i < 5; i++) G->timing[i] = -1.0f;
  if (mode == FAP_MODE_BATCHED && G->last_bmethod) {
    // Boundary-graph form: local closures of all parts, boundary-graph APSP,
    // boundary rows by expansion, then the min-plus merge.  The events keep
    // the stage slots in order of time: [gather, floyd, boundary graph +
    // expansion, min-plus] (fap_graph_last_timing maps them back).
    FAP_CK(record_event(c->ev[0], st));
    FAP_CK(launch_gather<T>(dp, np, G->max_ldf, ro, col, w, gid, st2ed, ed2st, D, G->ldD, F, st, &L));
    FAP_CK(record_event(c->ev[1], st));
    if (G->floyd_queue)
      FAP_CK(run_floyd_queue<T>(G, G->q, dp, F, G->max_ldf, false, nullptr, 0, D, G->max_rows, status, &L));
    else
      FAP_CK(launch_floyd_parts_multi<T>(dp, np, (int)ceil_div(G->max_s, kFloydTile), F, G->max_ldf,
                                         status, st, &L));
    FAP_CK(record_event(c->ev[2], st));
    FAP_TRY(close_bgraph<T>(G, dp, np, G->max_b, F, status, max_rounds, &L));
    FAP_TRY(expand_bgraph<T>(G, dp, np, G->max_s, F, D, G->max_ldf, status, &L));
    FAP_CK(launch_local_fixup<T>(dp, np, G->max_s, F, G->d_FB.as<const T>(), G->max_ldf, st, &L));
    FAP_CK(record_event(c->ev[3], st));
    FAP_CK(launch_minplus_thin<T>(dp, G->d_thin.as<int32_t>(), (int)G->thin.size(), G->max_s, G->n, F, D,
                                  G->ldD, gid, ed2st, st, &L));
    FAP_CK(launch_minplus_parts<T>(dp, np, dw, (int)G->work.size(), G->n, F, G->max_ldf, D, G->ldD,
                                   G->max_rows, gid, ed2st, status, st, &L, pack16_of(G)));
    if (G->paths) FAP_TRY(launch_paths<T>(G, dp, np, G->max_s, F, &L));
    FAP_CK(record_event(c->ev[4], st));
  } else if (mode == FAP_MODE_BATCHED && G->last_cached) {
    // Resident cache: boundary rows and closed Floyd matrices are ready;
    // copy the boundary rows into the block and run the min-plus merge.
    const T *cF = G->cF.as<const T>();
    FAP_CK(record_event(c->ev[0], st));
    FAP_CK(record_event(c->ev[1], st));
    FAP_CK(launch_bdy_copy<T>(dp, np, G->max_b, G->cBd.as<const T>(), D, G->ldD, st, &L));
    FAP_CK(record_event(c->ev[2], st));
    FAP_CK(record_event(c->ev[3], st));
    FAP_CK(launch_minplus_thin<T>(dp, G->d_thin.as<int32_t>(), (int)G->thin.size(), G->max_s, G->n, cF, D,
                                  G->ldD, gid, ed2st, st, &L));
    FAP_CK(launch_minplus_parts<T>(dp, (int)G->K, dw, (int)G->work.size(), G->n, cF, G->cache_ldf, D,
                                   G->ldD, G->max_rows, gid, ed2st, status, st, &L, pack16_of(G)));
    if (G->paths) FAP_TRY(launch_paths<T>(G, dp, np, G->max_s, cF, &L));
    FAP_CK(record_event(c->ev[4], st));
  } else if (mode == FAP_MODE_BATCHED) {
    FAP_CK(record_event(c->ev[0], st));
    FAP_TRY(run_stage1_sssp<T>(G, src, srow, (int)G->src.size(), D, status, max_rounds, &L));
    FAP_CK(record_event(c->ev[1], st));
    FAP_CK(launch_gather<T>(dp, np, G->max_ldf, ro, col, w, gid, st2ed, ed2st, D, G->ldD, F, st, &L));
    FAP_CK(record_event(c->ev[2], st));
    // With the work queue, the min-plus tiles run in the same launch as the
    // Floyd (each part's as soon as its closure and boundary rows are done)
    // unless they use the packed form, whose bounds need every boundary row.
    int mp_in_queue = 0;
    if (G->floyd_per_cta) {
      FAP_CK(launch_floyd_parts<T>(dp, np, F, G->max_ldf, D, G->ldD, st2ed, status, st, &L));
    } else if (G->floyd_queue) {
      mp_in_queue = pack16_of(G) == nullptr ? (int)G->work.size() : 0;
      FAP_CK(run_floyd_queue<T>(G, G->q, dp, F, G->max_ldf, true, dw, mp_in_queue, D, G->max_rows, status, &L));
    } else {
      FAP_CK(launch_floyd_parts_multi<T>(dp, np, (int)ceil_div(G->max_s, kFloydTile), F, G->max_ldf,
                                         status, st, &L));
      FAP_CK(launch_bdy_scatter<T>(dp, np, F, D, G->ldD, st2ed, G->max_b, G->max_s, st, &L));
    }
    FAP_CK(record_event(c->ev[3], st));
    FAP_CK(launch_minplus_thin<T>(dp, G->d_thin.as<int32_t>(), (int)G->thin.size(), G->max_s, G->n, F, D,
                                  G->ldD, gid, ed2st, st, &L));
    if (mp_in_queue == 0)
      FAP_CK(launch_minplus_parts<T>(dp, np, dw, (int)G->work.size(), G->n, F, G->max_ldf, D, G->ldD,
                                     G->max_rows, gid, ed2st, status, st, &L, pack16_of(G)));
    if (G->paths) FAP_TRY(launch_paths<T>(G, dp, np, G->max_s, F, &L));
    FAP_CK(record_event(c->ev[4], st));
  } else {
    FAP_CK(record_event(c->ev[0], st));
    for (int i = 0; i < np; i++) {
      const PartDesc &d = G->parts[i];
      const int s0 = G->part_src_off[i], s1 = G->part_src_off[i + 1];
      const int w0 = G->part_work_begin[i], w1 = G->part_work_end[i];
      FAP_CK(launch_sssp<T>(ro_s, col_s, w_s, G->n, src + s0, srow + s0, s1 - s0, D, G->ldD,
                            G->ldD, ed2st, scratch, delta, G->sssp_chain, G->sssp_precheck, max_rounds, status, st, &L));
      FAP_CK(launch_gather<T>(dp + i, 1, d.ldf, ro, col, w, gid, st2ed, ed2st, D, G->ldD, F, st, &L));
      FAP_CK(launch_floyd_matrix<T>(F + d.f_off, d.ldf, (int)ceil_div(d.s, kFloydTile), status, st, &L, d.s));
      FAP_CK(launch_bdy_scatter<T>(dp + i, 1, F, D, G->ldD, st2ed, d.b, d.s, st, &L));
      if (G->thin_pos[i] >= 0)
        FAP_CK(launch_minplus_thin<T>(dp, G->d_thin.as<int32_t>() + G->thin_pos[i], 1, d.s - d.b, G->n, F, D,
                                      G->ldD, gid, ed2st, st, &L));
      else
        FAP_CK(launch_minplus_parts<T>(dp, np, dw + w0, w1 - w0, G->n, F, G->max_ldf, D, G->ldD,
                                       G->max_rows, gid, ed2st, status, st, &L, pack16_of(G)));
      if (G->paths) FAP_TRY(launch_paths<T>(G, dp + i, 1, d.s, F, &L));
    }
    FAP_CK(record_event(c->ev[4], st));
  }
  G->launches = L;
  c->launches += L;
  return FAP_OK;
}

int status_code(int h) {
  if (h == kDevSsspRoundLimit)
    return fail(FAP_ERR_NOT_CONVERGED, "SSSP hit its round bound");
  if (h == kDevTmaTimeout) return fail(FAP_ERR_DEVICE, "a TMA tile load did not complete in time");
  if (h == kDevQueueTimeout)
    return fail(FAP_ERR_DEVICE, "a work-queue item waited too long for the items it depends on");
  if (h != kDevOk) return fail(FAP_ERR_DEVICE, "device-side error %d", h);
  return FAP_OK;
}

int read_status(fap_dgraph *G) {
  int h = 0;
  FAP_CK(cudaMemcpy(&h, G->d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
  return status_code(h);
}

}  // namespace

extern "C" int fap_solve(fap_dgraph *G, const int32_t *parts, int32_t count, int mode) try {
  if (!G) return fail(FAP_ERR_INVALID, "NULL graph");
  if (G->K == 0) return fail(FAP_ERR_STATE, "fap_solve before fap_graph_set_parts");
  if (mode != FAP_MODE_PLAIN && mode != FAP_MODE_BATCHED) return fail(FAP_ERR_INVALID, "bad mode %d", mode);
  std::vector<int32_t> ids;
  if (parts == nullptr) {
    for (int32_t p = 1; p <= G->K; p++) ids.push_back(p);
  } else {
    if (count < 0) return fail(FAP_ERR_INVALID, "negative count");
    std::vector<char> seen(G->K + 1, 0);
    for (int32_t i = 0; i < count; i++) {
      const int32_t p = parts[i];
      if (p < 1 || p > G->K) return fail(FAP_ERR_INVALID, "part id %d outside 1..%d", p, G->K);
      if (seen[p]) return fail(FAP_ERR_INVALID, "part id %d requested twice", p);
      seen[p] = 1;
      ids.push_back(p);
    }
  }
  if (ids.empty()) return FAP_OK;
  DeviceGuard g(G->ctx->device);
  if (G->max_rows == 0) FAP_TRY(fap_graph_reserve(G, 0));
  if (G->paths && G->P.bytes < (size_t)G->max_rows * G->ldD * 4) {
    FAP_CK(cudaStreamSynchronize(G->ctx->stream));
    G->P.release();
    FAP_TRY(G->P.ensure((size_t)G->max_rows * G->ldD * 4));
    G->epoch++;
  }
  const bool cached = mode == FAP_MODE_BATCHED && G->cache_ready && G->use_cache;
  if (cached && !G->cache_valid.empty())
    for (const int32_t p : ids)
      if (!G->cache_valid[p])
        return fail(FAP_ERR_STATE, "part %d is another rank's: the sharded cache holds this rank's parts only", p);
  const bool bmethod = !cached && mode == FAP_MODE_BATCHED && (int32_t)ids.size() == G->K && bmethod_ok(G);
  FAP_TRY(prepare_batch(G, ids, cached, bmethod));
  int rc = FAP_OK;
  cudaStream_t st = G->ctx->stream;
  // (the tiled SSSP form tests convergence on the host: not capturable)
  const bool host_loop = !cached && (bmethod ? bgraph_bf(G) : use_msbf(G));
  G->stage1_name = cached ? "resident cache (" + G->cache_stage1_name + ")" : stage1_form_name(G, bmethod);
  // A batch is captured the second time it is solved unchanged: a batch
  // solved once (a server's batches of changing composition) runs its
  // launches directly instead of paying for a capture and an instantiation.
  const bool replayable = G->gexec && G->gexec_epoch == G->epoch && G->gexec_stream == st;
  if (mode == FAP_MODE_BATCHED && G->use_graph && st != nullptr && !host_loop &&
      (replayable || G->direct_epoch == G->epoch)) {
    if (!replayable) {
      if (G->gexec) cudaGraphExecDestroy(G->gexec);
      G->gexec = nullptr;
      // Capture the whole batched launch sequence once; replay it while the
      // batch, its buffers, the parameters and the stream stay the same.
      FAP_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      rc = (G->dtype == FAP_DTYPE_I32) ? run_solve<int32_t>(G, mode) : run_solve<float>(G, mode);
      cudaGraph_t graph = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(st, &graph);
      if (rc != FAP_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      if (ec != cudaSuccess) return fail(FAP_ERR_CUDA, "stream capture: %s", cudaGetErrorString(ec));
      const cudaError_t ei = cudaGraphInstantiate(&G->gexec, graph, 0);
      cudaGraphDestroy(graph);
      if (ei != cudaSuccess) {
        G->gexec = nullptr;
        return fail(FAP_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ei));
      }
      G->gexec_epoch = G->epoch;
      G->gexec_stream = st;
      G->gexec_launches = G->launches;
    }
    FAP_CK(cudaGraphLaunch(G->gexec, st));
    G->launches = G->gexec_launches;
    G->ctx->launches += G->launches;
  } else {
    rc = (G->dtype == FAP_DTYPE_I32) ? run_solve<int32_t>(G, mode) : run_solve<float>(G, mode);
    if (rc != FAP_OK) return rc;
    G->direct_epoch = mode == FAP_MODE_BATCHED ? G->epoch : 0;
  }
  for (const PartDesc &d : G->parts) G->row_base[d.part] = d.row_base;
  G->path_ok.assign(G->K + 1, 0);
  if (G->paths)
    for (const PartDesc &d : G->parts) G->path_ok[d.part] = 1;
  G->last_mode = mode;
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_check(fap_dgraph *G) try {
  if (!G) return fail(FAP_ERR_INVALID, "NULL graph");
  DeviceGuard g(G->ctx->device);
  FAP_CK(cudaStreamSynchronize(G->ctx->stream));
  FAP_TRY(read_status(G));
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_last_timing(fap_dgraph *G, float *ms5) try {
  if (!G || !ms5) return fail(FAP_ERR_INVALID, "NULL argument");
  for (int i = 0; i < 5; i++) ms5[i] = -1.0f;
  if (G->last_mode < 0) return fail(FAP_ERR_STATE, "no solve yet");
  DeviceGuard g(G->ctx->device);
  fap_ctx *c = G->ctx;
  FAP_CK(cudaEventSynchronize(c->ev[4]));
  float t;
  FAP_CK(cudaEventElapsedTime(&t, c->ev[0], c->ev[4]));
  ms5[4] = t;
  if (G->last_mode == FAP_MODE_BATCHED) {
    float seg[4];
    for (int i = 0; i < 4; i++) {
      FAP_CK(cudaEventElapsedTime(&t, c->ev[i], c->ev[i + 1]));
      seg[i] = t;
    }
    if (G->last_bmethod) {  // recorded as [gather, floyd, boundary graph, min-plus]
      ms5[0] = seg[2];
      ms5[1] = seg[0];
      ms5[2] = seg[1];
      ms5[3] = seg[3];
    } else {
      for (int i = 0; i < 4; i++) ms5[i] = seg[i];
    }
  }
  for (int i = 0; i < 5; i++) G->timing[i] = ms5[i];
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_last_stage1(const fap_dgraph *G) try {
  if (!G) return fail(FAP_ERR_INVALID, "NULL graph");
  if (G->last_mode < 0) return 0;
  if (G->last_cached) return 3;
  return G->last_bmethod ? 2 : 1;
} catch (...) {
  return fail_exception();
}

extern "C" const char *fap_graph_stage1_name(const fap_dgraph *G) {
  if (!G) {
    fail(FAP_ERR_INVALID, "NULL graph");
    return "";
  }
  return G->stage1_name.c_str();
}

extern "C" int fap_graph_last_launches(fap_dgraph *G, int64_t *count) try {
  if (!G || !count) return fail(FAP_ERR_INVALID, "NULL argument");
  *count = G->launches;
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_block(fap_dgraph *G, int32_t part, void **dev_ptr, int64_t *rows,
                               int64_t *ld) try {
  if (!G || !dev_ptr || !rows || !ld) return fail(FAP_ERR_INVALID, "NULL argument");
  if (part < 1 || part > G->K) return fail(FAP_ERR_INVALID, "part %d outside 1..%d", part, G->K);
  if (G->row_base[part] < 0) return fail(FAP_ERR_STATE, "part %d is not resident", part);
  *dev_ptr = G->D.as<char>() + (size_t)G->row_base[part] * G->ldD * 4;
  *rows = G->vnum[part];
  *ld = G->ldD;
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_copy_block(fap_dgraph *G, int32_t part, void *host, int out_dtype) try {
  if (!G || !host) return fail(FAP_ERR_INVALID, "NULL argument");
  void *dp;
  int64_t rows, ld;
  FAP_TRY(fap_graph_block(G, part, &dp, &rows, &ld));
  DeviceGuard g(G->ctx->device);
  cudaStream_t st = G->ctx->stream;
  const int64_t n = G->n;
  if (rows == 0) return FAP_OK;
  if (out_dtype == G->dtype) {
    FAP_CK(cudaMemcpy2DAsync(host, (size_t)n * 4, dp, (size_t)ld * 4, (size_t)n * 4, (size_t)rows,
                             cudaMemcpyDeviceToHost, st));
  } else if (G->dtype == FAP_DTYPE_I32 && out_dtype == FAP_DTYPE_F32) {
    FAP_TRY(G->staging.ensure((size_t)rows * n * 4));
    int64_t L = 0;
    FAP_CK(launch_i32_to_f32(reinterpret_cast<const int32_t *>(dp), rows, n, ld,
                             G->staging.as<float>(), st, &L));
    FAP_CK(cudaMemcpyAsync(host, G->staging.p, (size_t)rows * n * 4, cudaMemcpyDeviceToHost, st));
  } else {
    return fail(FAP_ERR_INVALID, "cannot copy %s distances as int32",
                G->dtype == FAP_DTYPE_F32 ? "float" : "?");
  }
  FAP_CK(cudaStreamSynchronize(st));
  FAP_TRY(read_status(G));
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_copy_block_async(fap_dgraph *G, int32_t part, void *host, int out_dtype,
                                          int32_t slot) try {
  if (!G || !host) return fail(FAP_ERR_INVALID, "NULL argument");
  if (slot < 0 || slot >= FAP_COPY_SLOTS) return fail(FAP_ERR_INVALID, "slot %d outside 0..%d", slot, FAP_COPY_SLOTS - 1);
  if (out_dtype != G->dtype && !(G->dtype == FAP_DTYPE_I32 && out_dtype == FAP_DTYPE_F32))
    return fail(FAP_ERR_INVALID, "cannot copy %s distances as int32", G->dtype == FAP_DTYPE_F32 ? "float" : "?");
  void *dp;
  int64_t rows, ld;
  FAP_TRY(fap_graph_block(G, part, &dp, &rows, &ld));
  DeviceGuard g(G->ctx->device);
  cudaStream_t st = G->ctx->stream;
  const int64_t n = G->n;
  auto &cs = G->cslot[slot];
  // the slot's previous copy has finished reading its staging buffer and
  // writing its host memory
  if (cs.busy) FAP_CK(cudaEventSynchronize(cs.done));
  cs.busy = false;
  if (rows == 0) return FAP_OK;
  if (out_dtype == G->dtype) {
    // no conversion: the copy reads the block itself, so it runs on the
    // context stream, in order with the solves that may reuse the rows
    FAP_CK(cudaMemcpy2DAsync(host, (size_t)n * 4, dp, (size_t)ld * 4, (size_t)n * 4, (size_t)rows,
                             cudaMemcpyDeviceToHost, st));
    if (!cs.done) FAP_CK(cudaEventCreateWithFlags(&cs.done, cudaEventDisableTiming));
    FAP_CK(cudaEventRecord(cs.done, st));
    cs.busy = true;
    return FAP_OK;
  }
  if (!cs.stream) FAP_CK(cudaStreamCreateWithFlags(&cs.stream, cudaStreamNonBlocking));
  if (!cs.converted) FAP_CK(cudaEventCreateWithFlags(&cs.converted, cudaEventDisableTiming));
  if (!cs.done) FAP_CK(cudaEventCreateWithFlags(&cs.done, cudaEventDisableTiming));
  // (sized once for the largest part: growing it would free the buffer,
  // and a cudaFree waits for the other slot's copy)
  if (cs.staging.bytes < (size_t)rows * n * 4) {
    int32_t most = 0;
    for (int32_t q = 1; q <= G->K; q++) most = std::max(most, G->vnum[q]);
    FAP_TRY(cs.staging.ensure((size_t)std::max<int64_t>(most, rows) * n * 4));
  }
  int64_t L = 0;
  // the conversion on the context stream (after the solve that made the
  // block), the copy of the converted rows on the slot's stream
  FAP_CK(launch_i32_to_f32(reinterpret_cast<const int32_t *>(dp), rows, n, ld, cs.staging.as<float>(), st, &L));
  FAP_CK(cudaEventRecord(cs.converted, st));
  FAP_CK(cudaStreamWaitEvent(cs.stream, cs.converted, 0));
  FAP_CK(cudaMemcpyAsync(host, cs.staging.p, (size_t)rows * n * 4, cudaMemcpyDeviceToHost, cs.stream));
  FAP_CK(cudaEventRecord(cs.done, cs.stream));
  cs.busy = true;
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_copy_wait(fap_dgraph *G, int32_t slot) try {
  if (!G) return fail(FAP_ERR_INVALID, "NULL graph");
  if (slot < 0 || slot >= FAP_COPY_SLOTS) return fail(FAP_ERR_INVALID, "slot %d outside 0..%d", slot, FAP_COPY_SLOTS - 1);
  DeviceGuard g(G->ctx->device);
  auto &cs = G->cslot[slot];
  if (cs.busy) FAP_CK(cudaEventSynchronize(cs.done));
  cs.busy = false;
  FAP_TRY(read_status(G));
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_path_block(fap_dgraph *G, int32_t part, void **dev_ptr, int64_t *rows,
                                    int64_t *ld) try {
  if (!G || !dev_ptr || !rows || !ld) return fail(FAP_ERR_INVALID, "NULL argument");
  void *dp;
  FAP_TRY(fap_graph_block(G, part, &dp, rows, ld));
  if ((int)G->path_ok.size() <= part || !G->path_ok[part])
    return fail(FAP_ERR_STATE, "part %d was solved without paths", part);
  *dev_ptr = G->P.as<char>() + (size_t)G->row_base[part] * G->ldD * 4;
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_copy_path_block(fap_dgraph *G, int32_t part, int32_t *host) try {
  if (!G || !host) return fail(FAP_ERR_INVALID, "NULL argument");
  void *dp;
  int64_t rows, ld;
  FAP_TRY(fap_graph_path_block(G, part, &dp, &rows, &ld));
  if (rows == 0) return FAP_OK;
  DeviceGuard g(G->ctx->device);
  cudaStream_t st = G->ctx->stream;
  FAP_CK(cudaMemcpy2DAsync(host, (size_t)G->n * 4, dp, (size_t)ld * 4, (size_t)G->n * 4, (size_t)rows,
                           cudaMemcpyDeviceToHost, st));
  FAP_CK(cudaStreamSynchronize(st));
  FAP_TRY(read_status(G));
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_block_checksums(fap_dgraph *G, int32_t part, uint64_t *host_out) try {
  if (!G || !host_out) return fail(FAP_ERR_INVALID, "NULL argument");
  if (G->dtype != FAP_DTYPE_I32) return fail(FAP_ERR_INVALID, "checksums need the int32 path");
  void *dp;
  int64_t rows, ld;
  FAP_TRY(fap_graph_block(G, part, &dp, &rows, &ld));
  if (rows == 0) return FAP_OK;
  DeviceGuard g(G->ctx->device);
  cudaStream_t st = G->ctx->stream;
  FAP_TRY(G->d_checks.ensure((size_t)rows * 8));
  int64_t L = 0;
  FAP_CK(launch_row_checksums(reinterpret_cast<const int32_t *>(dp), rows, G->n, ld,
                              G->d_checks.as<uint64_t>(), st, &L));
  FAP_CK(cudaMemcpyAsync(host_out, G->d_checks.p, (size_t)rows * 8, cudaMemcpyDeviceToHost, st));
  FAP_CK(cudaStreamSynchronize(st));
  FAP_TRY(read_status(G));
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_checksums_async(fap_dgraph *G, int32_t part, uint64_t *d_out) try {
  if (!G || !d_out) return fail(FAP_ERR_INVALID, "NULL argument");
  if (G->dtype != FAP_DTYPE_I32) return fail(FAP_ERR_INVALID, "checksums need the int32 path");
  void *dp;
  int64_t rows, ld;
  FAP_TRY(fap_graph_block(G, part, &dp, &rows, &ld));
  DeviceGuard g(G->ctx->device);
  int64_t L = 0;
  FAP_CK(launch_row_checksums(reinterpret_cast<const int32_t *>(dp), rows, G->n, ld, d_out,
                              G->ctx->stream, &L));
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_status_async(fap_dgraph *G, int32_t *host_status) try {
  if (!G || !host_status) return fail(FAP_ERR_INVALID, "NULL argument");
  DeviceGuard g(G->ctx->device);
  FAP_CK(cudaMemcpyAsync(host_status, G->d_status.p, sizeof(int32_t), cudaMemcpyDeviceToHost,
                         G->ctx->stream));
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_status_code(int32_t device_status) { return status_code(device_status); }

// ---------------------------------------------------------------------------
// device-pointer operators
// ---------------------------------------------------------------------------
namespace {
int read_ctx_status(fap_ctx *c) {
  int h = 0;
  FAP_CK(cudaMemcpyAsync(&h, c->status.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  FAP_CK(cudaStreamSynchronize(c->stream));
  if (h == kDevSsspRoundLimit) return fail(FAP_ERR_NOT_CONVERGED, "SSSP hit its round bound");
  if (h != kDevOk) return fail(FAP_ERR_DEVICE, "device-side error %d", h);
  return FAP_OK;
}
}  // namespace

extern "C" int fap_op_sssp(fap_ctx *c, int dtype, int32_t n, int64_t m, const int32_t *row_offset,
                           const int32_t *col_val, const void *weight, const int32_t *sources,
                           int32_t num_sources, void *out, int64_t ld_out) try {
  if (!c || !row_offset || (m > 0 && (!col_val || !weight)) || (num_sources > 0 && (!sources || !out)))
    return fail(FAP_ERR_INVALID, "NULL argument");
  if (n <= 0 || m < 0 || num_sources < 0 || ld_out < n) return fail(FAP_ERR_INVALID, "bad sizes");
  if ((size_t)ceil_div(n, 32) * 8 > 227 * 1024)
    return fail(FAP_ERR_INVALID, "n=%d exceeds the shared-memory frontier limit", n);
  DeviceGuard g(c->device);
  FAP_CK(cudaMemsetAsync(c->status.p, 0, sizeof(int), c->stream));
  int64_t L = 0;
  const int64_t rounds = 8 * (int64_t)n + 1024;
  if (dtype == FAP_DTYPE_I32) {
    FAP_CK(launch_sssp<int32_t>(row_offset, col_val, (const int32_t *)weight, n, sources, nullptr,
                                num_sources, (int32_t *)out, ld_out, n, nullptr, nullptr, kInfI32, 0, 1,
                                rounds,
                                c->status.as<int>(), c->stream, &L));
  } else if (dtype == FAP_DTYPE_F32) {
    FAP_CK(launch_sssp<float>(row_offset, col_val, (const float *)weight, n, sources, nullptr,
                              num_sources, (float *)out, ld_out, n, nullptr, nullptr, kInfF32, 0, 1,
                              rounds,
                              c->status.as<int>(), c->stream, &L));
  } else {
    return fail(FAP_ERR_INVALID, "bad dtype %d", dtype);
  }
  c->launches += L;
  return read_ctx_status(c);
} catch (...) {
  return fail_exception();
}

extern "C" int fap_op_floyd(fap_ctx *c, int dtype, int32_t s, void *mat, int64_t ld) try {
  if (!c || (s > 0 && !mat)) return fail(FAP_ERR_INVALID, "NULL argument");
  if (s < 0 || ld < s) return fail(FAP_ERR_INVALID, "bad sizes");
  if (s == 0) return FAP_OK;
  if (dtype != FAP_DTYPE_I32 && dtype != FAP_DTYPE_F32) return fail(FAP_ERR_INVALID, "bad dtype");
  DeviceGuard g(c->device);
  cudaStream_t st = c->stream;
  const int64_t ldp = round_up(s, kFloydTile);
  FAP_CK(cudaMemsetAsync(c->status.p, 0, sizeof(int), st));
  FAP_TRY(c->scratch.ensure((size_t)ldp * ldp * 4));
  int64_t L = 0;
  // padded copy: sentinel everywhere, then the matrix
  if (dtype == FAP_DTYPE_I32)
    FAP_CK(launch_fill<int32_t>(c->scratch.as<int32_t>(), ldp, ldp, ldp, kInfI32, st, &L));
  else
    FAP_CK(launch_fill<float>(c->scratch.as<float>(), ldp, ldp, ldp, kInfF32, st, &L));
  FAP_CK(cudaMemcpy2DAsync(c->scratch.p, (size_t)ldp * 4, mat, (size_t)ld * 4, (size_t)s * 4, (size_t)s,
                           cudaMemcpyDeviceToDevice, st));
  if (dtype == FAP_DTYPE_I32)
    FAP_CK(launch_floyd_matrix<int32_t>(c->scratch.as<int32_t>(), ldp, (int)(ldp / kFloydTile),
                                        c->status.as<int>(), st, &L));
  else
    FAP_CK(launch_floyd_matrix<float>(c->scratch.as<float>(), ldp, (int)(ldp / kFloydTile),
                                      c->status.as<int>(), st, &L));
  FAP_CK(cudaMemcpy2DAsync(mat, (size_t)ld * 4, c->scratch.p, (size_t)ldp * 4, (size_t)s * 4, (size_t)s,
                           cudaMemcpyDeviceToDevice, st));
  c->launches += L;
  return read_ctx_status(c);
} catch (...) {
  return fail_exception();
}

extern "C" int fap_op_minplus(fap_ctx *c, int dtype, int32_t M, int32_t N, int32_t K, const void *A,
                              int64_t lda, const void *B, int64_t ldb, void *C, int64_t ldc) try {
  if (!c) return fail(FAP_ERR_INVALID, "NULL ctx");
  if (M < 0 || N < 0 || K < 0) return fail(FAP_ERR_INVALID, "negative size");
  if (M == 0 || N == 0) return FAP_OK;
  if (!C || (K > 0 && (!A || !B))) return fail(FAP_ERR_INVALID, "NULL matrix");
  if (ldc < N || (K > 0 && (lda < K || ldb < N))) return fail(FAP_ERR_INVALID, "bad leading dimension");
  DeviceGuard g(c->device);
  int64_t L = 0;
  if (dtype == FAP_DTYPE_I32)
    FAP_CK(launch_minplus_generic<int32_t>(M, N, K, (const int32_t *)A, lda, (const int32_t *)B, ldb,
                                           (int32_t *)C, ldc, c->stream, &L));
  else if (dtype == FAP_DTYPE_F32)
    FAP_CK(launch_minplus_generic<float>(M, N, K, (const float *)A, lda, (const float *)B, ldb,
                                         (float *)C, ldc, c->stream, &L));
  else
    return fail(FAP_ERR_INVALID, "bad dtype %d", dtype);
  FAP_CK(cudaStreamSynchronize(c->stream));
  c->launches += L;
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_measure_relax_peak(fap_ctx *c, int dtype, double *relax_per_s) try {
  if (!c || !relax_per_s) return fail(FAP_ERR_INVALID, "NULL argument");
  DeviceGuard g(c->device);
  cudaStream_t st = c->stream;
  FAP_TRY(c->sink.ensure(64));
  const int blocks = c->sm_count * 8;
  const int iters = 4096;
  double count = 0;
  float best = 1e30f;
  for (int rep = 0; rep < 4; rep++) {
    FAP_CK(record_event(c->ev[0], st));
    if (dtype == FAP_DTYPE_I32)
      FAP_CK(launch_relax_peak<int32_t>(c->sink.as<int32_t>(), blocks, iters, st, &count));
    else
      FAP_CK(launch_relax_peak<float>(c->sink.as<float>(), blocks, iters, st, &count));
    FAP_CK(record_event(c->ev[1], st));
    FAP_CK(cudaEventSynchronize(c->ev[1]));
    float t;
    FAP_CK(cudaEventElapsedTime(&t, c->ev[0], c->ev[1]));
    if (rep > 0) best = std::min(best, t);
  }
  *relax_per_s = count / (best * 1e-3);
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

namespace {
// Distance rows from original-id sources into rows (count x n, dense).  Uses
// the relabelled work space when the partition is known.
template <typename T>
cudaError_t sssp_rows_launch(fap_dgraph *G, const int32_t *h_sources, int32_t count, DevBuf &srcs,
                             DevBuf &rows, DevBuf &scratch, int64_t *L) {
  cudaStream_t st = G->ctx->stream;
  const int64_t n = G->n;
  const int64_t rounds = G->sssp_max_rounds > 0 ? G->sssp_max_rounds : 8 * n + 1024;
  const bool relabel = G->K > 0;
  std::vector<int32_t> work(h_sources, h_sources + count);
  if (relabel)
    for (auto &x : work) x = G->ed2st[x];
  cudaError_t e = cudaMemcpyAsync(srcs.p, work.data(), (size_t)count * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(G->d_status.p, 0, sizeof(int), st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e;
  if (relabel) {
    if (scratch.ensure((size_t)std::max(sssp_scratch_rows(G->n, count), 1) * n * 4) != FAP_OK)
      return cudaErrorMemoryAllocation;
    return launch_sssp<T>(G->ro_s.as<int32_t>(), G->col_s.as<int32_t>(), G->w_s.as<T>(), G->n,
                          srcs.as<int32_t>(), nullptr, count, rows.as<T>(), n, n,
                          G->d_ed2st.as<int32_t>(), scratch.as<T>(), sssp_delta_for<T>(G),
                          G->sssp_chain, G->sssp_precheck, rounds, G->d_status.as<int>(), st, L);
  }
  return launch_sssp<T>(G->ro.as<int32_t>(), G->col.as<int32_t>(), G->w.as<T>(), G->n,
                        srcs.as<int32_t>(), nullptr, count, rows.as<T>(), n, n, nullptr, nullptr,
                        sssp_delta_for<T>(G), G->sssp_chain, G->sssp_precheck, rounds,
                        G->d_status.as<int>(), st, L);
}
}  // namespace

extern "C" int fap_graph_sssp_rows(fap_dgraph *G, const int32_t *sources, int32_t count,
                                   float *host_out) try {
  if (!G || (count > 0 && (!sources || !host_out))) return fail(FAP_ERR_INVALID, "NULL argument");
  if (count < 0) return fail(FAP_ERR_INVALID, "negative count");
  if (count == 0) return FAP_OK;
  for (int32_t i = 0; i < count; i++)
    if (sources[i] < 0 || sources[i] >= G->n) return fail(FAP_ERR_INVALID, "source %d out of range", sources[i]);
  DeviceGuard g(G->ctx->device);
  cudaStream_t st = G->ctx->stream;
  const int64_t n = G->n;
  DevBuf srcs, rows, scratch;
  int rc = FAP_OK;
  int64_t L = 0;
  do {
    if ((rc = srcs.ensure((size_t)count * 4)) != FAP_OK) break;
    if ((rc = rows.ensure((size_t)count * n * 4)) != FAP_OK) break;
    cudaError_t e = (G->dtype == FAP_DTYPE_I32)
                        ? sssp_rows_launch<int32_t>(G, sources, count, srcs, rows, scratch, &L)
                        : sssp_rows_launch<float>(G, sources, count, srcs, rows, scratch, &L);
    if (e == cudaSuccess && G->dtype == FAP_DTYPE_I32)
      e = launch_i32_to_f32(rows.as<int32_t>(), count, n, n, rows.as<float>(), st, &L);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(host_out, rows.p, (size_t)count * n * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      rc = fail(e == cudaErrorMemoryAllocation ? FAP_ERR_NOMEM : FAP_ERR_CUDA,
                "fap_graph_sssp_rows: %s", cudaGetErrorString(e));
      break;
    }
    rc = read_status(G);
  } while (0);
  srcs.release();
  rows.release();
  scratch.release();
  G->ctx->launches += L;
  return rc;
} catch (...) {
  return fail_exception();
}

namespace {
int ensure_in_edges(fap_dgraph *G);

// Switches predecessor matrices on: checks that every weight is positive
// (with zero-weight edges, equal distances would not order the
// predecessors), then builds the in-edge CSR (sources ascending per vertex).
int enable_paths(fap_dgraph *G) {
  const int64_t m = (int64_t)G->h_col.size() < G->m ? (int64_t)G->h_col.size() : G->m;
  for (int64_t e = 0; e < m; e++) {
    uint32_t bits = G->h_w[e];
    bool pos;
    if (G->dtype == FAP_DTYPE_I32) {
      int32_t v;
      std::memcpy(&v, &bits, 4);
      pos = v > 0;
    } else {
      float v;
      std::memcpy(&v, &bits, 4);
      pos = v > 0.0f;
    }
    if (!pos) return fail(FAP_ERR_RANGE, "paths need positive edge weights (edge %lld)", (long long)e);
  }
  FAP_TRY(ensure_in_edges(G));
  G->paths = true;
  return FAP_OK;
}

// The in-edge CSR (sources ascending per vertex, original ids), built once.
int ensure_in_edges(fap_dgraph *G) {
  const int64_t m = (int64_t)G->h_col.size() < G->m ? (int64_t)G->h_col.size() : G->m;
  if (G->d_tro.bytes == 0) {
    const int32_t n = G->n;
    std::vector<int32_t> tro((size_t)n + 1, 0), tcol((size_t)std::max<int64_t>(m, 1));
    std::vector<uint32_t> tw((size_t)std::max<int64_t>(m, 1));
    for (int64_t e = 0; e < m; e++) tro[(size_t)G->h_col[e] + 1]++;
    for (int32_t j = 0; j < n; j++) tro[j + 1] += tro[j];
    std::vector<int32_t> fill(tro.begin(), tro.end() - 1);
    for (int32_t u = 0; u < n; u++)
      for (int32_t e = G->h_ro[u]; e < G->h_ro[u + 1]; e++) {
        const int32_t j = G->h_col[e];
        tcol[fill[j]] = u;
        tw[fill[j]] = G->h_w[e];
        fill[j]++;
      }
    DeviceGuard g(G->ctx->device);
    FAP_TRY(G->d_tro.ensure(tro.size() * 4));
    FAP_TRY(G->d_tcol.ensure(tcol.size() * 4));
    FAP_TRY(G->d_tw.ensure(tw.size() * 4));
    FAP_CK(cudaMemcpy(G->d_tro.p, tro.data(), tro.size() * 4, cudaMemcpyHostToDevice));
    FAP_CK(cudaMemcpy(G->d_tcol.p, tcol.data(), tcol.size() * 4, cudaMemcpyHostToDevice));
    FAP_CK(cudaMemcpy(G->d_tw.p, tw.data(), tw.size() * 4, cudaMemcpyHostToDevice));
  }
  return FAP_OK;
}
}  // namespace

extern "C" int fap_queue_order_check(const int32_t *part_sizes, int32_t nparts, int sym) try {
  if (!part_sizes || nparts < 0) return fail(FAP_ERR_INVALID, "NULL or negative argument");
  std::vector<PartDesc> parts((size_t)nparts);
  for (int32_t p = 0; p < nparts; p++) {
    if (part_sizes[p] < 0 || part_sizes[p] > 255 * kFloydTile) return fail(FAP_ERR_INVALID, "part size %d", part_sizes[p]);
    parts[p].s = part_sizes[p];
  }
  int32_t nfloyd = 0, mnb = 0;
  const std::vector<QItem> it = floyd_queue_items(parts, sym != 0, &nfloyd, &mnb);
  if (!queue_order_ok(parts, sym != 0, it, nfloyd)) return fail(FAP_ERR_STATE, "queue order breaks a dependency");
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_set_param(fap_dgraph *G, const char *key, double value) try {
  if (!G || !key) return fail(FAP_ERR_INVALID, "NULL argument");
  G->epoch++;  // a captured launch sequence no longer matches
  if (std::strcmp(key, "cuda_graph") == 0) {
    G->use_graph = value != 0.0;
    return FAP_OK;
  }
  if (std::strcmp(key, "sssp_delta") == 0) {
    G->sssp_delta = (value > 0 && value < 1e8) ? value : -1.0;
    return FAP_OK;
  }
  if (std::strcmp(key, "sssp_precheck") == 0) {
    G->sssp_precheck = value != 0.0 ? 1 : 0;
    return FAP_OK;
  }
  if (std::strcmp(key, "sssp_chain") == 0) {
    G->sssp_chain = value >= 0 ? (int)value : 0;
    return FAP_OK;
  }
  if (std::strcmp(key, "tile_mb") == 0) {
    if (!(value > 0.0) || value > 65536.0) return fail(FAP_ERR_INVALID, "tile_mb is in (0, 65536]");
    G->tile_bytes = std::max<int64_t>(1, (int64_t)(value * 1048576.0));
    G->bg_csr_ready = false;  // the closure's tile buffers are sized with it
    G->last_ids.clear();
    G->epoch++;
    return FAP_OK;
  }
  if (std::strcmp(key, "sssp_form") == 0) {
    if (value != 0.0 && value != 1.0 && value != 2.0) return fail(FAP_ERR_INVALID, "sssp_form is 0, 1 or 2");
    G->sssp_form = (int)value;
    return FAP_OK;
  }
  if (std::strcmp(key, "stage1") == 0) {
    if (value != 0.0 && value != 1.0 && value != 2.0) return fail(FAP_ERR_INVALID, "stage1 is 0, 1 or 2");
    G->stage1 = (int)value;
    G->last_ids.clear();
    return FAP_OK;
  }
  if (std::strcmp(key, "bgraph_form") == 0) {
    if (value != 0.0 && value != 1.0 && value != 2.0) return fail(FAP_ERR_INVALID, "bgraph_form is 0, 1 or 2");
    G->bgraph_form = (int)value;
    G->last_ids.clear();
    G->epoch++;
    return FAP_OK;
  }
  if (std::strcmp(key, "paths") == 0) {
    if (value == 0.0) {
      G->paths = false;
      return FAP_OK;
    }
    return enable_paths(G);
  }
  if (std::strcmp(key, "use_cache") == 0) {
    G->use_cache = value != 0.0;
    G->last_ids.clear();
    return FAP_OK;
  }
  if (std::strcmp(key, "floyd_queue") == 0) {
    G->floyd_queue = value != 0.0;
    return FAP_OK;
  }
  if (std::strcmp(key, "thin_max_b") == 0) {
    if (!(value >= 0.0) || value > kThinBoundary)
      return fail(FAP_ERR_INVALID, "thin_max_b is in [0, %d]", kThinBoundary);
    G->thin_max_b = (int)value;
    G->last_ids.clear();
    return FAP_OK;
  }
  if (std::strcmp(key, "floyd_symmetric") == 0) {
    G->floyd_sym = value != 0.0;
    G->last_ids.clear();
    return FAP_OK;
  }
  if (std::strcmp(key, "minplus_pack16") == 0) {
    G->pack16 = value != 0.0;
    G->last_ids.clear();
    return FAP_OK;
  }
  if (std::strcmp(key, "minplus_prepack") == 0) {
    G->prepack = value != 0.0;
    G->last_ids.clear();
    return FAP_OK;
  }
  if (std::strcmp(key, "floyd_per_cta") == 0) {
    G->floyd_per_cta = value != 0.0;
    return FAP_OK;
  }
  if (std::strcmp(key, "sssp_max_rounds") == 0) {
    G->sssp_max_rounds = value >= 1 ? (int64_t)value : -1;
    return FAP_OK;
  }
  if (std::strcmp(key, "max_resident_rows") == 0) {
    G->row_limit = value >= 1 ? (int64_t)value : 0;
    // Blocks reserved beyond the new bound are given back at once.
    if (G->row_limit > 0 && G->max_rows > G->row_limit) return fap_graph_release(G);
    return FAP_OK;
  }
  return fail(FAP_ERR_INVALID, "unknown parameter '%s'", key);
} catch (...) {
  return fail_exception();
}

// ---------------------------------------------------------------------------
// SSSP bucket-width tuning: times the SSSP stage on a sample of the graph's
// boundary sources (one wave of CTAs) for each candidate delta and keeps the
// fastest.
// ---------------------------------------------------------------------------
namespace {
template <typename T>
int tune_sssp_impl(fap_dgraph *G, const double *deltas, int32_t count, int32_t sample,
                   double *best_delta, float *ms_out) {
  fap_ctx *c = G->ctx;
  cudaStream_t st = c->stream;
  const int64_t n = G->n;
  // boundary sources of every part, in sorted-position space
  std::vector<int32_t> all;
  for (int32_t p = 1; p <= G->K; p++)
    for (int32_t k = 0; k < G->bnum[p]; k++) all.push_back(G->voff[p] + k);
  if (all.empty()) return fail(FAP_ERR_STATE, "graph has no boundary vertices to tune on");
  const int want = sample > 0 ? sample : sssp_scratch_rows(G->n, (int)all.size());
  const int ns = std::max(1, std::min<int>(want, (int)all.size()));
  std::vector<int32_t> src(ns);
  for (int i = 0; i < ns; i++) src[i] = all[(int64_t)i * (int64_t)all.size() / ns];
  DevBuf d_src, rows, scratch;
  FAP_TRY(d_src.ensure((size_t)ns * 4));
  FAP_TRY(rows.ensure((size_t)ns * n * 4));
  FAP_TRY(scratch.ensure((size_t)std::max(sssp_scratch_rows(G->n, ns), 1) * n * 4));
  FAP_CK(cudaMemcpy(d_src.p, src.data(), (size_t)ns * 4, cudaMemcpyHostToDevice));
  const int64_t rounds = G->sssp_max_rounds > 0 ? G->sssp_max_rounds : 8 * n + 1024;
  double best = -1.0;
  float best_ms = 1e30f;
  int64_t L = 0;
  for (int32_t i = 0; i < count; i++) {
    const double dd = deltas[i];
    double d = (dd > 0 && dd < (double)Dist<T>::inf()) ? dd : (double)Dist<T>::inf();
    if (Dist<T>::kDtype == FAP_DTYPE_I32) d = std::max(1.0, std::floor(d));
    float t_best = 1e30f;
    for (int rep = 0; rep < 2; rep++) {
      FAP_CK(cudaMemsetAsync(G->d_status.p, 0, sizeof(int), st));
      FAP_CK(cudaEventRecord(c->ev[0], st));
      FAP_CK(launch_sssp<T>(G->ro_s.as<int32_t>(), G->col_s.as<int32_t>(), G->w_s.as<T>(), G->n,
                            d_src.as<int32_t>(), nullptr, ns, rows.as<T>(), n, n,
                            G->d_ed2st.as<int32_t>(), scratch.as<T>(), (T)d, G->sssp_chain,
                            G->sssp_precheck, rounds,
                            G->d_status.as<int>(), st, &L));
      FAP_CK(cudaEventRecord(c->ev[1], st));
      FAP_CK(cudaEventSynchronize(c->ev[1]));
      FAP_TRY(read_status(G));
      float t;
      FAP_CK(cudaEventElapsedTime(&t, c->ev[0], c->ev[1]));
      if (rep > 0 || count == 1) t_best = std::min(t_best, t);
    }
    if (ms_out) ms_out[i] = t_best;
    if (t_best < best_ms) {
      best_ms = t_best;
      best = dd;
    }
  }
  d_src.release();
  rows.release();
  scratch.release();
  G->sssp_delta = (best > 0 && best < 1e8) ? best : -2.0;  // -2: plain Bellman-Ford chosen
  G->epoch++;
  if (best_delta) *best_delta = best;
  return FAP_OK;
}
}  // namespace

extern "C" int fap_graph_tune_sssp(fap_dgraph *G, const double *deltas, int32_t count, int32_t sample,
                                   double *best_delta, float *ms_out) try {
  if (!G || !deltas || count <= 0) return fail(FAP_ERR_INVALID, "need a graph and candidate deltas");
  if (G->K == 0) return fail(FAP_ERR_STATE, "tune before fap_graph_set_parts");
  DeviceGuard g(G->ctx->device);
  return G->dtype == FAP_DTYPE_I32 ? tune_sssp_impl<int32_t>(G, deltas, count, sample, best_delta, ms_out)
                                   : tune_sssp_impl<float>(G, deltas, count, sample, best_delta, ms_out);
} catch (...) {
  return fail_exception();
}

extern "C" double fap_graph_mean_weight(const fap_dgraph *G) { return G ? G->mean_w : 0.0; }

// ---------------------------------------------------------------------------
// Memory release and asynchronous distance rows (used by the serving loop)
// ---------------------------------------------------------------------------
extern "C" int fap_graph_pack16_tiles(fap_dgraph *G, int64_t *packed, int64_t *total) try {
  if (!G || !packed || !total) return fail(FAP_ERR_INVALID, "NULL argument");
  *packed = *total = 0;
  if (!G->d_pk_tiles.p) return FAP_OK;
  DeviceGuard g(G->ctx->device);
  unsigned long long h[2] = {0, 0};
  FAP_CK(cudaMemcpyAsync(h, G->d_pk_tiles.p, sizeof(h), cudaMemcpyDeviceToHost, G->ctx->stream));
  FAP_CK(cudaStreamSynchronize(G->ctx->stream));
  *packed = (int64_t)h[0];
  *total = (int64_t)h[1];
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_expand16_tiles(fap_dgraph *G, int64_t *packed, int64_t *total) try {
  if (!G || !packed || !total) return fail(FAP_ERR_INVALID, "NULL argument");
  *packed = *total = 0;
  if (!G->d_xk_tiles.p) return FAP_OK;
  DeviceGuard g(G->ctx->device);
  unsigned long long h[2] = {0, 0};
  FAP_CK(cudaMemcpyAsync(h, G->d_xk_tiles.p, sizeof(h), cudaMemcpyDeviceToHost, G->ctx->stream));
  FAP_CK(cudaStreamSynchronize(G->ctx->stream));
  *packed = (int64_t)h[0];
  *total = (int64_t)h[1];
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_release(fap_dgraph *G) try {
  if (!G) return fail(FAP_ERR_INVALID, "NULL graph");
  DeviceGuard g(G->ctx->device);
  FAP_CK(cudaStreamSynchronize(G->ctx->stream));
  G->D.release();
  G->F.release();
  G->sssp_scratch.release();
  G->staging.release();
  G->d_checks.release();
  G->P.release();
  G->d_dB.release();
  G->d_FB.release();
  G->d_bTc.release();
  G->bTc_maxb = 0;
  G->d_pk_off.release();
  G->d_pk_range.release();
  G->d_pk_maxa.release();
  G->d_pk_s16.release();
  G->d_pk_at.release();
  G->d_pk_krow.release();
  G->d_xk_ap.release();
  G->d_xk_bd.release();
  for (auto &cs : G->cslot) {
    if (cs.stream) FAP_CK(cudaStreamSynchronize(cs.stream));
    cs.busy = false;
    cs.staging.release();
  }
  G->max_rows = 0;
  std::fill(G->row_base.begin(), G->row_base.end(), -1);
  G->last_ids.clear();
  G->epoch++;
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_device_bytes(const fap_dgraph *G, int64_t *bytes) try {
  if (!G || !bytes) return fail(FAP_ERR_INVALID, "NULL argument");
  int64_t t = 0;
  for (const DevBuf *b : {&G->ro, &G->col, &G->w, &G->ro_s, &G->col_s, &G->w_s, &G->sssp_scratch,
                          &G->d_thin, &G->d_gid, &G->d_st2ed, &G->d_ed2st, &G->D, &G->F, &G->d_parts,
                          &G->d_work, &G->d_src, &G->d_srcrows, &G->d_status, &G->d_checks, &G->staging,
                          &G->cBd, &G->cF, &G->d_cparts, &G->d_rowgroups, &G->d_rowloc, &G->d_rowout,
                          &G->d_rowidx, &G->P, &G->d_tro, &G->d_tcol, &G->d_tw, &G->d_dB,
                          &G->d_bpart, &G->d_brows, &G->d_FB, &G->d_msbf_items, &G->d_msbf_act,
                          &G->d_msbf_changed, &G->d_bitro, &G->d_bitcol, &G->d_botro, &G->d_botcol, &G->d_bitw, &G->d_bitems,
                          &G->d_bDt, &G->d_bact, &G->d_bpact, &G->d_bgpart, &G->d_bpcolmap, &G->d_grow,
                          &G->d_bTc, &G->d_pk_off, &G->d_pk_range, &G->d_pk_maxa, &G->d_pk_tiles, &G->d_pk_s16,
                          &G->d_pk_at, &G->d_pk_krow, &G->d_xk_off, &G->d_xk_range, &G->d_xk_maxb, &G->d_xk_tiles,
                          &G->d_xk_ap, &G->d_xk_bd})
    t += (int64_t)b->bytes;
  *bytes = t;
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_resident(fap_dgraph *G, int32_t part) try {
  if (!G || part < 1 || part > G->K) return 0;
  return G->row_base[part] >= 0 ? 1 : 0;
} catch (...) {
  return fail_exception();
}

// ---------------------------------------------------------------------------
// Resident cache (stages 1-2 of every part, kept in HBM for serving)
// ---------------------------------------------------------------------------
namespace {

struct CacheShape {
  int32_t ldf = kFloydTile, max_b = 0, max_s = 0;
  int64_t total_b = 0;
  int64_t bytes(const fap_dgraph *G) const {
    // boundary rows + Floyd squares + descriptors + the sources' lists
    auto a = [](int64_t b) { return (int64_t)alloc_size((size_t)b); };
    return a(std::max<int64_t>(total_b, 1) * G->ldD * 4) + a((int64_t)G->K * ldf * ldf * 4) +
           a((int64_t)G->K * (int64_t)sizeof(PartDesc)) + a(std::max<int64_t>(total_b, 1) * 4) +
           a(std::max<int64_t>(total_b, 1) * 8);
  }
};

CacheShape cache_shape(const fap_dgraph *G) {
  CacheShape c;
  for (int32_t p = 1; p <= G->K; p++) {
    c.ldf = std::max<int32_t>(c.ldf, (int32_t)round_up(std::max(G->vnum[p], 1), kFloydTile));
    c.max_b = std::max(c.max_b, G->bnum[p]);
    c.max_s = std::max(c.max_s, G->vnum[p]);
    c.total_b += G->bnum[p];
  }
  return c;
}

template <typename T>
int cache_build_impl(fap_dgraph *G) {
  fap_ctx *c = G->ctx;
  cudaStream_t st = c->stream;
  const int32_t K = G->K;
  const CacheShape cs = cache_shape(G);
  if (cs.total_b > INT32_MAX) return fail(FAP_ERR_RANGE, "too many boundary vertices for the cache");
  FAP_CK(cudaStreamSynchronize(st));
  FAP_TRY(G->cBd.ensure((size_t)std::max<int64_t>(cs.total_b, 1) * G->ldD * 4));
  FAP_TRY(G->cF.ensure((size_t)K * cs.ldf * cs.ldf * 4));
  G->cb_off.assign(K + 2, 0);
  for (int32_t p = 1; p <= K; p++) G->cb_off[p + 1] = G->cb_off[p] + G->bnum[p];
  G->cparts.clear();
  std::vector<int32_t> src;
  std::vector<int64_t> srows;
  const bool bm = bmethod_ok(G);
  for (int32_t p = 1; p <= K; p++) {
    PartDesc d{};
    d.part = p;
    d.start = G->voff[p];
    d.s = G->vnum[p];
    d.b = G->bnum[p];
    d.row_base = G->cb_off[p];
    d.ldf = cs.ldf;
    d.f_off = (int64_t)(p - 1) * cs.ldf * cs.ldf;
    d.bd_row = (int32_t)G->cb_off[p];
    d.flags = bm ? kPartLocal : 0;
    d.bd_col = G->bpcol[p];
    G->cparts.push_back(d);
    for (int32_t k = 0; k < d.b; k++) {
      src.push_back(d.start + k);
      srows.push_back(d.row_base + k);
    }
  }
  FAP_TRY(G->d_cparts.ensure(G->cparts.size() * sizeof(PartDesc)));
  FAP_TRY(G->d_src.ensure(std::max<size_t>(src.size(), 1) * 4));
  FAP_TRY(G->d_srcrows.ensure(std::max<size_t>(srows.size(), 1) * 8));
  if (!bm && !use_msbf(G))  // (the tiled form sizes its own tiles)
    FAP_TRY(G->sssp_scratch.ensure(
        (size_t)std::max(sssp_scratch_rows(G->n, (int)src.size()), 1) * (size_t)G->n * 4));
  {
    int32_t mnb = 0;
    G->cq.sym = bm && G->sym_local && G->floyd_sym;
    const std::vector<QItem> qitems = floyd_queue_items(G->cparts, G->cq.sym, &G->cq.nfloyd, &mnb);
    G->cq.nitems = (int32_t)qitems.size();
    G->cq.stride = 2 + 2 * mnb;
    G->cq.nparts = (int32_t)G->cparts.size();
    FAP_TRY(G->cq.items.ensure(std::max<size_t>(qitems.size(), 1) * sizeof(QItem)));
    FAP_TRY(G->cq.cnt.ensure(((size_t)G->cq.nparts * G->cq.stride + 2) * 4));
    if (!qitems.empty())
      FAP_CK(cudaMemcpy(G->cq.items.p, qitems.data(), qitems.size() * sizeof(QItem), cudaMemcpyHostToDevice));
  }
  FAP_CK(cudaMemcpy(G->d_cparts.p, G->cparts.data(), G->cparts.size() * sizeof(PartDesc),
                    cudaMemcpyHostToDevice));
  if (!src.empty()) {
    FAP_CK(cudaMemcpy(G->d_src.p, src.data(), src.size() * 4, cudaMemcpyHostToDevice));
    FAP_CK(cudaMemcpy(G->d_srcrows.p, srows.data(), srows.size() * 8, cudaMemcpyHostToDevice));
  }
  G->last_ids.clear();  // d_src / d_srcrows now hold the cache's sources
  G->epoch++;
  const PartDesc *dp = G->d_cparts.as<const PartDesc>();
  T *Bd = G->cBd.as<T>();
  T *F = G->cF.as<T>();
  int *status = G->d_status.as<int>();
  const int32_t *gid = G->d_gid.as<const int32_t>(), *st2ed = G->d_st2ed.as<const int32_t>(),
                *ed2st = G->d_ed2st.as<const int32_t>();
  const int64_t rounds = G->sssp_max_rounds > 0 ? G->sssp_max_rounds : 8 * (int64_t)G->n + 1024;
  int64_t L = 0;
  for (cudaEvent_t &ev : G->cev)
    if (!ev) FAP_CK(cudaEventCreate(&ev));
  FAP_CK(cudaMemsetAsync(status, 0, sizeof(int), st));
  if (bm) {
    // Boundary-graph form: local closures, boundary-graph APSP, expansion.
    FAP_TRY(prepare_bgraph(G, G->cparts));
    FAP_CK(cudaEventRecord(G->cev[0], st));
    FAP_CK(launch_gather<T>(dp, K, cs.ldf, G->ro.as<const int32_t>(), G->col.as<const int32_t>(),
                            G->w.as<const T>(), gid, st2ed, ed2st, Bd, G->ldD, F, st, &L));
    if (G->floyd_queue)
      FAP_CK(run_floyd_queue<T>(G, G->cq, dp, F, cs.ldf, false, nullptr, 0, Bd, 0, status, &L));
    else
      FAP_CK(launch_floyd_parts_multi<T>(dp, K, (int)ceil_div(cs.max_s, kFloydTile), F, cs.ldf, status, st, &L));
    FAP_CK(cudaEventRecord(G->cev[1], st));
    FAP_TRY(close_bgraph<T>(G, dp, K, cs.max_b, F, status, rounds, &L));
    FAP_CK(cudaEventRecord(G->cev[2], st));
    FAP_TRY(expand_bgraph<T>(G, dp, K, cs.max_s, F, Bd, cs.ldf, status, &L));
    FAP_CK(cudaEventRecord(G->cev[3], st));
    FAP_CK(launch_local_fixup<T>(dp, K, cs.max_s, F, G->d_FB.as<const T>(), cs.ldf, st, &L));
    FAP_CK(cudaEventRecord(G->cev[4], st));
    G->cache_bmethod = true;
    G->cache_stage1_name = stage1_form_name(G, true);
  } else {
  G->cache_stage1_name = stage1_form_name(G, false);
  FAP_CK(cudaEventRecord(G->cev[0], st));
  FAP_TRY(run_stage1_sssp<T>(G, G->d_src.as<const int32_t>(), G->d_srcrows.as<const int64_t>(),
                             (int)src.size(), Bd, status, rounds, &L));
  FAP_CK(cudaEventRecord(G->cev[1], st));
  FAP_CK(launch_gather<T>(dp, K, cs.ldf, G->ro.as<const int32_t>(), G->col.as<const int32_t>(),
                          G->w.as<const T>(), gid, st2ed, ed2st, Bd, G->ldD, F, st, &L));
  FAP_CK(cudaEventRecord(G->cev[2], st));
  G->cache_bmethod = false;
  if (G->floyd_per_cta) {
    FAP_CK(launch_floyd_parts<T>(dp, K, F, cs.ldf, Bd, G->ldD, st2ed, status, st, &L));
  } else if (G->floyd_queue) {
    FAP_CK(run_floyd_queue<T>(G, G->cq, dp, F, cs.ldf, true, nullptr, 0, Bd, 0, status, &L));
  } else {
    FAP_CK(launch_floyd_parts_multi<T>(dp, K, (int)ceil_div(cs.max_s, kFloydTile), F, cs.ldf, status,
                                       st, &L));
    FAP_CK(launch_bdy_scatter<T>(dp, K, F, Bd, G->ldD, st2ed, cs.max_b, cs.max_s, st, &L));
  }
  FAP_CK(cudaEventRecord(G->cev[3], st));
  FAP_CK(cudaEventRecord(G->cev[4], st));
  }
  G->cache_ldf = cs.ldf;
  G->cache_max_b = cs.max_b;
  G->cache_max_s = cs.max_s;
  G->cache_ready = true;
  G->cache_valid.clear();  // every part
  G->launches = L;
  c->launches += L;
  // The SSSP scratch (up to one row of n per resident CTA) is not needed by
  // the cached path: wait for the build and give it back.
  FAP_CK(cudaStreamSynchronize(st));
  for (int i = 0; i < 4; i++) FAP_CK(cudaEventElapsedTime(&G->cache_ms[i], G->cev[i], G->cev[i + 1]));
  G->sssp_scratch.release();
  return FAP_OK;
}

// Distance rows from the cache: boundary sources copy their cached row;
// inner sources take the min-plus of their closed Floyd row with the part's
// boundary rows (the block min-plus restricted to the requested rows).
template <typename T>
int rows_cached_impl(fap_dgraph *G, const int32_t *sources, int32_t count, float *d_out) {
  cudaStream_t st = G->ctx->stream;
  const int32_t K = G->K;
  std::vector<int64_t> gather;  // pairs: cache row, output row
  std::vector<std::vector<std::pair<int32_t, int64_t>>> inner(K + 1);
  for (int32_t r = 0; r < count; r++) {
    const int32_t v = sources[r];
    const int32_t p = G->gid[v];
    const int32_t i = G->ed2st[v] - G->voff[p];
    if (i < G->bnum[p]) {
      gather.push_back(G->cb_off[p] + i);
      gather.push_back(r);
    } else {
      inner[p].push_back({i, (int64_t)r});
    }
  }
  std::vector<RowGroup> groups;
  std::vector<int32_t> loc;
  std::vector<int64_t> orow;
  for (int32_t p = 1; p <= K; p++)
    for (size_t a = 0; a < inner[p].size(); a += kRowsGroup) {
      const int32_t cnt = (int32_t)std::min<size_t>(kRowsGroup, inner[p].size() - a);
      groups.push_back(RowGroup{p - 1, (int32_t)loc.size(), cnt, 0});
      for (int32_t j = 0; j < cnt; j++) {
        loc.push_back(inner[p][a + j].first);
        orow.push_back(inner[p][a + j].second);
      }
    }
  const int64_t ng = (int64_t)gather.size() / 2;
  std::vector<int64_t> gidx(ng), gout(ng);
  for (int64_t k = 0; k < ng; k++) {
    gidx[k] = gather[2 * k];
    gout[k] = gather[2 * k + 1];
  }
  // (grown in stream order: cudaFree would wait for the whole device, other
  // graphs' streams of a server included)
  FAP_TRY(G->d_rowgroups.ensure_async(std::max<size_t>(groups.size(), 1) * sizeof(RowGroup), st));
  FAP_TRY(G->d_rowloc.ensure_async(std::max<size_t>(loc.size(), 1) * 4, st));
  FAP_TRY(G->d_rowout.ensure_async(std::max<size_t>(orow.size(), 1) * 8, st));
  FAP_TRY(G->d_rowidx.ensure_async(std::max<size_t>(2 * ng, 1) * 8, st));
  FAP_CK(cudaStreamSynchronize(st));  // earlier launches may still read these buffers
  if (!groups.empty()) {
    FAP_CK(cudaMemcpy(G->d_rowgroups.p, groups.data(), groups.size() * sizeof(RowGroup), cudaMemcpyHostToDevice));
    FAP_CK(cudaMemcpy(G->d_rowloc.p, loc.data(), loc.size() * 4, cudaMemcpyHostToDevice));
    FAP_CK(cudaMemcpy(G->d_rowout.p, orow.data(), orow.size() * 8, cudaMemcpyHostToDevice));
  }
  if (ng > 0) {
    FAP_CK(cudaMemcpy(G->d_rowidx.p, gidx.data(), ng * 8, cudaMemcpyHostToDevice));
    FAP_CK(cudaMemcpy(G->d_rowidx.as<int64_t>() + ng, gout.data(), ng * 8, cudaMemcpyHostToDevice));
  }
  const int64_t n = G->n;
  T *out = reinterpret_cast<T *>(d_out);
  int64_t L = 0;
  FAP_CK(launch_row_gather<T>(G->cBd.as<const T>(), G->ldD, G->d_rowidx.as<const int64_t>(), ng, (int)n,
                              out, n, G->d_rowidx.as<const int64_t>() + ng, st, &L));
  FAP_CK(launch_minplus_rows<T>(G->d_cparts.as<const PartDesc>(), G->d_rowgroups.as<const RowGroup>(),
                                (int)groups.size(), G->d_rowloc.as<const int32_t>(),
                                G->d_rowout.as<const int64_t>(), G->cache_max_b, (int)n,
                                G->cF.as<const T>(), G->cBd.as<const T>(), G->ldD,
                                G->d_gid.as<const int32_t>(), G->d_ed2st.as<const int32_t>(), out, n, st, &L));
  if (Dist<T>::kDtype == FAP_DTYPE_I32)
    FAP_CK(launch_i32_to_f32(reinterpret_cast<int32_t *>(d_out), count, n, n, d_out, st, &L));
  G->ctx->launches += L;
  G->launches = L;
  return FAP_OK;
}
}  // namespace

extern "C" int fap_graph_cache_build(fap_dgraph *G) try {
  if (!G) return fail(FAP_ERR_INVALID, "NULL graph");
  if (G->K == 0) return fail(FAP_ERR_STATE, "fap_graph_cache_build before fap_graph_set_parts");
  if (G->cache_ready) return FAP_OK;
  DeviceGuard g(G->ctx->device);
  const int rc = G->dtype == FAP_DTYPE_I32 ? cache_build_impl<int32_t>(G) : cache_build_impl<float>(G);
  if (rc != FAP_OK) cache_drop(G);
  return rc;
} catch (...) {
  if (G) cache_drop(G);  // a half-built cache is not kept
  return fail_exception();
}

extern "C" int fap_graph_cache_rebuild(fap_dgraph *G) try {
  if (!G) return fail(FAP_ERR_INVALID, "NULL graph");
  if (G->K == 0) return fail(FAP_ERR_STATE, "fap_graph_cache_rebuild before fap_graph_set_parts");
  DeviceGuard g(G->ctx->device);
  const int rc = G->dtype == FAP_DTYPE_I32 ? cache_build_impl<int32_t>(G) : cache_build_impl<float>(G);
  if (rc != FAP_OK) cache_drop(G);
  return rc;
} catch (...) {
  if (G) cache_drop(G);  // a half-built cache is not kept
  return fail_exception();
}

// ---------------------------------------------------------------------------
// Sharded boundary-graph form: parts split over ranks (one process per GPU).
// Each rank closes its own parts locally, the ranks all-gather the boundary
// rows of those local closures, and each rank then closes the boundary graph
// itself (the same work on every rank), expands the boundary rows of its own
// parts and makes their closures exact, leaving them in the resident cache
// for fap_solve.  The layout of a rank's send buffer: its own parts in
// ascending order, each part's rows 0..b-1, columns 0..s-1 of its local
// closure, row-major.
// ---------------------------------------------------------------------------
namespace {
template <typename T>
int shard_begin_impl(fap_dgraph *G, void *send, int64_t send_cap, int64_t *send_elems) {
  fap_ctx *c = G->ctx;
  cudaStream_t st = c->stream;
  const int32_t K = G->K;
  const CacheShape cs = cache_shape(G);
  if (cs.total_b > INT32_MAX) return fail(FAP_ERR_RANGE, "too many boundary vertices for the cache");
  int64_t need = 0;
  for (const int32_t p : G->shard_own) need += (int64_t)G->bnum[p] * G->vnum[p];
  *send_elems = need;
  if (need > send_cap) return fail(FAP_ERR_INVALID, "send buffer holds %lld elements, %lld needed",
                                   (long long)send_cap, (long long)need);
  FAP_CK(cudaStreamSynchronize(st));
  FAP_TRY(G->cBd.ensure((size_t)std::max<int64_t>(cs.total_b, 1) * G->ldD * 4));
  FAP_TRY(G->cF.ensure((size_t)K * cs.ldf * cs.ldf * 4));
  G->cb_off.assign(K + 2, 0);
  for (int32_t p = 1; p <= K; p++) G->cb_off[p + 1] = G->cb_off[p] + G->bnum[p];
  G->cparts.clear();
  std::vector<PartDesc> own;
  for (int32_t p = 1; p <= K; p++) {
    PartDesc d{};
    d.part = p;
    d.start = G->voff[p];
    d.s = G->vnum[p];
    d.b = G->bnum[p];
    d.row_base = G->cb_off[p];
    d.ldf = cs.ldf;
    d.f_off = (int64_t)(p - 1) * cs.ldf * cs.ldf;
    d.bd_row = (int32_t)G->cb_off[p];
    d.flags = kPartLocal;
    d.bd_col = G->bpcol[p];
    G->cparts.push_back(d);
  }
  for (const int32_t p : G->shard_own) own.push_back(G->cparts[p - 1]);
  FAP_TRY(G->d_cparts.ensure(G->cparts.size() * sizeof(PartDesc)));
  FAP_TRY(G->d_cown.ensure(std::max<size_t>(own.size(), 1) * sizeof(PartDesc)));
  {
    int32_t mnb = 0;
    G->cq.sym = G->sym_local && G->floyd_sym;
    const std::vector<QItem> qitems = floyd_queue_items(own, G->cq.sym, &G->cq.nfloyd, &mnb);
    G->cq.nitems = (int32_t)qitems.size();
    G->cq.stride = 2 + 2 * mnb;
    G->cq.nparts = (int32_t)own.size();
    FAP_TRY(G->cq.items.ensure(std::max<size_t>(qitems.size(), 1) * sizeof(QItem)));
    FAP_TRY(G->cq.cnt.ensure(((size_t)G->cq.nparts * G->cq.stride + 2) * 4));
    if (!qitems.empty())
      FAP_CK(cudaMemcpy(G->cq.items.p, qitems.data(), qitems.size() * sizeof(QItem), cudaMemcpyHostToDevice));
  }
  FAP_CK(cudaMemcpy(G->d_cparts.p, G->cparts.data(), G->cparts.size() * sizeof(PartDesc), cudaMemcpyHostToDevice));
  if (!own.empty())
    FAP_CK(cudaMemcpy(G->d_cown.p, own.data(), own.size() * sizeof(PartDesc), cudaMemcpyHostToDevice));
  G->last_ids.clear();
  G->epoch++;
  T *F = G->cF.as<T>();
  int *status = G->d_status.as<int>();
  int64_t L = 0;
  FAP_CK(cudaMemsetAsync(status, 0, sizeof(int), st));
  if (!own.empty()) {
    // local closures of the own parts (their slots of the cache's arena)
    FAP_CK(launch_gather<T>(G->d_cown.as<const PartDesc>(), (int)own.size(), cs.ldf, G->ro.as<const int32_t>(),
                            G->col.as<const int32_t>(), G->w.as<const T>(), G->d_gid.as<const int32_t>(),
                            G->d_st2ed.as<const int32_t>(), G->d_ed2st.as<const int32_t>(), G->cBd.as<T>(),
                            G->ldD, F, st, &L));
    FAP_CK(run_floyd_queue<T>(G, G->cq, G->d_cown.as<const PartDesc>(), F, cs.ldf, false, nullptr, 0,
                              G->cBd.as<T>(), 0, status, &L, (int)K));
    // their boundary rows, packed
    int64_t off = 0;
    for (const PartDesc &d : own) {
      if (d.b > 0)
        FAP_CK(cudaMemcpy2DAsync(static_cast<T *>(send) + off, (size_t)d.s * 4, F + d.f_off, (size_t)cs.ldf * 4,
                                 (size_t)d.s * 4, (size_t)d.b, cudaMemcpyDeviceToDevice, st));
      off += (int64_t)d.b * d.s;
    }
  }
  G->launches = L;
  c->launches += L;
  FAP_TRY(read_status(G));
  G->cache_ldf = cs.ldf;
  G->cache_max_b = cs.max_b;
  G->cache_max_s = cs.max_s;
  G->shard_begun = true;
  return FAP_OK;
}

template <typename T>
int shard_finish_impl(fap_dgraph *G, const void *recv, int32_t world, const int32_t *owner, int64_t stride) {
  fap_ctx *c = G->ctx;
  cudaStream_t st = c->stream;
  const int32_t K = G->K;
  const int64_t ldf = G->cache_ldf;
  T *F = G->cF.as<T>();
  const T *R = static_cast<const T *>(recv);
  std::vector<char> mine((size_t)K + 1, 0);
  for (const int32_t p : G->shard_own) mine[p] = 1;
  // other ranks' boundary rows into their parts' slots
  std::vector<int64_t> off((size_t)world, 0);
  for (int32_t p = 1; p <= K; p++) {
    const int32_t r = owner[p];
    const PartDesc &d = G->cparts[p - 1];
    const int64_t elems = (int64_t)d.b * d.s;
    if (off[r] + elems > stride) return fail(FAP_ERR_INVALID, "rank %d's parts exceed the stride", r);
    if (!mine[p] && d.b > 0)
      FAP_CK(cudaMemcpy2DAsync(F + d.f_off, (size_t)ldf * 4, R + (int64_t)r * stride + off[r], (size_t)d.s * 4,
                               (size_t)d.s * 4, (size_t)d.b, cudaMemcpyDeviceToDevice, st));
    off[r] += elems;
  }
  FAP_CK(cudaStreamSynchronize(st));
  FAP_TRY(prepare_bgraph(G, G->cparts));
  // the staged expansion writes only the listed rows: the own parts' first
  int64_t nrows = -1;
  if (!bgraph_bf(G) && !bgraph_tiled_expand(G)) {
    std::vector<int64_t> rows;
    for (const int32_t p : G->shard_own) {
      const PartDesc &d = G->cparts[p - 1];
      for (int32_t k = 0; k < d.b; k++) {
        rows.push_back(G->boff[p] + k);
        rows.push_back(d.row_base + k);
      }
    }
    nrows = (int64_t)rows.size() / 2;
    if (!rows.empty())
      FAP_CK(cudaMemcpy(G->d_brows.p, rows.data(), rows.size() * 8, cudaMemcpyHostToDevice));
  }
  const PartDesc *dp = G->d_cparts.as<const PartDesc>();
  T *Bd = G->cBd.as<T>();
  int *status = G->d_status.as<int>();
  const int64_t rounds = G->sssp_max_rounds > 0 ? G->sssp_max_rounds : 8 * (int64_t)G->n + 1024;
  int64_t L = 0;
  FAP_CK(cudaMemsetAsync(status, 0, sizeof(int), st));
  FAP_TRY(close_bgraph<T>(G, dp, K, G->cache_max_b, F, status, rounds, &L));
  FAP_TRY(expand_bgraph<T>(G, dp, K, G->cache_max_s, F, Bd, ldf, status, &L, nrows));
  if (!G->shard_own.empty())
    FAP_CK(launch_local_fixup<T>(G->d_cown.as<const PartDesc>(), (int)G->shard_own.size(), G->cache_max_s, F,
                                 G->d_FB.as<const T>(), ldf, st, &L));
  G->launches = L;
  c->launches += L;
  FAP_TRY(read_status(G));
  G->cache_bmethod = true;
  G->cache_stage1_name = std::string("sharded ") + stage1_form_name(G, true);
  G->cache_ready = true;
  G->cache_valid = mine;
  G->last_ids.clear();
  G->epoch++;
  return FAP_OK;
}
}  // namespace

extern "C" int fap_graph_shard_begin(fap_dgraph *G, const int32_t *own_parts, int32_t count, void *send,
                                     int64_t send_cap, int64_t *send_elems) try {
  if (!G || !send_elems || (count > 0 && (!own_parts || !send))) return fail(FAP_ERR_INVALID, "NULL argument");
  if (G->K == 0) return fail(FAP_ERR_STATE, "fap_graph_shard_begin before fap_graph_set_parts");
  if (!bmethod_ok(G) || !G->floyd_queue)
    return fail(FAP_ERR_STATE, "the sharded form needs the boundary-graph form of stage 1 (an int32 graph "
                               "without duplicate arcs inside a part) and the Floyd work queue");
  std::vector<char> seen((size_t)G->K + 1, 0);
  std::vector<int32_t> own;
  for (int32_t i = 0; i < count; i++) {
    const int32_t p = own_parts[i];
    if (p < 1 || p > G->K || seen[p]) return fail(FAP_ERR_INVALID, "bad or repeated part id %d", p);
    seen[p] = 1;
    own.push_back(p);
  }
  std::sort(own.begin(), own.end());
  DeviceGuard g(G->ctx->device);
  cache_drop(G);
  G->shard_own = own;
  const int rc = G->dtype == FAP_DTYPE_I32 ? shard_begin_impl<int32_t>(G, send, send_cap, send_elems)
                                           : shard_begin_impl<float>(G, send, send_cap, send_elems);
  if (rc != FAP_OK) cache_drop(G);
  return rc;
} catch (...) {
  if (G) cache_drop(G);
  return fail_exception();
}

extern "C" int fap_graph_shard_finish(fap_dgraph *G, const void *recv, int32_t world, const int32_t *owner,
                                      int64_t stride) try {
  if (!G || !recv || !owner) return fail(FAP_ERR_INVALID, "NULL argument");
  if (!G->shard_begun) return fail(FAP_ERR_STATE, "fap_graph_shard_finish before fap_graph_shard_begin");
  if (world < 1 || stride < 0) return fail(FAP_ERR_INVALID, "bad world or stride");
  for (int32_t p = 1; p <= G->K; p++)
    if (owner[p] < 0 || owner[p] >= world) return fail(FAP_ERR_INVALID, "part %d: owner %d outside 0..%d", p,
                                                       owner[p], world - 1);
  // this rank's parts are exactly the parts of one owner rank
  if (!G->shard_own.empty()) {
    const int32_t r0 = owner[G->shard_own[0]];
    std::vector<char> mine((size_t)G->K + 1, 0);
    for (const int32_t p : G->shard_own) mine[p] = 1;
    for (int32_t p = 1; p <= G->K; p++)
      if ((owner[p] == r0) != (mine[p] != 0))
        return fail(FAP_ERR_INVALID, "owner[] does not give this rank's parts (part %d)", p);
  }
  DeviceGuard g(G->ctx->device);
  const int rc = G->dtype == FAP_DTYPE_I32 ? shard_finish_impl<int32_t>(G, recv, world, owner, stride)
                                           : shard_finish_impl<float>(G, recv, world, owner, stride);
  if (rc != FAP_OK) cache_drop(G);
  return rc;
} catch (...) {
  if (G) cache_drop(G);
  return fail_exception();
}

extern "C" int fap_graph_cache_timing(const fap_dgraph *G, float *ms4) try {
  if (!G || !ms4) return fail(FAP_ERR_INVALID, "NULL argument");
  if (!G->cache_ready) return fail(FAP_ERR_STATE, "no resident cache");
  for (int i = 0; i < 4; i++) ms4[i] = G->cache_ms[i];
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_cache_release(fap_dgraph *G) try {
  if (!G) return fail(FAP_ERR_INVALID, "NULL graph");
  DeviceGuard g(G->ctx->device);
  FAP_CK(cudaStreamSynchronize(G->ctx->stream));
  cache_drop(G);
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

extern "C" int fap_graph_cache_bytes(const fap_dgraph *G, int64_t *bytes, int *built) try {
  if (!G || !bytes) return fail(FAP_ERR_INVALID, "NULL argument");
  if (G->K == 0) return fail(FAP_ERR_STATE, "no partition");
  if (built) *built = G->cache_ready ? 1 : 0;
  if (G->cache_ready) {
    *bytes = (int64_t)(G->cBd.bytes + G->cF.bytes + G->d_cparts.bytes);
    if (G->cache_bmethod)  // the boundary graph's buffers stay for rebuilds
      for (const DevBuf *b : {&G->d_dB, &G->d_FB, &G->d_bitro, &G->d_bitcol, &G->d_botro, &G->d_botcol, &G->d_bitw, &G->d_bitems, &G->d_bDt,
                              &G->d_bact, &G->d_bpact, &G->d_bgpart, &G->d_bpcolmap, &G->d_grow})
        *bytes += (int64_t)b->bytes;
  } else {
    // plus what the build needs while it runs: the SSSP scratch, or the
    // boundary-graph matrix and tables
    const CacheShape cs = cache_shape(G);
    if (bmethod_ok(G)) {
      const int64_t ldB =
          round_up(std::max<int64_t>(bgraph_bf(G) ? G->bpcol[G->K + 1] : G->total_b, 1), kFloydTile);
      *bytes = cs.bytes(G) + (int64_t)alloc_size((size_t)(ldB * ldB * 4)) +
               (int64_t)alloc_size((size_t)std::max<int64_t>(G->total_b, 1) * cs.ldf * 4) +
               (int64_t)alloc_size((size_t)(G->K + 1) * sizeof(BPart)) +
               (int64_t)alloc_size((size_t)std::max<int64_t>(2 * G->total_b, 2) * 8);
      if (bgraph_tiled_expand(G)) *bytes += (int64_t)alloc_size((size_t)G->total_b * 8);
      if (bgraph_bf(G)) {  // cross-arc CSR, work lists, tiles, stamps, part table
        const int64_t xe = std::max<int64_t>(G->bgraph_cross, 1);
        *bytes += 3 * (int64_t)alloc_size((size_t)(G->total_b + 1) * 4) + 3 * (int64_t)alloc_size((size_t)xe * 4) +
                  (int64_t)alloc_size((size_t)2 * bgraph_ztiles(G) * G->total_b * 4 + 4 * sizeof(int)) +
                  (int64_t)alloc_size((size_t)bgraph_ztiles(G) * G->total_b * kMsbfS * 4) +
                  (int64_t)alloc_size((size_t)3 * bgraph_ztiles(G) * G->total_b * 4) +
                  (int64_t)alloc_size((size_t)bgraph_ztiles(G) * (G->K + 1) * 4);
      }
    } else {
      const int cnt = (int)std::min<int64_t>(cs.total_b, INT32_MAX);
      if (use_msbf(G))  // tiles, bitmaps, work items
        *bytes = cs.bytes(G) + (int64_t)alloc_size((size_t)msbf_ztiles(G, cnt) * G->n * kMsbfS * 4) +
                 (int64_t)alloc_size((size_t)2 * msbf_ztiles(G, cnt) * ceil_div(G->n, 32) * 4) +
                 (int64_t)alloc_size((size_t)(G->m / 32 + G->n + 1) * sizeof(MsbfItem));
      else
        *bytes = cs.bytes(G) + (int64_t)alloc_size((size_t)std::max(sssp_scratch_rows(G->n, cnt), 1) *
                                                   (size_t)G->n * 4);
    }
  }
  return FAP_OK;
} catch (...) {
  return fail_exception();
}

namespace {
template <typename T>
int rows_async_impl(fap_dgraph *G, const int32_t *sources, int32_t count, float *d_out) {
  cudaStream_t st = G->ctx->stream;
  const int64_t n = G->n;
  std::vector<int32_t> work(sources, sources + count);
  const bool relabel = G->K > 0;
  if (relabel)
    for (auto &x : work) x = G->ed2st[x];
  FAP_TRY(G->d_src.ensure(std::max<size_t>((size_t)count, G->d_src.bytes / 4) * 4));
  // the batch descriptors on the device no longer match d_src
  G->last_ids.clear();
  FAP_CK(cudaMemcpyAsync(G->d_src.p, work.data(), (size_t)count * 4, cudaMemcpyHostToDevice, st));
  FAP_CK(cudaStreamSynchronize(st));  // the host vector goes out of scope
  FAP_CK(cudaMemsetAsync(G->d_status.p, 0, sizeof(int), st));
  const int64_t rounds = G->sssp_max_rounds > 0 ? G->sssp_max_rounds : 8 * n + 1024;
  int64_t L = 0;
  T *out = reinterpret_cast<T *>(d_out);
  if (relabel) {
    FAP_TRY(G->sssp_scratch.ensure((size_t)std::max(sssp_scratch_rows(G->n, count), 1) * n * 4));
    FAP_CK(launch_sssp<T>(G->ro_s.as<int32_t>(), G->col_s.as<int32_t>(), G->w_s.as<T>(), G->n,
                          G->d_src.as<int32_t>(), nullptr, count, out, n, n, G->d_ed2st.as<int32_t>(),
                          G->sssp_scratch.as<T>(), sssp_delta_for<T>(G), G->sssp_chain, G->sssp_precheck,
                          rounds, G->d_status.as<int>(), st, &L));
  } else {
    FAP_CK(launch_sssp<T>(G->ro.as<int32_t>(), G->col.as<int32_t>(), G->w.as<T>(), G->n,
                          G->d_src.as<int32_t>(), nullptr, count, out, n, n, nullptr, nullptr,
                          sssp_delta_for<T>(G), G->sssp_chain, G->sssp_precheck, rounds,
                          G->d_status.as<int>(), st, &L));
  }
  if (Dist<T>::kDtype == FAP_DTYPE_I32)
    FAP_CK(launch_i32_to_f32(reinterpret_cast<int32_t *>(d_out), count, n, n, d_out, st, &L));
  G->ctx->launches += L;
  G->launches = L;
  G->epoch++;
  return FAP_OK;
}
}  // namespace

extern "C" int fap_graph_rows_async(fap_dgraph *G, const int32_t *sources, int32_t count, float *d_out) try {
  if (!G || (count > 0 && (!sources || !d_out))) return fail(FAP_ERR_INVALID, "NULL argument");
  if (count < 0) return fail(FAP_ERR_INVALID, "negative count");
  if (count == 0) return FAP_OK;
  for (int32_t i = 0; i < count; i++)
    if (sources[i] < 0 || sources[i] >= G->n) return fail(FAP_ERR_INVALID, "source %d out of range", sources[i]);
  DeviceGuard g(G->ctx->device);
  if (G->cache_ready && G->use_cache)
    return G->dtype == FAP_DTYPE_I32 ? rows_cached_impl<int32_t>(G, sources, count, d_out)
                                     : rows_cached_impl<float>(G, sources, count, d_out);
  return G->dtype == FAP_DTYPE_I32 ? rows_async_impl<int32_t>(G, sources, count, d_out)
                                   : rows_async_impl<float>(G, sources, count, d_out);
} catch (...) {
  return fail_exception();
}
