// Serving loop over resident graphs: continuous batching of sub-graph and
// distance-row requests, HBM-footprint admission, one stream per graph so
// batches of different graphs overlap on the GPU.  See include/fap_serve.h.
#include "fap_serve.h"

#include <cuda_runtime.h>

#include "fap_internal.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <exception>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

double now_s() {
  return std::chrono::duration<double>(Clock::now().time_since_epoch()).count();
}

struct Req {
  int64_t id = 0;
  int32_t graph = 0;
  int kind = FAP_REQ_SUBGRAPH;
  std::vector<int32_t> ids;
  float *host_out = nullptr;
  uint64_t *cs_out = nullptr;
  double t_submit = 0, t_start = 0, t_done = 0;
  int state = FAP_REQ_PENDING;
  int status = FAP_OK;
  int64_t rows = 0;
  int64_t entries = 0;
  int64_t row_off = 0;  // first row of the request in the batch's checksums / rows buffer
};

// Grows a pinned host buffer (rare: only when a batch is larger than every
// earlier one).
template <typename T>
bool grow_host(T **p, int64_t *cap, int64_t want) {
  if (want <= *cap) return true;
  if (*p) cudaFreeHost(*p);
  *p = nullptr;
  *cap = 0;
  if (cudaHostAlloc(reinterpret_cast<void **>(p), (size_t)want * sizeof(T), cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return false;
  }
  *cap = want;
  return true;
}

struct GSlot {
  fap_ctx *ctx = nullptr;
  fap_dgraph *dg = nullptr;
  int32_t n = 0, K = 0;
  int dtype = FAP_DTYPE_I32;
  int64_t ldD = 0;
  int64_t base_bytes = 0;  // CSR + partition, always resident
  std::vector<int32_t> vnum, voff, bnum;
  int64_t max_part = 0;        // largest part (rows)
  int64_t reserved_rows = 0;   // output rows the graph's D holds (0: released)
  // the batch in flight: distance rows, checksums on the device and their
  // pinned host copy, status word (buffers grow with the largest batch)
  // distance rows of the batch in flight: a small batch uses the graph's own
  // buffer (rows_small, at most kSmallRowsBytes), a larger one a block of the
  // server's pool freed after it (rows_pooled)
  float *rows_out = nullptr;
  bool rows_pooled = false;
  float *rows_small = nullptr;
  int64_t rows_small_cap = 0;
  uint64_t *cs_dev = nullptr;
  int64_t cs_cap = 0;
  uint64_t *cs_host = nullptr;
  int64_t cs_host_cap = 0;
  int32_t *status_host = nullptr;
  int64_t status_host_cap = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t start = nullptr, done = nullptr;  // around the batch in flight
  bool busy = false;
  int batch_kind = FAP_REQ_SUBGRAPH;
  std::vector<Req *> inflight;
  std::deque<Req *> pending;
  double last_used = 0;
};

}  // namespace

// Kinds of host calls the worker times (fap_server_stats 11..18).
enum HostStep : int {
  kStepLaunch = 0,     // one launch(): assembling and queueing a batch
  kStepComplete = 1,   // one complete(): retiring a finished batch
  kStepCache = 2,      // fap_graph_cache_build
  kStepRoom = 3,       // make_room (admission, evictions)
  kStepReserve = 4,    // fap_graph_reserve (output buffer growth)
  kStepSolve = 5,      // fap_solve of a sub-graph batch
  kStepRows = 6,       // rows buffer + fap_graph_rows_async
  kStepTail = 7,       // checksums, status and event queued after the batch
  kHostSteps = 8
};

constexpr int kMaxGraphs = 256;
constexpr int64_t kSmallRowsBytes = int64_t(32) << 20;

struct fap_server {
  int device = 0;
  // limits (fap_server_set_option may change them while the worker runs)
  std::atomic<int64_t> budget{0};
  std::atomic<int64_t> max_batch_rows{0};
  std::atomic<int64_t> max_batch_bytes{int64_t(512) << 20};
  // Stream-ordered pool shared by all graphs for the distance-row buffers of
  // the batches in flight: freed after each batch without synchronising the
  // device; up to a quarter of the budget stays mapped for reuse.
  cudaMemPool_t pool = nullptr;
  // Slots [0, ngraphs) are complete; fap_server_add_graph fills the next slot
  // before publishing it, so the worker never sees a slot being built.
  std::unique_ptr<GSlot> graphs[kMaxGraphs];
  std::atomic<int> ngraphs{0};
  std::mutex mu;
  std::mutex add_mu;  // serialises fap_server_add_graph
  std::condition_variable cv_work, cv_done;
  std::deque<Req *> incoming;
  std::unordered_map<int64_t, Req *> reqs;
  int64_t next_id = 1;
  int64_t outstanding = 0;  // submitted, not yet done/failed
  bool stop = false;
  std::thread worker;
  // Host time of the worker's calls, the longest single call of each kind
  // since the last reset (the worker is one thread, so a slow call delays
  // every graph's next batch): indices are the HostStep values.
  double host_max_ms[kHostSteps] = {};
  void note_host(int step, double t0) {
    const double ms = (now_s() - t0) * 1e3;
    std::lock_guard<std::mutex> lk(mu);
    host_max_ms[step] = std::max(host_max_ms[step], ms);
  }
  // stats (guarded by mu)
  std::vector<double> lat_ms;
  int64_t entries = 0, batches = 0, resident_hits = 0, peak_bytes = 0, cache_builds = 0, failed = 0;
  double busy_ms = 0;  // device time of finished batches

  void loop();
  bool complete(GSlot &g);
  bool launch(int gi);
  int64_t held_bytes();
  bool make_room(int64_t need, int self, bool *hopeless);
  void finish(Req *r, int state, int status);
};

namespace {
thread_local std::string s_err;
int serr(int code, const char *msg) {
  s_err = msg;
  return code;
}

// No C++ exception leaves an entry point of the server's C ABI.
int serr_exception() {
  try {
    throw;
  } catch (const std::bad_alloc &) {
    return serr(FAP_ERR_NOMEM, "host allocation failed");
  } catch (const std::exception &e) {
    return serr(FAP_ERR_INVALID, e.what());
  } catch (...) {
    return serr(FAP_ERR_INVALID, "unknown C++ exception");
  }
}
}  // namespace

namespace {
// Times one host call of the worker into fap_server::host_max_ms.
struct HostTimer {
  fap_server *s;
  int step;
  double t0;
  HostTimer(fap_server *srv, int st) : s(srv), step(st), t0(now_s()) {}
  ~HostTimer() { s->note_host(step, t0); }
};
}  // namespace

// Device bytes held: every graph's buffers and the server's per-graph
// batch buffers.
int64_t fap_server::held_bytes() {
  int64_t t = 0;
  const int ng = ngraphs.load(std::memory_order_acquire);
  for (int i = 0; i < ng; i++) {
    int64_t b = 0;
    if (fap_graph_device_bytes(graphs[i]->dg, &b) == FAP_OK) t += b;
    t += graphs[i]->cs_cap * 8 + graphs[i]->rows_small_cap * 4;
  }
  uint64_t pooled = 0;
  if (pool && cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &pooled) == cudaSuccess)
    t += (int64_t)pooled;
  return t;
}

namespace {
bool cache_built(const GSlot &g) {
  int64_t b = 0;
  int built = 0;
  return fap_graph_cache_bytes(g.dg, &b, &built) == FAP_OK && built;
}

// Bytes of g beyond its CSR, partition and resident cache.
int64_t output_bytes(const GSlot &g) {
  int64_t all = 0, cache = 0;
  int built = 0;
  fap_graph_device_bytes(g.dg, &all);
  if (fap_graph_cache_bytes(g.dg, &cache, &built) != FAP_OK || !built) cache = 0;
  return all - g.base_bytes - cache + g.cs_cap * 8 + g.rows_small_cap * 4;
}

void release_outputs(GSlot &g) {
  fap_graph_release(g.dg);
  g.reserved_rows = 0;
  if (g.cs_dev) cudaFree(g.cs_dev);
  g.cs_dev = nullptr;
  g.cs_cap = 0;
  if (g.rows_small) cudaFree(g.rows_small);
  g.rows_small = nullptr;
  g.rows_small_cap = 0;
}

// Grows a device buffer of the graph (frees the old one first: the graph
// is idle when its next batch is assembled).
template <typename T>
bool grow_dev(T **p, int64_t *cap, int64_t want) {
  if (want <= *cap) return true;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  if (cudaMalloc(reinterpret_cast<void **>(p), (size_t)want * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return false;
  }
  *cap = want;
  return true;
}
}  // namespace

// Frees memory until `need` more bytes fit in the budget: first the output
// buffers of idle graphs (least recently used first), then their resident
// caches, then graph `self`'s own output buffers.  Returns whether they fit;
// *hopeless is set when they cannot fit even after every busy graph
// finishes (nothing else holds memory that could be freed).
bool fap_server::make_room(int64_t need, int self, bool *hopeless) {
  HostTimer timer(this, kStepRoom);
  *hopeless = false;
  if (held_bytes() + need <= budget) return true;
  std::vector<int> idle;
  bool others_busy = false;
  const int ng = ngraphs.load(std::memory_order_acquire);
  for (int i = 0; i < ng; i++) {
    if (i == self) continue;
    if (graphs[i]->busy) others_busy = true;
    else idle.push_back(i);
  }
  std::sort(idle.begin(), idle.end(),
            [&](int a, int b) { return graphs[a]->last_used < graphs[b]->last_used; });
  if (pool) {  // pooled memory of finished batches first
    cudaMemPoolTrimTo(pool, 0);
    if (held_bytes() + need <= budget) return true;
  }
  for (int i : idle)
    if (output_bytes(*graphs[i]) > 0) {
      release_outputs(*graphs[i]);
      if (held_bytes() + need <= budget) return true;
    }
  for (int i : idle)
    if (cache_built(*graphs[i])) {
      fap_graph_cache_release(graphs[i]->dg);
      if (held_bytes() + need <= budget) return true;
    }
  if (output_bytes(*graphs[self]) > 0) {
    release_outputs(*graphs[self]);
    if (held_bytes() + need <= budget) return true;
  }
  *hopeless = !others_busy;
  return false;
}

void fap_server::finish(Req *r, int state, int status) {
  r->t_done = now_s();
  std::lock_guard<std::mutex> lk(mu);
  r->state = state;
  r->status = status;
  outstanding--;
  if (state == FAP_REQ_DONE) {
    lat_ms.push_back((r->t_done - r->t_submit) * 1e3);
    entries += r->entries;
  } else {
    failed++;
  }
  cv_done.notify_all();
}

// Retires g's finished batch: its status word and checksums are already in
// pinned host memory; distances asked for on the host are copied now.
bool fap_server::complete(GSlot &g) {
  HostTimer timer(this, kStepComplete);
  int rc = fap_status_code(*g.status_host);
  if (cudaEventQuery(g.done) != cudaSuccess) {
    cudaGetLastError();
    rc = FAP_ERR_CUDA;
  }
  float ms = 0.0f;
  if (cudaEventElapsedTime(&ms, g.start, g.done) == cudaSuccess) {
    std::lock_guard<std::mutex> lk(mu);
    busy_ms += ms;
  } else {
    cudaGetLastError();
  }
  const bool cs_ok = g.dtype == FAP_DTYPE_I32;
  for (Req *r : g.inflight) {
    int st = rc;
    if (st == FAP_OK && r->cs_out && cs_ok)
      std::memcpy(r->cs_out, g.cs_host + r->row_off, (size_t)r->rows * 8);
    if (st == FAP_OK && r->host_out) {
      if (r->kind == FAP_REQ_SUBGRAPH) {
        st = fap_graph_copy_block(g.dg, r->ids[0], r->host_out, FAP_DTYPE_F32);
      } else if (cudaMemcpyAsync(r->host_out, g.rows_out + r->row_off * g.n, (size_t)r->rows * g.n * 4,
                                 cudaMemcpyDeviceToHost, g.stream) != cudaSuccess ||
                 cudaStreamSynchronize(g.stream) != cudaSuccess) {
        cudaGetLastError();
        st = FAP_ERR_CUDA;
      }
    }
    finish(r, st == FAP_OK ? FAP_REQ_DONE : FAP_REQ_FAILED, st);
  }
  if (g.rows_out && g.rows_pooled) cudaFreeAsync(g.rows_out, g.stream);
  g.rows_out = nullptr;
  g.inflight.clear();
  g.busy = false;
  g.last_used = now_s();
  return true;
}

// Starts the next batch of graph gi, if one fits.  Returns whether anything
// was started or answered.
bool fap_server::launch(int gi) {
  HostTimer timer(this, kStepLaunch);
  GSlot &g = *graphs[gi];
  bool progressed = false;
  // Sub-graph requests whose block is still resident: answer at once (the
  // graph's stream is idle, so the copies do not wait on other work).
  while (!g.pending.empty()) {
    Req *r = g.pending.front();
    if (r->kind != FAP_REQ_SUBGRAPH || !fap_graph_resident(g.dg, r->ids[0])) break;
    g.pending.pop_front();
    r->t_start = now_s();
    int st = FAP_OK;
    if (r->host_out) st = fap_graph_copy_block(g.dg, r->ids[0], r->host_out, FAP_DTYPE_F32);
    if (st == FAP_OK && r->cs_out && g.dtype == FAP_DTYPE_I32)
      st = fap_graph_block_checksums(g.dg, r->ids[0], r->cs_out);
    {
      std::lock_guard<std::mutex> lk(mu);
      resident_hits++;
    }
    finish(r, st == FAP_OK ? FAP_REQ_DONE : FAP_REQ_FAILED, st);
    progressed = true;
  }
  if (g.pending.empty()) return progressed;
  cudaEventRecord(g.start, g.stream);
  // Resident cache (every part's boundary rows and closed Floyd matrix):
  // built on the graph's first batch when it fits, queued on the graph's
  // stream ahead of the batch.
  bool cached = cache_built(g);
  if (!cached) {
    int64_t cb = 0;
    int built = 0;
    bool hopeless = false;
    if (fap_graph_cache_bytes(g.dg, &cb, &built) == FAP_OK && make_room(cb, gi, &hopeless) &&
        [&] {
          HostTimer t(this, kStepCache);
          return fap_graph_cache_build(g.dg);
        }() == FAP_OK) {
      cached = true;
      std::lock_guard<std::mutex> lk(mu);
      cache_builds++;
    }
  }
  const int kind = g.pending.front()->kind;
  std::vector<Req *> batch;
  std::vector<int32_t> parts;
  std::vector<int64_t> part_row(g.K + 1, -1);  // first row of a batch part in the checksums
  // Batch buffers are sized once from the batch cap (output matrix, distance
  // rows, checksums), so that steady-state batches allocate nothing: only a
  // single request larger than the cap grows them.
  const int64_t cap = max_batch_bytes > 0 ? (int64_t)max_batch_bytes : INT64_MAX / 4;
  const int64_t row_bytes = kind == FAP_REQ_ROWS ? (int64_t)g.n * 4 : g.ldD * 4;
  int64_t limit_rows = std::max<int64_t>(1, cap / row_bytes);
  if (max_batch_rows > 0) limit_rows = std::min<int64_t>(limit_rows, max_batch_rows);
  if (kind == FAP_REQ_SUBGRAPH) limit_rows = std::min<int64_t>(std::max<int64_t>(limit_rows, g.max_part), g.n);
  // Device bytes the batch still needs beyond what the graph holds (upper
  // bounds of what fap_solve / fap_graph_copy_block / fap_graph_rows_async
  // allocate): the output matrix or rows buffer and the checksums up to
  // their target sizes; without the resident cache also one padded Floyd
  // square per part (all of the batch's largest side) and SSSP scratch rows
  // (at most one per source); the int32->float staging of the largest block
  // copied to the host.
  // When the buffers at their target size do not fit the budget, the batch
  // is sized exactly (its own rows only).
  int64_t rows = 0, nparts = 0, ldf = 0, srcs = 0, stage_rows = 0;
  bool exact = false;
  auto footprint = [&](int64_t r, int64_t np, int64_t lf, int64_t sc, int64_t sg) -> int64_t {
    const int64_t target = exact ? r : std::max(r, limit_rows);
    int64_t need = std::max<int64_t>(0, target - g.cs_cap) * 8 + sg * (int64_t)g.n * 4;
    if (kind == FAP_REQ_ROWS) {
      const int64_t b = r * (int64_t)g.n * 4;
      // (the small buffer grows to kSmallRowsBytes at once unless the batch is sized exactly)
      need += b > kSmallRowsBytes ? b : std::max<int64_t>(0, (exact ? b : kSmallRowsBytes) - g.rows_small_cap * 4);
      if (!cached) need += r * (int64_t)g.n * 4;
    } else {
      need += std::max<int64_t>(0, target - g.reserved_rows) * g.ldD * 4;
      if (!cached) need += np * lf * lf * 4 + sc * (int64_t)g.n * 4;
    }
    return need;
  };
  for (auto it = g.pending.begin(); it != g.pending.end();) {
    Req *r = *it;
    if (r->kind != kind) break;  // one kind per batch, in arrival order
    int64_t add_rows = 0, n_parts = nparts, n_ldf = ldf, n_srcs = srcs, n_stage = stage_rows;
    if (kind == FAP_REQ_SUBGRAPH) {
      const int32_t p = r->ids[0];
      if (part_row[p] < 0) {
        add_rows = g.vnum[p];
        n_parts++;
        n_ldf = std::max<int64_t>(n_ldf, ((int64_t)std::max(g.vnum[p], 1) + 127) / 128 * 128);
        n_srcs += g.bnum[p];
      }
      if (r->host_out && g.dtype == FAP_DTYPE_I32) n_stage = std::max<int64_t>(n_stage, g.vnum[p]);
    } else {
      add_rows = (int64_t)r->ids.size();
    }
    if (!batch.empty() && rows + add_rows > limit_rows) break;
    bool hopeless = false;
    bool fits = make_room(footprint(rows + add_rows, n_parts, n_ldf, n_srcs, n_stage), gi, &hopeless);
    if (!fits && batch.empty() && !exact) {
      exact = true;
      fits = make_room(footprint(rows + add_rows, n_parts, n_ldf, n_srcs, n_stage), gi, &hopeless);
    }
    if (!fits) {
      if (!batch.empty()) break;  // run what fits
      if (!hopeless) return true;  // wait for another graph's batch to finish
      it = g.pending.erase(it);  // larger than the whole budget
      finish(r, FAP_REQ_FAILED, FAP_ERR_NOMEM);
      progressed = true;
      continue;
    }
    nparts = n_parts;
    ldf = n_ldf;
    srcs = n_srcs;
    stage_rows = n_stage;
    batch.push_back(r);
    if (kind == FAP_REQ_SUBGRAPH) {
      const int32_t p = r->ids[0];
      if (part_row[p] < 0) {
        part_row[p] = rows;
        parts.push_back(p);
      }
      r->row_off = part_row[p];
    } else {
      r->row_off = rows;
    }
    rows += add_rows;
    it = g.pending.erase(it);
  }
  if (batch.empty()) return progressed;
  bool want_cs = false;
  for (Req *r : batch) want_cs |= (r->cs_out != nullptr);
  want_cs &= (g.dtype == FAP_DTYPE_I32);
  int rc = FAP_OK;
  const int64_t target = exact ? rows : std::max(rows, limit_rows);
  if (want_cs && (!grow_dev(&g.cs_dev, &g.cs_cap, target) || !grow_host(&g.cs_host, &g.cs_host_cap, target)))
    rc = FAP_ERR_NOMEM;
  const double t0 = now_s();
  if (rc == FAP_OK && kind == FAP_REQ_SUBGRAPH) {
    if (rows > g.reserved_rows) {
      HostTimer t(this, kStepReserve);
      rc = fap_graph_reserve(g.dg, target);
      if (rc == FAP_OK) g.reserved_rows = target;
    }
    if (rc == FAP_OK) {
      HostTimer t(this, kStepSolve);
      rc = fap_solve(g.dg, parts.data(), (int32_t)parts.size(), FAP_MODE_BATCHED);
    }
    if (want_cs)
      for (size_t i = 0; rc == FAP_OK && i < parts.size(); i++)
        rc = fap_graph_checksums_async(g.dg, parts[i], g.cs_dev + part_row[parts[i]]);
  } else if (rc == FAP_OK) {
    // every rows request of the batch in one launch sequence
    HostTimer t(this, kStepRows);
    std::vector<int32_t> sources;
    for (Req *r : batch) sources.insert(sources.end(), r->ids.begin(), r->ids.end());
    const int64_t bytes = rows * (int64_t)g.n * 4;
    g.rows_pooled = bytes > kSmallRowsBytes;
    if (g.rows_pooled) {
      if (cudaMallocFromPoolAsync(reinterpret_cast<void **>(&g.rows_out), (size_t)bytes, pool, g.stream) !=
          cudaSuccess) {
        cudaGetLastError();
        g.rows_out = nullptr;
        rc = FAP_ERR_NOMEM;
      }
    } else if (grow_dev(&g.rows_small, &g.rows_small_cap,
                        exact ? rows * (int64_t)g.n : kSmallRowsBytes / 4)) {  // once per graph
      g.rows_out = g.rows_small;
    } else {
      rc = FAP_ERR_NOMEM;
    }
    float *out = g.rows_out;
    if (rc == FAP_OK) rc = fap_graph_rows_async(g.dg, sources.data(), (int32_t)sources.size(), out);
    if (rc == FAP_OK && want_cs) {
      int64_t launches = 0;
      if (fapb::launch_row_checksums(out, rows, g.n, g.n, g.cs_dev, g.stream, &launches) !=
          cudaSuccess) {
        cudaGetLastError();
        rc = FAP_ERR_CUDA;
      }
    }
  }
  HostTimer tail_timer(this, kStepTail);
  if (rc == FAP_OK && want_cs &&
      cudaMemcpyAsync(g.cs_host, g.cs_dev, (size_t)rows * 8, cudaMemcpyDeviceToHost, g.stream) != cudaSuccess) {
    cudaGetLastError();
    rc = FAP_ERR_CUDA;
  }
  if (rc == FAP_OK) rc = fap_graph_status_async(g.dg, g.status_host);
  if (rc == FAP_OK && cudaEventRecord(g.done, g.stream) != cudaSuccess) {
    cudaGetLastError();
    rc = FAP_ERR_CUDA;
  }
  if (rc != FAP_OK) {
    cudaStreamSynchronize(g.stream);
    if (g.rows_out && g.rows_pooled) cudaFreeAsync(g.rows_out, g.stream);
    g.rows_out = nullptr;
    for (Req *r : batch) finish(r, FAP_REQ_FAILED, rc);
    return true;
  }
  for (Req *r : batch) {
    r->t_start = t0;
    std::lock_guard<std::mutex> lk(mu);
    r->state = FAP_REQ_RUNNING;
  }
  g.inflight = std::move(batch);
  g.batch_kind = kind;
  g.busy = true;
  {
    std::lock_guard<std::mutex> lk(mu);
    batches++;
    peak_bytes = std::max(peak_bytes, held_bytes());
  }
  return true;
}

void fap_server::loop() {
  cudaSetDevice(device);
  size_t rr = 0;
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(mu);
      const int ng = ngraphs.load(std::memory_order_acquire);
      bool any_busy = false, any_pending = !incoming.empty();
      for (int i = 0; i < ng; i++) {
        any_busy |= graphs[i]->busy;
        any_pending |= !graphs[i]->pending.empty();
      }
      if (!any_busy && !any_pending) {
        if (stop) break;
        cv_work.wait_for(lk, std::chrono::milliseconds(2));
      }
      while (!incoming.empty()) {
        Req *r = incoming.front();
        incoming.pop_front();
        graphs[r->graph]->pending.push_back(r);
      }
      if (stop && !any_busy) {
        // fail what is still queued
        std::vector<Req *> dead;
        for (int i = 0; i < ng; i++) {
          for (Req *r : graphs[i]->pending) dead.push_back(r);
          graphs[i]->pending.clear();
        }
        lk.unlock();
        for (Req *r : dead) finish(r, FAP_REQ_FAILED, FAP_ERR_STATE);
        break;
      }
    }
    bool progressed = false;
    const int ng = ngraphs.load(std::memory_order_acquire);
    for (int i = 0; i < ng; i++)
      if (graphs[i]->busy && cudaEventQuery(graphs[i]->done) != cudaErrorNotReady)
        progressed |= complete(*graphs[i]);
    if (!stop) {
      for (int k = 0; k < ng; k++) {
        const int gi = (int)((rr + (size_t)k) % (size_t)ng);
        if (!graphs[gi]->busy && !graphs[gi]->pending.empty()) progressed |= launch(gi);
      }
      rr++;
    }
    if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

extern "C" {

int fap_server_create(int device, double budget_bytes, int64_t max_batch_rows, fap_server **out) try {
  if (!out) return serr(FAP_ERR_INVALID, "NULL out");
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return serr(FAP_ERR_CUDA, "cannot use the device");
  }
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
    cudaGetLastError();
    return serr(FAP_ERR_CUDA, "cudaMemGetInfo failed");
  }
  auto *s = new fap_server();
  s->device = device;
  s->budget = budget_bytes > 0 ? (int64_t)budget_bytes : (int64_t)(0.6 * (double)free_b);
  s->max_batch_rows = max_batch_rows;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  if (cudaMemPoolCreate(&s->pool, &props) != cudaSuccess) {
    cudaGetLastError();
    delete s;
    return serr(FAP_ERR_CUDA, "cudaMemPoolCreate failed");
  }
  uint64_t keep = (uint64_t)(s->budget / 4);
  cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  s->worker = std::thread([s] { s->loop(); });
  *out = s;
  return FAP_OK;
} catch (...) {
  return serr_exception();
}

int fap_server_destroy(fap_server *s) try {
  if (!s) return FAP_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv_work.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();
  // requests submitted after the worker stopped
  for (Req *r : s->incoming) {
    r->state = FAP_REQ_FAILED;
    r->status = FAP_ERR_STATE;
  }
  s->incoming.clear();
  const int ng = s->ngraphs.load();
  for (int i = 0; i < ng; i++) {
    GSlot &g = *s->graphs[i];
    cudaStreamSynchronize(g.stream);
    if (g.start) cudaEventDestroy(g.start);
    if (g.done) cudaEventDestroy(g.done);
    if (g.cs_dev) cudaFree(g.cs_dev);
    if (g.rows_small) cudaFree(g.rows_small);
    if (g.cs_host) cudaFreeHost(g.cs_host);
    if (g.status_host) cudaFreeHost(g.status_host);
    fap_graph_destroy(g.dg);
    fap_ctx_destroy(g.ctx);
  }
  if (s->pool) cudaMemPoolDestroy(s->pool);
  for (auto &kv : s->reqs) delete kv.second;
  delete s;
  return FAP_OK;
} catch (...) {
  return serr_exception();
}

int fap_server_add_graph(fap_server *s, int32_t n, int64_t m, const int32_t *row_offset,
                         const int32_t *col_val, const float *weight, int dtype, int32_t K,
                         const int32_t *graph_id, const int32_t *st2ed, const int32_t *ver_num,
                         const int32_t *ver_offset, const int32_t *bdy_num, int32_t *index) try {
  if (!s || !index) return serr(FAP_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> add_lock(s->add_mu);
  const int slot = s->ngraphs.load();
  if (slot >= kMaxGraphs) return serr(FAP_ERR_NOMEM, "too many graphs");
  auto g = std::make_unique<GSlot>();
  int rc = fap_ctx_create(s->device, &g->ctx);
  if (rc != FAP_OK) return serr(rc, fap_last_error());
  rc = fap_graph_create(g->ctx, n, m, row_offset, col_val, weight, dtype, &g->dg);
  if (rc == FAP_OK)
    rc = fap_graph_set_parts(g->dg, K, graph_id, st2ed, ver_num, ver_offset, bdy_num);
  if (rc != FAP_OK) {
    std::string msg = fap_last_error();
    if (g->dg) fap_graph_destroy(g->dg);
    fap_ctx_destroy(g->ctx);
    return serr(rc, msg.c_str());
  }
  g->n = n;
  g->K = K;
  g->dtype = fap_graph_dtype(g->dg);
  g->ldD = ((int64_t)n + 127) / 128 * 128;
  g->vnum.assign(ver_num, ver_num + K + 1);
  g->voff.assign(ver_offset, ver_offset + K + 1);
  g->bnum.assign(bdy_num, bdy_num + K + 1);
  for (int32_t p = 1; p <= K; p++) g->max_part = std::max<int64_t>(g->max_part, ver_num[p]);
  // Batches change from one launch to the next: launch the stages directly
  // instead of capturing a CUDA graph per batch.
  fap_graph_set_param(g->dg, "cuda_graph", 0);
  // (the admission footprint does not count pre-packed min-plus operands)
  fap_graph_set_param(g->dg, "minplus_prepack", 0);
  fap_graph_device_bytes(g->dg, &g->base_bytes);
  void *stream = nullptr;
  fap_ctx_get_stream(g->ctx, &stream);
  g->stream = reinterpret_cast<cudaStream_t>(stream);
  if (cudaEventCreate(&g->start) != cudaSuccess || cudaEventCreate(&g->done) != cudaSuccess ||
      !grow_host(&g->status_host, &g->status_host_cap, 1)) {
    cudaGetLastError();
    if (g->start) cudaEventDestroy(g->start);
    if (g->done) cudaEventDestroy(g->done);
    fap_graph_destroy(g->dg);
    fap_ctx_destroy(g->ctx);
    return serr(FAP_ERR_CUDA, "cudaEventCreate failed");
  }
  s->graphs[slot] = std::move(g);
  s->ngraphs.store(slot + 1, std::memory_order_release);
  *index = slot;
  return FAP_OK;
} catch (...) {
  return serr_exception();
}

int fap_server_submit(fap_server *s, int32_t graph, int kind, const int32_t *ids, int32_t count,
                      float *host_out, uint64_t *checksums_out, int64_t *req_id) try {
  if (!s || !ids || !req_id || count <= 0) return serr(FAP_ERR_INVALID, "bad request arguments");
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return serr(FAP_ERR_STATE, "server is stopping");
  if (graph < 0 || graph >= s->ngraphs.load()) return serr(FAP_ERR_INVALID, "no such graph");
  GSlot &g = *s->graphs[graph];
  auto *r = new Req();
  r->graph = graph;
  r->kind = kind;
  r->ids.assign(ids, ids + count);
  r->host_out = host_out;
  r->cs_out = checksums_out;
  if (kind == FAP_REQ_SUBGRAPH) {
    if (count != 1 || ids[0] < 1 || ids[0] > g.K) {
      delete r;
      return serr(FAP_ERR_INVALID, "a sub-graph request names one part id in 1..K");
    }
    r->rows = g.vnum[ids[0]];
  } else if (kind == FAP_REQ_ROWS) {
    for (int32_t i = 0; i < count; i++)
      if (ids[i] < 0 || ids[i] >= g.n) {
        delete r;
        return serr(FAP_ERR_INVALID, "source vertex out of range");
      }
    r->rows = count;
  } else {
    delete r;
    return serr(FAP_ERR_INVALID, "unknown request kind");
  }
  r->entries = r->rows * (int64_t)g.n;
  r->id = s->next_id++;
  r->t_submit = now_s();
  s->reqs[r->id] = r;
  s->outstanding++;
  s->incoming.push_back(r);
  s->cv_work.notify_all();
  *req_id = r->id;
  return FAP_OK;
} catch (...) {
  return serr_exception();
}

int fap_server_wait(fap_server *s, int64_t req_id, double timeout_s, int *state) try {
  if (!s) return serr(FAP_ERR_INVALID, "NULL server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(req_id);
  if (it == s->reqs.end()) return serr(FAP_ERR_INVALID, "unknown request");
  Req *r = it->second;
  auto done = [&] { return r->state == FAP_REQ_DONE || r->state == FAP_REQ_FAILED; };
  if (timeout_s < 0) s->cv_done.wait(lk, done);
  else s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done);
  if (state) *state = r->state;
  return FAP_OK;
} catch (...) {
  return serr_exception();
}

int fap_server_request_info(fap_server *s, int64_t req_id, double *out4) try {
  if (!s || !out4) return serr(FAP_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(req_id);
  if (it == s->reqs.end()) return serr(FAP_ERR_INVALID, "unknown request");
  Req *r = it->second;
  const bool fin = r->state == FAP_REQ_DONE || r->state == FAP_REQ_FAILED;
  out4[0] = fin ? (r->t_done - r->t_submit) * 1e3 : -1.0;
  out4[1] = r->t_start > 0 ? (r->t_start - r->t_submit) * 1e3 : -1.0;
  out4[2] = (double)r->entries;
  out4[3] = (double)r->status;
  return FAP_OK;
} catch (...) {
  return serr_exception();
}

int fap_server_forget(fap_server *s, int64_t req_id) try {
  if (!s) return serr(FAP_ERR_INVALID, "NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(req_id);
  if (it == s->reqs.end()) return FAP_OK;
  if (it->second->state != FAP_REQ_DONE && it->second->state != FAP_REQ_FAILED)
    return serr(FAP_ERR_STATE, "request still in flight");
  delete it->second;
  s->reqs.erase(it);
  return FAP_OK;
} catch (...) {
  return serr_exception();
}

int fap_server_drain(fap_server *s) try {
  if (!s) return serr(FAP_ERR_INVALID, "NULL server");
  std::unique_lock<std::mutex> lk(s->mu);
  s->cv_done.wait(lk, [&] { return s->outstanding == 0; });
  return FAP_OK;
} catch (...) {
  return serr_exception();
}

int fap_server_stats(fap_server *s, double *out, int32_t count) try {
  if (!s || (!out && count > 0)) return serr(FAP_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  std::vector<double> v = s->lat_ms;
  std::sort(v.begin(), v.end());
  auto pct = [&](double q) {
    if (v.empty()) return 0.0;
    const size_t i = std::min(v.size() - 1, (size_t)(q * (double)(v.size() - 1) + 0.5));
    return v[i];
  };
  double mean = 0;
  for (double x : v) mean += x;
  const double all[FAP_SERVER_NSTATS] = {(double)v.size(),
                                         (double)s->entries,
                                         pct(0.50),
                                         pct(0.99),
                                         v.empty() ? 0.0 : mean / (double)v.size(),
                                         (double)s->peak_bytes,
                                         (double)s->batches,
                                         (double)s->resident_hits,
                                         (double)s->failed,
                                         (double)s->cache_builds,
                                         s->busy_ms,
                                         s->host_max_ms[kStepLaunch],
                                         s->host_max_ms[kStepComplete],
                                         s->host_max_ms[kStepCache],
                                         s->host_max_ms[kStepRoom],
                                         s->host_max_ms[kStepReserve],
                                         s->host_max_ms[kStepSolve],
                                         s->host_max_ms[kStepRows],
                                         s->host_max_ms[kStepTail]};
  for (int32_t i = 0; i < count; i++) out[i] = i < FAP_SERVER_NSTATS ? all[i] : 0.0;
  return FAP_OK;
} catch (...) {
  return serr_exception();
}

int fap_server_reset_stats(fap_server *s) try {
  if (!s) return serr(FAP_ERR_INVALID, "NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  s->lat_ms.clear();
  s->entries = 0;
  s->batches = 0;
  s->resident_hits = 0;
  s->peak_bytes = 0;
  s->failed = 0;
  s->cache_builds = 0;
  s->busy_ms = 0;
  for (double &x : s->host_max_ms) x = 0;
  return FAP_OK;
} catch (...) {
  return serr_exception();
}

int fap_server_set_option(fap_server *s, const char *key, double value) try {
  if (!s || !key) return serr(FAP_ERR_INVALID, "NULL argument");
  if (std::strcmp(key, "max_batch_bytes") == 0) {
    s->max_batch_bytes = value > 0 ? (int64_t)value : 0;
    return FAP_OK;
  }
  if (std::strcmp(key, "max_batch_rows") == 0) {
    s->max_batch_rows = value > 0 ? (int64_t)value : 0;
    return FAP_OK;
  }
  if (std::strcmp(key, "budget_bytes") == 0 && value > 0) {
    s->budget = (int64_t)value;
    return FAP_OK;
  }
  return serr(FAP_ERR_INVALID, "unknown option");
} catch (...) {
  return serr_exception();
}

const char *fap_server_last_error(void) { return s_err.c_str(); }

}  // extern "C"
