// Kernels and launchers of the per-subgraph solve path (sm_100a).
//
// Stage map (reference fapGraph::run, fap/fap.cpp:92-181):
//   stage 1   boundary SSSP            sssp_frontier_kernel      (sssp.cuh)
//   stage 2.1 Floyd matrix build       gather_kernel             (util_Myalgorithm.h:30-73)
//   stage 2.2 Floyd-Warshall           floyd_part_kernel / floyd_phase*_kernel (floyd.cuh)
//   stage 3.1 thin matrix              read in place from F      (util_Myalgorithm.h:88-95)
//   stage 3.2 min-plus                 minplus_part_kernel       (minplus.h:51-65)
//   stage 3.3 decode                   fused into the min-plus epilogue (inner rows) and
//                                      the Floyd epilogue (boundary rows)
//                                                                (util_Myalgorithm.h:75-86)
#include <cuda_runtime.h>

#include <algorithm>

#include "fap_common.cuh"
#include "fap_internal.h"
#include "floyd.cuh"
#include "minplus_tile.cuh"
#include "sssp.cuh"
#include "tma.cuh"
#include "tma_tile.cuh"

#include <cooperative_groups.h>
#include <cuda.h>
#include <cudaTypedefs.h>

#include <atomic>
#include <map>
#include <mutex>
#include <type_traits>
#include <utility>

namespace fapb {

namespace cg = cooperative_groups;

// ---------------------------------------------------------------------------
// Launch shapes: grid sizes are multiples of the current device's SM count,
// queried once per device.
// ---------------------------------------------------------------------------
namespace {
constexpr int kMaxSmDevices = 64;
std::atomic<int> g_sm_count[kMaxSmDevices];

int device_sm_count() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxSmDevices) {
    cudaGetLastError();
    return 148;
  }
  int v = g_sm_count[dev].load(std::memory_order_relaxed);
  if (v <= 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) {
      cudaGetLastError();
      v = 148;
    }
    g_sm_count[dev].store(v, std::memory_order_relaxed);
  }
  return v;
}
}  // namespace

// ---------------------------------------------------------------------------
// Tensor maps (host).  cuTensorMapEncodeTiled comes from the driver through
// the runtime's entry-point query, so the library needs no link-time
// dependency on libcuda.
// ---------------------------------------------------------------------------
namespace {
PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    else
      cudaGetLastError();
  }
  return fn;
}
}  // namespace

// (elements of `esize` bytes of type dt; d0 x esize must be a multiple of 16)
cudaError_t make_tmap_3d_dt(CUtensorMap *map, const void *base, CUtensorMapDataType dt, uint64_t esize,
                            uint64_t d0, uint64_t d1, uint64_t d2, uint32_t box0, uint32_t box1) {
  auto enc = tmap_encoder();
  if (!enc) return cudaErrorNotSupported;
  const cuuint64_t dims[3] = {d0, d1, d2};
  const cuuint64_t strides[2] = {d0 * esize, d0 * d1 * esize};
  const cuuint32_t box[3] = {box0, box1, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = enc(map, dt, 3, const_cast<void *>(base), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t make_tmap_3d(CUtensorMap *map, const void *base, bool is_float, uint64_t d0, uint64_t d1,
                         uint64_t d2, uint32_t box0, uint32_t box1) {
  return make_tmap_3d_dt(map, base, is_float ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_INT32,
                         4, d0, d1, d2, box0, box1);
}

template <typename T>
cudaError_t make_arena_tmaps(const T *F, int64_t ld, int nparts, CUtensorMap *mapA, CUtensorMap *mapB) {
  using TC = typename FloydCfg<T, kFloydTile>::TC;
  const bool f = Dist<T>::kDtype == FAP_DTYPE_F32;
  cudaError_t e = make_tmap_3d(mapA, F, f, ld, ld, nparts, TC::BK, TC::BM);
  if (e == cudaSuccess) e = make_tmap_3d(mapB, F, f, ld, ld, nparts, TC::BN, TC::BK);
  return e;
}

using MPCfg32 = TileCfg<int32_t, kMinplusBM, kMinplusBN, 16, 8, 8>;

template <typename T>
using MPCfg = TileCfg<T, kMinplusBM, kMinplusBN, 16, 8, 8>;

// ---------------------------------------------------------------------------
// Stage 2.1: build each part's padded Floyd matrix.
// CTA (i, pidx): row i of part pidx.  Inner rows take the part's own edges
// in CSR order, a later duplicate overwriting an earlier one (resolved by
// keeping the largest edge index per column), then a zero diagonal.
// Boundary rows copy the SSSP row restricted to the part's columns.
// Padding rows/columns hold the sentinel.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256)
    gather_kernel(const PartDesc *__restrict__ parts, const int32_t *__restrict__ row_offset,
                  const int32_t *__restrict__ col, const T *__restrict__ w,
                  const int32_t *__restrict__ graph_id, const int32_t *__restrict__ st2ed,
                  const int32_t *__restrict__ ed2st, const T *__restrict__ D, int64_t ldD,
                  T *__restrict__ F) {
  extern __shared__ int32_t winner[];
  const PartDesc pd = parts[blockIdx.y];
  const int i = blockIdx.x;
  if (i >= pd.ldf) return;
  const T inf = Dist<T>::inf();
  T *Fi = F + pd.f_off + (int64_t)i * pd.ldf;
  if (i >= pd.s) {
    for (int j = threadIdx.x; j < pd.ldf; j += blockDim.x) Fi[j] = inf;
    return;
  }
  if (i < pd.b && !(pd.flags & kPartLocal)) {
    const T *Si = D + (pd.row_base + i) * ldD;
    for (int j = threadIdx.x; j < pd.ldf; j += blockDim.x) {
      T v = inf;
      if (j < pd.s) v = (j == i) ? T(0) : Si[__ldg(st2ed + pd.start + j)];
      Fi[j] = v;
    }
    return;
  }
  for (int j = threadIdx.x; j < pd.s; j += blockDim.x) winner[j] = -1;
  __syncthreads();
  const int v = st2ed[pd.start + i];
  const int e0 = row_offset[v], e1 = row_offset[v + 1];
  for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    const int nb = __ldg(col + e);
    if (__ldg(graph_id + nb) != pd.part) continue;
    const int j = __ldg(ed2st + nb) - pd.start;
    if (j >= 0 && j < pd.s) atomicMax(&winner[j], e);
  }
  __syncthreads();
  for (int j = threadIdx.x; j < pd.ldf; j += blockDim.x) {
    T val = inf;
    if (j < pd.s) {
      if (j == i) val = T(0);
      else if (winner[j] >= 0) val = __ldg(w + winner[j]);
    }
    Fi[j] = val;
  }
}

template <typename T>
cudaError_t launch_gather(const PartDesc *parts, int nparts, int max_ldf, const int32_t *row_offset,
                          const int32_t *col, const T *w, const int32_t *graph_id,
                          const int32_t *st2ed, const int32_t *ed2st, const T *D, int64_t ldD,
                          T *F, cudaStream_t stream, int64_t *launches) {
  if (nparts <= 0) return cudaSuccess;
  size_t smem = (size_t)max_ldf * sizeof(int32_t);
  auto kern = gather_kernel<T>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  kern<<<dim3(max_ldf, nparts), 256, smem, stream>>>(parts, row_offset, col, w, graph_id, st2ed,
                                                     ed2st, D, ldD, F);
  *launches += 1;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Stage 1 launcher
// ---------------------------------------------------------------------------
namespace {
int sssp_resident_ctas(int n) {
  // resident frontier-SSSP CTAs per (device, n): shared memory grows with n
  static std::mutex mu;
  static std::map<std::pair<int, int>, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(dev, n);
  const auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int per_sm = 0;
  const size_t smem = sssp_smem_bytes(n);
  cudaFuncSetAttribute(sssp_frontier_kernel<int32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaFuncSetAttribute(sssp_frontier_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sssp_frontier_kernel<int32_t>, kSsspThreads, smem);
  cudaGetLastError();
  const int v = std::max(1, per_sm) * device_sm_count();
  cache[key] = v;
  return v;
}
}  // namespace

int sssp_scratch_rows(int n, int num_sources) {
  return std::max(0, std::min(num_sources, sssp_resident_ctas(n)));
}

template <typename T>
cudaError_t launch_sssp(const int32_t *row_offset, const int32_t *col, const T *w, int n,
                        const int32_t *sources, const int64_t *out_rows, int num_sources, T *out,
                        int64_t ld, int64_t init_cols, const int32_t *perm_out, T *scratch,
                        T delta, int chain, int precheck, int64_t max_rounds, int *status,
                        cudaStream_t stream, int64_t *launches) {
  if (num_sources <= 0) return cudaSuccess;
  const size_t smem = sssp_smem_bytes(n);
  auto kern = sssp_frontier_kernel<T>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // With a relabelled work space every CTA needs a scratch row, so the grid
  // is the resident CTA count and CTAs loop over sources.
  const int grid = perm_out ? sssp_scratch_rows(n, num_sources) : num_sources;
  kern<<<grid, kSsspThreads, smem, stream>>>(row_offset, col, w, n, sources, out_rows, num_sources,
                                             out, ld, init_cols, perm_out, scratch, delta,
                                             chain, precheck, max_rounds, status);
  *launches += 1;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Stage 1, tiled form: multi-source Bellman-Ford over in-edges
// ---------------------------------------------------------------------------
// kMsbfS sources at a time share one pass over the graph per iteration.  The
// tile Dt[v][s] (vertex-major, the sources of a vertex contiguous: one
// 16-byte load per lane for a whole row) stays in L2 on mid-size graphs.  An
// iteration pulls, for every work item (a vertex and up to 32 of its
// in-edges), only from in-neighbours that changed in the previous iteration,
// and lowers the vertex's row with atomic minima where it improves; the tile
// is updated in place, so values are monotone and the fixed point is the
// exact shortest distances, each the sum along its path edge by edge (the
// same additions in the same order as Dijkstra's).  The host repeats
// iterations until one changes nothing (or the round bound is reached).
// Source s of the tile (global index s0 + s): vertex st2ed[sources[s0 + s]];
// without a source list the work graph's own vertex s0 + s.
// Several tiles run side by side: tile z (blockIdx.y here) at
// Dt + z * n * kMsbfS with its bitmaps at act + z * words, sources
// s0 + z * kMsbfS + s.
template <typename T>
__global__ void msbf_seed_kernel(T *Dt, int n, const int32_t *__restrict__ sources, const int32_t *__restrict__ st2ed,
                                 int s0, int num_sources, int64_t words, uint32_t *act) {
  const int64_t z = blockIdx.y;
  const int s = threadIdx.x, g = s0 + (int)z * kMsbfS + s;
  if (g >= num_sources) return;
  const int v = sources ? __ldg(st2ed + __ldg(sources + g)) : g;
  Dt[(z * n + v) * kMsbfS + s] = T(0);
  atomicOr(act + z * words + (v >> 5), 1u << (v & 31));
}

// One warp lowers row v of the tile from up to 32 in-edges e0..e1 whose
// tails pass `active` (warp-uniform loop, four tail rows in flight, read
// through L1: a tail row that another SM lowers during this iteration may be
// seen stale here, which is harmless, because that lowering marks the tail
// as changed and its out-neighbours pull from it again next iteration); the
// row's lanes each hold 4 sources.  Returns (warp-uniform) whether any entry
// improved.  Atomic minima: other warps may lower the same row meanwhile.
template <typename T, class Active>
__device__ __forceinline__ bool msbf_pull_row(T *Dt, int v, int e0, int e1, const int32_t *__restrict__ tcol,
                                              const T *__restrict__ tw, Active active) {
  using V = typename Vec4<T>::type;
  const T inf = Dist<T>::inf();
  const int lane = threadIdx.x & 31;
  const int e = e0 + lane;
  int u = -1;
  T w = T(0);
  if (e < e1) {
    u = __ldg(tcol + e);
    if (active(u)) w = __ldg(tw + e);
    else u = -1;
  }
  unsigned mask = __ballot_sync(0xffffffffu, u >= 0);
  if (!mask) return false;
  T acc[4] = {inf, inf, inf, inf};
  while (mask) {  // warp-uniform: four active in-edges per step, loads in flight together
    int uu[4];
    T ww[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      uu[q] = -1;
      ww[q] = T(0);
      if (mask) {
        const int k = __ffs(mask) - 1;
        mask &= mask - 1;
        uu[q] = __shfl_sync(0xffffffffu, u, k);
        ww[q] = __shfl_sync(0xffffffffu, w, k);
      }
    }
    V d[4];
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (uu[q] >= 0) d[q] = __ldca(reinterpret_cast<const V *>(Dt + (int64_t)uu[q] * kMsbfS) + lane);
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (uu[q] >= 0) {
        acc[0] = Dist<T>::relax(d[q].x, ww[q], acc[0]);
        acc[1] = Dist<T>::relax(d[q].y, ww[q], acc[1]);
        acc[2] = Dist<T>::relax(d[q].z, ww[q], acc[2]);
        acc[3] = Dist<T>::relax(d[q].w, ww[q], acc[3]);
      }
  }
  T *row = Dt + (int64_t)v * kMsbfS + 4 * lane;
  const V cur = __ldcg(reinterpret_cast<const V *>(row));
  const T cv[4] = {cur.x, cur.y, cur.z, cur.w};
  bool imp = false;
#pragma unroll
  for (int q = 0; q < 4; q++)
    if (acc[q] < cv[q]) imp |= acc[q] < Dist<T>::atomic_min(row + q, acc[q]);
  return __any_sync(0xffffffffu, imp);
}

template <typename T>
__global__ void __launch_bounds__(256)
    msbf_iter_kernel(T *Dt, int n, int ntiles, const MsbfItem *__restrict__ items, int nitems,
                     const int32_t *__restrict__ tro, const int32_t *__restrict__ tcol, const T *__restrict__ tw,
                     const uint32_t *__restrict__ act_cur, uint32_t *act_next, int64_t words, int *changed) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t total = (int64_t)ntiles * nitems;
  for (int64_t it = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); it < total; it += nwarps) {
    const int64_t z = it / nitems;
    const MsbfItem m = items[it - z * nitems];
    const uint32_t *ac = act_cur + z * words;
    auto active = [ac](int u) { return ((__ldg(ac + (u >> 5)) >> (u & 31)) & 1u) != 0; };
    const int e1 = min(m.e0 + 32, __ldg(tro + m.v + 1));
    if (msbf_pull_row<T>(Dt + z * n * kMsbfS, m.v, m.e0, e1, tcol, tw, active) && lane == 0) {
      atomicOr(act_next + z * words + (m.v >> 5), 1u << (m.v & 31));
      *changed = 1;
    }
  }
}

// out[out_rows[s0 + s]][v] = Dt[v][s] for s < ns (row s0 + s without a row
// list), all init_cols columns (INF past n; column col_map[v] with a column
// map, then init_cols <= n): 32 vertices per CTA, transposed through shared
// memory, 128-byte row segments stored.
template <typename T>
__global__ void __launch_bounds__(256)
    msbf_store_kernel(const T *__restrict__ Dt, int n, int s0, int ns, T *out, int64_t ld,
                      const int64_t *__restrict__ out_rows, int64_t init_cols, const int32_t *__restrict__ col_map) {
  __shared__ T tile[32][kMsbfS + 1];
  const int64_t v0 = (int64_t)blockIdx.x * 32;
  const T inf = Dist<T>::inf();
  for (int t = threadIdx.x; t < 32 * kMsbfS; t += blockDim.x) {
    const int vv = t / kMsbfS, s = t % kMsbfS;
    const int64_t v = v0 + vv;
    tile[vv][s] = v < n ? __ldcg(Dt + v * kMsbfS + s) : inf;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (int s = threadIdx.x >> 5; s < ns; s += blockDim.x >> 5) {
    const int64_t v = v0 + lane;
    const int64_t row = out_rows ? out_rows[s0 + s] : (int64_t)(s0 + s);
    if (v < init_cols) out[row * ld + (col_map ? (int64_t)__ldg(col_map + v) : v)] = tile[lane][s];
  }
}

template <typename T>
cudaError_t launch_msbf(const MsbfItem *items, int nitems, const int32_t *tro, const int32_t *tcol, const T *tw,
                        int n, const int32_t *st2ed, const int32_t *sources, const int64_t *out_rows,
                        int num_sources, T *out, int64_t ld, int64_t init_cols, int ztiles, T *Dt, uint32_t *act,
                        int *changed, int *host_changed, int64_t max_rounds, int *status, cudaStream_t stream,
                        int64_t *launches) {
  if (num_sources <= 0) return cudaSuccess;
  if (ztiles < 1 || ztiles > 64) return cudaErrorInvalidValue;
  const int64_t words = ceil_div(n, 32);
  uint32_t *act_a = act, *act_b = act + ztiles * words;
  const int iter_blocks = device_sm_count() * 8;
  constexpr int kChunk = 4;  // iterations between convergence checks
  for (int s0 = 0; s0 < num_sources; s0 += ztiles * kMsbfS) {
    const int z = (int)std::min<int64_t>(ztiles, ceil_div(num_sources - s0, kMsbfS));  // tiles side by side
    cudaError_t e = launch_fill<T>(Dt, (int64_t)z * n, kMsbfS, kMsbfS, Dist<T>::inf(), stream, launches);
    if (e == cudaSuccess) e = cudaMemsetAsync(act_a, 0, z * words * 4, stream);
    if (e != cudaSuccess) return e;
    msbf_seed_kernel<T><<<dim3(1, z), kMsbfS, 0, stream>>>(Dt, n, sources, st2ed, s0, num_sources, words, act_a);
    *launches += 1;
    bool done = false;
    for (int64_t round = 0; !done; round += kChunk) {
      if (round >= max_rounds) {
        // the bound: report it (the host status path reads it)
        e = cudaMemcpyAsync(status, &kMsbfRoundLimit, sizeof(int), cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return e;
        break;
      }
      e = cudaMemsetAsync(changed, 0, kChunk * sizeof(int), stream);
      if (e != cudaSuccess) return e;
      for (int c = 0; c < kChunk; c++) {
        e = cudaMemsetAsync(act_b, 0, z * words * 4, stream);
        if (e != cudaSuccess) return e;
        msbf_iter_kernel<T><<<iter_blocks, 256, 0, stream>>>(Dt, n, z, items, nitems, tro, tcol, tw, act_a, act_b,
                                                            words, changed + c);
        *launches += 1;
        std::swap(act_a, act_b);
      }
      e = cudaMemcpyAsync(host_changed, changed, kChunk * sizeof(int), cudaMemcpyDeviceToHost, stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
      if (e != cudaSuccess) return e;
      for (int c = 0; c < kChunk; c++) done |= host_changed[c] == 0;
    }
    for (int q = 0; q < z; q++) {
      const int sq = s0 + q * kMsbfS;
      msbf_store_kernel<T><<<(unsigned)ceil_div(init_cols, 32), 256, 0, stream>>>(
          Dt + (int64_t)q * n * kMsbfS, n, sq, std::min(kMsbfS, num_sources - sq), out, ld, out_rows, init_cols,
          nullptr);
    }
    *launches += z;
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// ---------------------------------------------------------------------------
// Stage 2.2: Floyd-Warshall
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(FloydCfg<T, kFloydTile>::THREADS, 2)
    floyd_part_kernel(const PartDesc *__restrict__ parts, T *F, T *D, int64_t ldD,
                      const int32_t *__restrict__ st2ed, const __grid_constant__ CUtensorMap mapA,
                      const __grid_constant__ CUtensorMap mapB, int *status) {
  using TC = typename FloydCfg<T, kFloydTile>::TC;
  extern __shared__ __align__(128) unsigned char fp_smem_raw[];
  auto sm = tma_smem_init<T, TC>(fp_smem_raw);
  const PartDesc pd = parts[blockIdx.x];
  T *mat = F + pd.f_off;
  const int nb = (int)ceil_div(pd.s, kFloydTile);
  if (!floyd_close_cta<T, kFloydTile>(&mapA, &mapB, blockIdx.x, mat, pd.ldf, nb, pd.s, sm)) {
    if (threadIdx.x == 0) set_status(status, kDevTmaTimeout);
    return;
  }
  // Decode of the boundary rows (util_Myalgorithm.h:75-86 for rows < b).
  const int64_t cnt = (int64_t)pd.b * pd.s;
  for (int64_t t = threadIdx.x; t < cnt; t += blockDim.x) {
    const int i = (int)(t / pd.s), j = (int)(t % pd.s);
    D[(pd.row_base + i) * ldD + st2ed[pd.start + j]] = mat[(int64_t)i * pd.ldf + j];
  }
}

template <typename T>
cudaError_t launch_floyd_parts(const PartDesc *parts, int nparts, T *F, int64_t ld, T *D,
                               int64_t ldD, const int32_t *st2ed, int *status, cudaStream_t stream,
                               int64_t *launches) {
  if (nparts <= 0) return cudaSuccess;
  CUtensorMap mapA, mapB;
  cudaError_t e = make_arena_tmaps<T>(F, ld, nparts, &mapA, &mapB);
  if (e != cudaSuccess) return e;
  const size_t smem = FloydCfg<T, kFloydTile>::SMEM_BYTES;
  auto kern = floyd_part_kernel<T>;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<nparts, FloydCfg<T, kFloydTile>::THREADS, smem, stream>>>(parts, F, D, ldD, st2ed, mapA, mapB,
                                                                   status);
  *launches += 1;
  return cudaGetLastError();
}

// One matrix (leading dimension ld, a multiple of kFloydTile, padded with the
// sentinel to nb tiles per side), one launch per phase per pivot block.
template <typename T>
__global__ void __launch_bounds__(FloydCfg<T, kFloydTile>::THREADS, 2)
    floyd_mat_phase1_kernel(T *mat, int64_t ld, int kb, int s) {
  using TC = typename FloydCfg<T, kFloydTile>::TC;
  extern __shared__ __align__(128) unsigned char fq_smem_raw[];
  auto sm = tma_smem_init<T, TC>(fq_smem_raw);
  floyd_diag_close<T, kFloydTile>(mat, ld, kb * kFloydTile, sm.ring, min(kFloydTile, s - kb * kFloydTile));
}

// blockIdx.x in [0, 2*(nb-1)): first nb-1 are row-panel tiles, rest column.
template <typename T>
__global__ void __launch_bounds__(FloydCfg<T, kFloydTile>::THREADS, 2)
    floyd_mat_phase2_kernel(T *mat, int64_t ld, int kb, int nb, int s,
                            const __grid_constant__ CUtensorMap mapA,
                            const __grid_constant__ CUtensorMap mapB, int *status) {
  using TC = typename FloydCfg<T, kFloydTile>::TC;
  extern __shared__ __align__(128) unsigned char fq_smem_raw[];
  auto sm = tma_smem_init<T, TC>(fq_smem_raw);
  auto valid = [s](int t) { return min(kFloydTile, s - t * kFloydTile); };
  int t = blockIdx.x;
  bool ok;
  if (t < nb - 1) {
    const int j = t < kb ? t : t + 1;
    ok = floyd_tile_update<T, kFloydTile>(&mapA, &mapB, 0, mat, ld, kb, j, kb, sm, valid(kb), valid(kb), valid(j));
  } else {
    t -= nb - 1;
    const int i = t < kb ? t : t + 1;
    ok = floyd_tile_update<T, kFloydTile>(&mapA, &mapB, 0, mat, ld, i, kb, kb, sm, valid(kb), valid(i), valid(kb));
  }
  if (!ok && threadIdx.x == 0 && status) set_status(status, kDevTmaTimeout);
}

template <typename T>
__global__ void __launch_bounds__(FloydCfg<T, kFloydTile>::THREADS, 2)
    floyd_mat_phase3_kernel(T *mat, int64_t ld, int kb, int nb, int s,
                            const __grid_constant__ CUtensorMap mapA,
                            const __grid_constant__ CUtensorMap mapB, int *status) {
  using TC = typename FloydCfg<T, kFloydTile>::TC;
  extern __shared__ __align__(128) unsigned char fq_smem_raw[];
  auto sm = tma_smem_init<T, TC>(fq_smem_raw);
  auto valid = [s](int t) { return min(kFloydTile, s - t * kFloydTile); };
  const int t = blockIdx.x;
  int i = t / (nb - 1), j = t % (nb - 1);
  i = i < kb ? i : i + 1;
  j = j < kb ? j : j + 1;
  if (!floyd_tile_update<T, kFloydTile>(&mapA, &mapB, 0, mat, ld, i, j, kb, sm, valid(kb), valid(i), valid(j)) &&
      threadIdx.x == 0 && status)
    set_status(status, kDevTmaTimeout);
}

template <typename T>
cudaError_t launch_floyd_matrix(T *mat, int64_t ld, int nb, int *status, cudaStream_t stream,
                                int64_t *launches, int s) {
  using FC = FloydCfg<T, kFloydTile>;
  if (nb <= 0) return cudaSuccess;
  if (s < 0 || s > nb * kFloydTile) s = nb * kFloydTile;
  if (s <= (nb - 1) * kFloydTile) return cudaErrorInvalidValue;  // the last block holds real rows
  CUtensorMap mapA, mapB;
  cudaError_t e = make_arena_tmaps<T>(mat, ld, 1, &mapA, &mapB);
  if (e != cudaSuccess) return e;
  const size_t smem = FC::SMEM_BYTES;
  for (auto k : {(const void *)floyd_mat_phase1_kernel<T>, (const void *)floyd_mat_phase2_kernel<T>,
                 (const void *)floyd_mat_phase3_kernel<T>}) {
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  for (int kb = 0; kb < nb; kb++) {
    floyd_mat_phase1_kernel<T><<<1, FC::THREADS, smem, stream>>>(mat, ld, kb, s);
    *launches += 1;
    if (nb > 1) {
      floyd_mat_phase2_kernel<T><<<2 * (nb - 1), FC::THREADS, smem, stream>>>(mat, ld, kb, nb, s, mapA, mapB,
                                                                             status);
      floyd_mat_phase3_kernel<T><<<(nb - 1) * (nb - 1), FC::THREADS, smem, stream>>>(mat, ld, kb, nb, s, mapA,
                                                                                    mapB, status);
      *launches += 2;
    }
  }
  return cudaGetLastError();
}

// Batched multi-launch form: pivot round kb of every part in three
// launches (diagonal tiles, panel tiles, remainder tiles), so thousands of
// tile CTAs keep every SM busy whatever the number of parts.  Part z has
// nb_z = ceil(s_z / kFloydTile) tiles per side in an arena of equal squares;
// CTAs beyond a part's tiles exit.
template <typename T>
__global__ void __launch_bounds__(FloydCfg<T, kFloydTile>::THREADS, 2)
    floyd_parts_phase1_kernel(const PartDesc *__restrict__ parts, T *F, int kb) {
  using TC = typename FloydCfg<T, kFloydTile>::TC;
  extern __shared__ __align__(128) unsigned char fm_smem_raw[];
  const PartDesc pd = parts[blockIdx.x];
  if (kb >= (int)ceil_div(pd.s, kFloydTile)) return;
  auto sm = tma_smem_init<T, TC>(fm_smem_raw);
  floyd_diag_close<T, kFloydTile>(F + pd.f_off, pd.ldf, kb * kFloydTile, sm.ring,
                                  min(kFloydTile, pd.s - kb * kFloydTile));
}

template <typename T>
__global__ void __launch_bounds__(FloydCfg<T, kFloydTile>::THREADS, 2)
    floyd_parts_phase2_kernel(const PartDesc *__restrict__ parts, T *F, int kb,
                              const __grid_constant__ CUtensorMap mapA,
                              const __grid_constant__ CUtensorMap mapB, int *status) {
  using TC = typename FloydCfg<T, kFloydTile>::TC;
  extern __shared__ __align__(128) unsigned char fm_smem_raw[];
  const PartDesc pd = parts[blockIdx.y];
  const int nb = (int)ceil_div(pd.s, kFloydTile);
  int t = blockIdx.x;
  if (kb >= nb || t >= 2 * (nb - 1)) return;
  auto sm = tma_smem_init<T, TC>(fm_smem_raw);
  T *mat = F + pd.f_off;
  bool ok;
  if (t < nb - 1) {
    const int j = t < kb ? t : t + 1;
    ok = floyd_tile_update<T, kFloydTile>(&mapA, &mapB, blockIdx.y, mat, pd.ldf, kb, j, kb, sm,
                                          min(kFloydTile, pd.s - kb * kFloydTile),
                                          min(kFloydTile, pd.s - kb * kFloydTile),
                                          min(kFloydTile, pd.s - j * kFloydTile));
  } else {
    t -= nb - 1;
    const int i = t < kb ? t : t + 1;
    ok = floyd_tile_update<T, kFloydTile>(&mapA, &mapB, blockIdx.y, mat, pd.ldf, i, kb, kb, sm,
                                          min(kFloydTile, pd.s - kb * kFloydTile),
                                          min(kFloydTile, pd.s - i * kFloydTile),
                                          min(kFloydTile, pd.s - kb * kFloydTile));
  }
  if (!ok && threadIdx.x == 0) set_status(status, kDevTmaTimeout);
}

template <typename T>
__global__ void __launch_bounds__(FloydCfg<T, kFloydTile>::THREADS, 2)
    floyd_parts_phase3_kernel(const PartDesc *__restrict__ parts, T *F, int kb,
                              const __grid_constant__ CUtensorMap mapA,
                              const __grid_constant__ CUtensorMap mapB, int *status) {
  using TC = typename FloydCfg<T, kFloydTile>::TC;
  extern __shared__ __align__(128) unsigned char fm_smem_raw[];
  const PartDesc pd = parts[blockIdx.y];
  const int nb = (int)ceil_div(pd.s, kFloydTile);
  const int t = blockIdx.x;
  if (kb >= nb || t >= (nb - 1) * (nb - 1)) return;
  auto sm = tma_smem_init<T, TC>(fm_smem_raw);
  int i = t / (nb - 1), j = t % (nb - 1);
  i = i < kb ? i : i + 1;
  j = j < kb ? j : j + 1;
  if (!floyd_tile_update<T, kFloydTile>(&mapA, &mapB, blockIdx.y, F + pd.f_off, pd.ldf, i, j, kb, sm,
                                        min(kFloydTile, pd.s - kb * kFloydTile),
                                        min(kFloydTile, pd.s - i * kFloydTile),
                                        min(kFloydTile, pd.s - j * kFloydTile)) &&
      threadIdx.x == 0)
    set_status(status, kDevTmaTimeout);
}

template <typename T>
cudaError_t launch_floyd_parts_multi(const PartDesc *parts, int nparts, int max_nb, T *F, int64_t ld,
                                     int *status, cudaStream_t stream, int64_t *launches) {
  if (nparts <= 0 || max_nb <= 0) return cudaSuccess;
  using FC = FloydCfg<T, kFloydTile>;
  CUtensorMap mapA, mapB;
  cudaError_t e = make_arena_tmaps<T>(F, ld, nparts, &mapA, &mapB);
  if (e != cudaSuccess) return e;
  const size_t smem = FC::SMEM_BYTES;
  for (auto k : {(const void *)floyd_parts_phase1_kernel<T>, (const void *)floyd_parts_phase2_kernel<T>,
                 (const void *)floyd_parts_phase3_kernel<T>}) {
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  for (int kb = 0; kb < max_nb; kb++) {
    floyd_parts_phase1_kernel<T><<<nparts, FC::THREADS, smem, stream>>>(parts, F, kb);
    *launches += 1;
    if (max_nb > 1) {
      floyd_parts_phase2_kernel<T><<<dim3(2 * (max_nb - 1), nparts), FC::THREADS, smem, stream>>>(
          parts, F, kb, mapA, mapB, status);
      floyd_parts_phase3_kernel<T><<<dim3((max_nb - 1) * (max_nb - 1), nparts), FC::THREADS, smem, stream>>>(
          parts, F, kb, mapA, mapB, status);
      *launches += 2;
    }
  }
  return cudaGetLastError();
}

template <typename T>
__global__ void bdy_scatter_kernel(const PartDesc *__restrict__ parts, const T *__restrict__ F,
                                   T *D, int64_t ldD, const int32_t *__restrict__ st2ed) {
  const PartDesc pd = parts[blockIdx.y];
  const int i = blockIdx.x;
  if (i >= pd.b) return;
  const T *Fi = F + pd.f_off + (int64_t)i * pd.ldf;
  T *Di = D + (pd.row_base + i) * ldD;
  for (int j = threadIdx.x; j < pd.s; j += blockDim.x) Di[st2ed[pd.start + j]] = Fi[j];
}

template <typename T>
cudaError_t launch_bdy_scatter(const PartDesc *parts, int nparts, const T *F, T *D, int64_t ldD,
                               const int32_t *st2ed, int max_b, int max_s, cudaStream_t stream,
                               int64_t *launches) {
  if (nparts <= 0 || max_b <= 0) return cudaSuccess;
  (void)max_s;
  bdy_scatter_kernel<T><<<dim3(max_b, nparts), 256, 0, stream>>>(parts, F, D, ldD, st2ed);
  *launches += 1;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Stage 3: min-plus merge with the fused decode of own-part columns.
// grid (ldD / BN, nwork): CTA (x, y) computes rows work[y].m0 .. +BM of the
// part's inner block against columns x*BN .. +BN.
//   R[i][j] = min(INF, min_{k<b} F[b+i][k] + S[k][j])   (S = the part's
//   boundary rows of D), then for own-part columns j the closed Floyd value
//   F[b+i][ed2st[j]-start] replaces it, as the reference's decode does.
// ---------------------------------------------------------------------------
// Epilogue of a min-plus tile: own-part columns take the closed Floyd value
// (the reference's decode), then 16-byte streaming stores of the rows that
// exist.
template <typename T, class C>
__device__ __forceinline__ void minplus_part_epilogue(const PartDesc &pd, const MPWork &wk, int n0, int n,
                                                      const T *__restrict__ F, T *Cm, int64_t ldD,
                                                      const int32_t *__restrict__ graph_id,
                                                      const int32_t *__restrict__ ed2st,
                                                      T (&acc)[C::TM][C::TN]) {
  const int M = pd.s - pd.b;
  const int tid = threadIdx.x, ty = tid / C::TX, tx = tid % C::TX;
  // Own-part columns of this thread (fused decode).
  int own[C::TN];
  bool any_own = false;
#pragma unroll
  for (int gj = 0; gj < C::GN; gj++)
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int c = n0 + tile_col<C>(tx, gj, q);
      int o = -1;
      if (c < n && __ldg(graph_id + c) == pd.part) o = __ldg(ed2st + c) - pd.start;
      own[4 * gj + q] = o;
      any_own |= (o >= 0);
    }
  using V = typename Vec4<T>::type;
#pragma unroll
  for (int gi = 0; gi < C::GM; gi++)
#pragma unroll
    for (int l = 0; l < 4; l++) {
      const int r = wk.m0 + tile_row<C>(ty, gi, l);
      if (r >= M) continue;
      if (any_own) {
        const T *Fr = F + pd.f_off + (int64_t)(pd.b + r) * pd.ldf;
#pragma unroll
        for (int j = 0; j < C::TN; j++)
          if (own[j] >= 0) acc[4 * gi + l][j] = __ldcg(Fr + own[j]);   // (L2: see acc_load)
      }
      T *dst = Cm + (int64_t)r * ldD + n0;
#pragma unroll
      for (int gj = 0; gj < C::GN; gj++) {
        V v;
        v.x = acc[4 * gi + l][4 * gj + 0];
        v.y = acc[4 * gi + l][4 * gj + 1];
        v.z = acc[4 * gi + l][4 * gj + 2];
        v.w = acc[4 * gi + l][4 * gj + 3];
        __stcs(reinterpret_cast<V *>(dst + tile_col<C>(tx, gj, 0)), v);
      }
    }
}

// ---------------------------------------------------------------------------
// Stage 3: min-plus merge with the fused decode of own-part columns.
// grid (ldD / BN, nwork): CTA (x, y) computes rows work[y].m0 .. +BM of the
// part's inner block against columns x*BN .. +BN.
//   R[i][j] = min(INF, min_{k<b} F[b+i][k] + S[k][j])   (S = the part's
//   boundary rows of D), then for own-part columns j the closed Floyd value
//   F[b+i][ed2st[j]-start] replaces it, as the reference's decode does.
// PACK (int32): a tile whose entries provably fit (Pack16) runs the packed
// 16-bit engine and shifts its results back by the column offsets; the
// others run the int32 engine.  Both give the same int32 values.  PACK 1
// converts the int32 stages in shared memory, PACK 2 reads the operands
// packed beforehand (Pack16::s16 / at, tensor maps mapAT / mapS).
// ---------------------------------------------------------------------------
// One min-plus tile: rows wk.m0 .. +BM of the part's inner block against
// columns n0 .. +BN.  Block-wide; raw is the CTA's dynamic shared memory
// (the TMA ring at its start, the packed buffers after it).  Returns false
// (in every thread) if a TMA stage never completed.
template <typename T, int PACK>
__device__ __forceinline__ bool minplus_part_tile(const PartDesc &pd, const MPWork &wk, int tile_x, int n,
                                                  const T *__restrict__ F, T *D, int64_t ldD,
                                                  const int32_t *__restrict__ graph_id,
                                                  const int32_t *__restrict__ ed2st, const CUtensorMap *mapF,
                                                  const CUtensorMap *mapD, const Pack16 &pk,
                                                  TmaSmem<T, typename FloydCfg<T, kFloydTile>::TC> &sm,
                                                  unsigned char *raw, const CUtensorMap *mapAT = nullptr,
                                                  const CUtensorMap *mapS = nullptr) {
  using C = MPCfg<T>;
  using TC = typename FloydCfg<T, kFloydTile>::TC;
  const int n0 = tile_x * C::BN;
  const int K = pd.b;
  T *Cm = D + (pd.row_base + pd.b) * ldD;
  T acc[C::TM][C::TN];
  // A = F rows b+m0.. of the part (columns 0..b-1); B = D rows
  // row_base..row_base+b-1 (the part's boundary rows).  Rows and columns past
  // the part's extent are never stored; k past b is never read.
  // The part's square in the arena (its index there: a batch index, or the
  // part's slot in the resident cache).
  const int fz = (int)(pd.f_off / ((int64_t)pd.ldf * pd.ldf));
  bool packed = false;
  if constexpr (PACK != 0) {
    packed = __ldg(pk.maxA + wk.pidx) + __ldg(pk.range + (int64_t)wk.pidx * pk.ntiles + tile_x) < kPackCap;
    if (threadIdx.x == 0) {
      atomicAdd(pk.tiles + 1, 1ull);
      if (packed) atomicAdd(pk.tiles, 1ull);
    }
  }
  if (packed && PACK == 2) {
    if constexpr (PACK == 2) {
      // column offsets after the ring's memory (unused by the packed ring)
      int32_t *coff = reinterpret_cast<int32_t *>(reinterpret_cast<unsigned char *>(sm.ring) +
                                                  Pack16pCfg<TC>::STAGE_WORDS * 4 * TC::STAGES);
      for (int c = threadIdx.x; c < C::BN; c += blockDim.x)
        coff[c] = __ldg(pk.off + (int64_t)wk.pidx * ldD + n0 + c);
      uint32_t a16[8][4];
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) a16[i][j] = kPackInit;
      // (the engine's first barrier orders the column offsets before use)
      if (!tma_minplus_tile16p<TC>(mapAT, wk.m0, mapS, n0, __ldg(pk.krow + wk.pidx), K, a16, sm,
                                   pd.s - pd.b - wk.m0))
        return false;
      const int tx = threadIdx.x % C::TX;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        // acc16[.][p] holds columns tile_col(tx, p / 2, 2 (p % 2)) and the next
        const int32_t off = coff[tile_col<C>(tx, j / 4, j % 4)];
        const int p = j / 2;
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const int32_t v = (j % 2) ? (int32_t)(int16_t)(a16[i][p] >> 16) : (int32_t)(int16_t)(a16[i][p] & 0xffffu);
          acc[i][j] = v < kPackCap ? v + off : Dist<T>::inf();
        }
      }
      // every thread has read its offsets before the shared memory is reused
      __syncthreads();
    }
  } else if (packed) {
    if constexpr (PACK == 1) {
      using P = Pack16Cfg<TC>;
      uint32_t *pbuf = reinterpret_cast<uint32_t *>(smem_align128(raw) + P::BUF_OFFSET);
      int32_t *coff = reinterpret_cast<int32_t *>(pbuf + 2 * P::BUF_ELEMS);
      for (int c = threadIdx.x; c < C::BN; c += blockDim.x)
        coff[c] = __ldg(pk.off + (int64_t)wk.pidx * ldD + n0 + c);
      uint32_t a16[4][8];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) a16[i][j] = kPackInit;
      // (the engine's first barrier orders the column offsets before use)
      if (!tma_minplus_tile16<TC>(mapF, 0, pd.b + wk.m0, fz, mapD, n0, (int)pd.row_base, 0, K, a16, sm, pbuf,
                                  nullptr, coff, pd.s - pd.b - wk.m0))
        return false;
      const int tx = threadIdx.x % C::TX;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int32_t off = coff[tile_col<C>(tx, j / 4, j % 4)];
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const int32_t lo = (int32_t)(int16_t)(a16[i][j] & 0xffffu);
          const int32_t hi = (int32_t)(int16_t)(a16[i][j] >> 16);
          // pair i = 2g + h holds rows 4g + 2h and 4g + 2h + 1 of the thread
          const int r0 = 4 * (i / 2) + 2 * (i % 2);
          acc[r0][j] = lo < kPackCap ? lo + off : Dist<T>::inf();
          acc[r0 + 1][j] = hi < kPackCap ? hi + off : Dist<T>::inf();
        }
      }
      // every thread has read its offsets before the buffers are reused
      __syncthreads();
    }
  } else {
    acc_fill<T, C>(acc, Dist<T>::inf());
    // (rows past the part's inner block are never stored: their warps skip
    // the relaxations)
    if (!tma_minplus_tile<T, TC, true>(mapF, 0, pd.b + wk.m0, fz, mapD, n0, (int)pd.row_base, 0, K, acc, sm,
                                       pd.s - pd.b - wk.m0, C::BN))
      return false;
  }
  minplus_part_epilogue<T, C>(pd, wk, n0, n, F, Cm, ldD, graph_id, ed2st, acc);
  return true;
}

// ---------------------------------------------------------------------------
// Stage 3: min-plus merge with the fused decode of own-part columns.
// grid (ldD / BN, nwork): CTA (x, y) computes rows work[y].m0 .. +BM of the
// part's inner block against columns x*BN .. +BN.
//   R[i][j] = min(INF, min_{k<b} F[b+i][k] + S[k][j])   (S = the part's
//   boundary rows of D), then for own-part columns j the closed Floyd value
//   F[b+i][ed2st[j]-start] replaces it, as the reference's decode does.
// PACK (int32): a tile whose entries provably fit (Pack16) runs the packed
// 16-bit engine and shifts its results back by the column offsets; the
// others run the int32 engine.  Both give the same int32 values.
// ---------------------------------------------------------------------------
template <typename T, int PACK>
__global__ void __launch_bounds__(MPCfg<T>::THREADS, 2)
    minplus_part_kernel(const PartDesc *__restrict__ parts, const MPWork *__restrict__ work, int n,
                        const T *__restrict__ F, T *D, int64_t ldD,
                        const int32_t *__restrict__ graph_id, const int32_t *__restrict__ ed2st,
                        const __grid_constant__ CUtensorMap mapF, const __grid_constant__ CUtensorMap mapD,
                        const __grid_constant__ CUtensorMap mapAT, const __grid_constant__ CUtensorMap mapS,
                        int *status, Pack16 pk) {
  using TC = typename FloydCfg<T, kFloydTile>::TC;
  extern __shared__ __align__(128) unsigned char mp_smem_raw[];
  auto sm = tma_smem_init<T, TC>(mp_smem_raw);
  const MPWork wk = work[blockIdx.y];
  const PartDesc pd = parts[wk.pidx];
  if (!minplus_part_tile<T, PACK>(pd, wk, blockIdx.x, n, F, D, ldD, graph_id, ed2st, &mapF, &mapD, pk, sm,
                                  mp_smem_raw, &mapAT, &mapS) &&
      threadIdx.x == 0)
    set_status(status, kDevTmaTimeout);
}

// Packed-form bounds of a batch (see Pack16): one CTA per (column tile, work
// item); only a part's first work item (m0 == 0) works, so each part is
// scanned once.  Thread t owns column n0 + t and walks the part's b boundary
// rows of D; columns past n read as having no finite entry.
__global__ void __launch_bounds__(kMinplusBN)
    pack16_cols_kernel(const PartDesc *__restrict__ parts, const MPWork *__restrict__ work, int n,
                       const int32_t *__restrict__ D, int64_t ldD, Pack16 pk) {
  const MPWork wk = work[blockIdx.y];
  if (wk.m0 != 0) return;
  const PartDesc pd = parts[wk.pidx];
  const int j = blockIdx.x * kMinplusBN + threadIdx.x;
  int32_t lo = INT32_MAX, hi = 0;
  if (j < n) {
    const int32_t *col = D + pd.row_base * ldD + j;
    int k = 0;
    for (; k + 4 <= pd.b; k += 4) {
      int32_t v[4];
#pragma unroll
      for (int q = 0; q < 4; q++) v[q] = __ldg(col + (int64_t)(k + q) * ldD);
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (v[q] < kInfI32) {
          lo = min(lo, v[q]);
          hi = max(hi, v[q]);
        }
    }
    for (; k < pd.b; k++) {
      const int32_t v = __ldg(col + (int64_t)k * ldD);
      if (v < kInfI32) {
        lo = min(lo, v);
        hi = max(hi, v);
      }
    }
  }
  int32_t range = 0;
  if (lo == INT32_MAX) lo = 0;
  else range = hi - lo;
  pk.off[(int64_t)wk.pidx * ldD + j] = lo;
  if (pk.s16 != nullptr) {
    // the pre-packed boundary rows (columns past n: no finite entry)
    uint16_t *dst = pk.s16 + (int64_t)pk.krow[wk.pidx] * ldD + j;
    const int32_t *col = D + pd.row_base * ldD + j;
    for (int k = 0; k < pd.b; k++)
      dst[(int64_t)k * ldD] = (uint16_t)(j < n ? pack_clamp(__ldg(col + (int64_t)k * ldD), lo) : kPackCap);
  }
  // the tile's largest range
  __shared__ int32_t red[kMinplusBN / 32];
  for (int o = 16; o > 0; o >>= 1) range = max(range, __shfl_xor_sync(0xffffffffu, range, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = range;
  __syncthreads();
  if (threadIdx.x == 0) {
    int32_t m = 0;
    for (int w = 0; w < kMinplusBN / 32; w++) m = max(m, red[w]);
    pk.range[(int64_t)wk.pidx * pk.ntiles + blockIdx.x] = m;
  }
}

// Largest finite A = F[b+i][k] (i < s-b, k < b) of each part of the work
// (one CTA per work item; a part's first item does it).  A negative entry
// (never produced from non-negative weights) makes the part run in int32.
__global__ void __launch_bounds__(256)
    pack16_maxa_kernel(const PartDesc *__restrict__ parts, const MPWork *__restrict__ work,
                       const int32_t *__restrict__ F, Pack16 pk) {
  const MPWork wk = work[blockIdx.x];
  if (wk.m0 != 0) return;
  const PartDesc pd = parts[wk.pidx];
  const int64_t cnt = (int64_t)(pd.s - pd.b) * pd.b;
  int32_t m = 0;
  for (int64_t e = threadIdx.x; e < cnt; e += blockDim.x) {
    const int64_t i = e / pd.b, k = e % pd.b;
    const int32_t v = __ldg(F + pd.f_off + (pd.b + i) * pd.ldf + k);
    if (v < 0) m = kPackCap;
    else if (v < kInfI32) m = max(m, v);
  }
  __shared__ int32_t red[8];
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    int32_t x = 0;
    for (int w = 0; w < 8; w++) x = max(x, red[w]);
    pk.maxA[wk.pidx] = x;
  }
}

// Pre-packed A operand of the packed tiles (Pack16::at): CTA (x, y) moves
// boundary indices 32x .. 32x+31 of work item y's 128 inner rows through a
// shared-memory transpose, reading F[b+m0+r][k] along k and writing
// at[krow + k][m0 + r] along r, clamped at kPackCap in both halves.  Rows
// past the part's inner block (up to at_ld) read as having no finite entry.
__global__ void __launch_bounds__(256)
    pack16_at_kernel(const PartDesc *__restrict__ parts, const MPWork *__restrict__ work,
                     const int32_t *__restrict__ F, Pack16 pk) {
  const MPWork wk = work[blockIdx.y];
  const PartDesc pd = parts[wk.pidx];
  const int k0 = blockIdx.x * 32;
  if (k0 >= pd.b) return;
  const int M = pd.s - pd.b;
  __shared__ uint32_t t[kMinplusBM][33];
  const int tid = threadIdx.x;
#pragma unroll 4
  for (int q = 0; q < kMinplusBM / 8; q++) {
    const int r = tid / 32 + 8 * q, c = tid % 32;
    const int i = wk.m0 + r, k = k0 + c;
    int32_t v = kPackCap;
    if (i < M && k < pd.b) v = pack_clamp(__ldg(F + pd.f_off + (int64_t)(pd.b + i) * pd.ldf + k), 0);
    t[r][c] = pack_pair(v, v);
  }
  __syncthreads();
  uint32_t *at = pk.at + (int64_t)pk.krow[wk.pidx] * pk.at_ld;
#pragma unroll 4
  for (int q = 0; q < 16; q++) {
    const int r = tid % kMinplusBM, c = tid / kMinplusBM + 2 * q;
    const int k = k0 + c, i = wk.m0 + r;
    if (k < pd.b && i < pk.at_ld) at[(int64_t)k * pk.at_ld + i] = t[r][c];
  }
}

// ---------------------------------------------------------------------------
// Work-queue form of the batched Floyd-Warshall (FloydQueue).  One
// persistent launch: each CTA claims the next item of the list, waits for
// the per-part counters of the items it depends on, runs it, and counts it
// done.  Items are claimed in list order and every dependency of an item
// comes earlier in the list, so every awaited item has been claimed by a
// running CTA and finishes: the waits end (they are bounded all the same;
// on a timeout the CTA records kDevQueueTimeout and raises the abort flag,
// which ends every other wait).  Dependencies of part p:
//   Floyd-1 (pivot block kb)   every Floyd-3 item of block kb-1
//   Floyd-2 (block kb)         Floyd-1 of block kb
//   Floyd-3 (block kb)         every Floyd-2 item of block kb
//   scatter                    the last block's Floyd-3 items (Floyd-1 when
//                              the part is one tile)
//   min-plus tile              every scatter item of the part
// A finished item's global writes are made visible to the TMA (async proxy)
// and to other CTAs (fence, then the counter increment); a waiting CTA reads
// the counter with acquire semantics before it loads anything.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int ld_acquire_gpu(const int32_t *p) {
  int32_t v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

constexpr uint32_t kQueuePollLimit = 1u << 24;   // x ~150 ns: a few seconds

__device__ bool queue_wait(const int32_t *ctr, int need, const int32_t *abort) {
  for (uint32_t i = 0; i < kQueuePollLimit; i++) {
    if (ld_acquire_gpu(ctr) >= need) return true;
    if (ld_acquire_gpu(abort) != 0) return false;
    __nanosleep(128);
  }
  return false;
}

// Claimed item, decoded by thread 0 into shared memory (so that nothing of
// the dispatch stays live in registers across an item's body).
struct QClaim {
  int kind;     // kQFloyd1..3, kQScatter; 0 = min-plus tile; -1 = stop
  int pidx, kb, t, m0;
};

template <typename T, bool WITH_MP>
__global__ void __launch_bounds__(FloydCfg<T, kFloydTile>::THREADS, 2)
    floyd_queue_kernel(const PartDesc *__restrict__ parts, T *F, FloydQueue q,
                       const MPWork *__restrict__ work, int n, T *D, int64_t ldD,
                       const int32_t *__restrict__ st2ed, const int32_t *__restrict__ graph_id,
                       const int32_t *__restrict__ ed2st, const __grid_constant__ CUtensorMap mapA,
                       const __grid_constant__ CUtensorMap mapB, const __grid_constant__ CUtensorMap mapD,
                       int *status, Pack16 pk) {
  using TC = typename FloydCfg<T, kFloydTile>::TC;
  extern __shared__ __align__(128) unsigned char fq_smem_raw[];
  auto sm = tma_smem_init<T, TC>(fq_smem_raw);
  __shared__ QClaim cl;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) {
      int32_t *abort = q.cnt + (int64_t)q.nparts * q.stride;
      const int64_t ntiles = ldD / kMinplusBN;
      const int64_t total = q.nitems + (int64_t)q.mp_work * ntiles;
      const int64_t it = atomicAdd(abort + 1, 1);
      QClaim c{-1, 0, 0, 0, 0};
      if (it < total) {
        if (it < q.nitems) {
          const QItem qi = q.items[it];
          c = QClaim{qi.kind, qi.pidx, qi.kb, qi.t, 0};
        } else {
          const int64_t m = it - q.nitems;
          const MPWork wk = work[m / ntiles];
          c = QClaim{0, wk.pidx, 0, (int)(m % ntiles), wk.m0};
        }
        const PartDesc pd = parts[c.pidx];
        const int nb = (int)ceil_div(pd.s, kFloydTile);
        const int32_t *cn = q.cnt + (int64_t)c.pidx * q.stride;
        const int32_t *p2 = cn + 2, *p3 = cn + 2 + (q.stride - 2) / 2;
        // items per pivot block (symmetric: the row panel, the tiles on and
        // above the diagonal)
        const int n2 = q.sym ? nb - 1 : 2 * (nb - 1);
        const int n3 = q.sym ? (nb - 1) * nb / 2 : (nb - 1) * (nb - 1);
        bool ok = true;
        if (c.kind == kQFloyd1) {
          if (c.kb > 0) ok = queue_wait(p3 + c.kb - 1, n3, abort);
        } else if (c.kind == kQFloyd2 || c.kind == kQFloyd2S) {
          ok = queue_wait(cn, c.kb + 1, abort);
        } else if (c.kind == kQFloyd3 || c.kind == kQFloyd3S) {
          ok = queue_wait(p2 + c.kb, n2, abort);
        } else if (c.kind == kQScatter) {
          ok = nb == 1 ? queue_wait(cn, 1, abort) : queue_wait(p3 + nb - 1, n3, abort);
        } else {
          ok = queue_wait(cn + 1, (int)ceil_div(pd.b, kQScatterRows), abort);
        }
        if (!ok) {
          set_status(status, kDevQueueTimeout);
          atomicExch(abort, 1);
          c.kind = -1;
        }
        // the items waited for wrote with generic stores; this CTA reads
        // them with the TMA too
        fence_proxy_async_all();
      }
      cl = c;
    }
    __syncthreads();
    const int kind = cl.kind;
    if (kind < 0) break;
    bool ok = true;
    if (kind == kQFloyd1) {
      const PartDesc pd = parts[cl.pidx];
      const int kb = cl.kb;
      floyd_diag_close<T, kFloydTile>(F + pd.f_off, pd.ldf, kb * kFloydTile, sm.ring,
                                      min(kFloydTile, pd.s - kb * kFloydTile));
    } else if (kind == kQFloyd2 || kind == kQFloyd3 || kind == kQFloyd2S || kind == kQFloyd3S) {
      const PartDesc pd = parts[cl.pidx];
      const int kb = cl.kb, t = cl.t;
      const int nb = (int)ceil_div(pd.s, kFloydTile);
      int i, j;
      if (kind == kQFloyd2S || kind == kQFloyd3S) {
        i = t >> 16;
        j = t & 0xffff;
      } else if (kind == kQFloyd3) {
        i = t / (nb - 1);
        j = t % (nb - 1);
        i = i < kb ? i : i + 1;
        j = j < kb ? j : j + 1;
      } else if (t < nb - 1) {
        i = kb;
        j = t < kb ? t : t + 1;
      } else {
        const int t2 = t - (nb - 1);
        i = t2 < kb ? t2 : t2 + 1;
        j = kb;
      }
      const int z = (int)(pd.f_off / ((int64_t)pd.ldf * pd.ldf));
      ok = floyd_tile_update_sym<T, kFloydTile>(&mapA, &mapB, z, F + pd.f_off, pd.ldf, i, j, kb, sm,
                                                min(kFloydTile, pd.s - kb * kFloydTile),
                                                min(kFloydTile, pd.s - i * kFloydTile),
                                                min(kFloydTile, pd.s - j * kFloydTile),
                                                kind == kQFloyd2S || kind == kQFloyd3S);
    } else if (kind == kQScatter) {
      // boundary rows kb .. kb + kQScatterRows of the closed matrix into D
      // (the reference's decode of rows < b, util_Myalgorithm.h:75-86)
      const PartDesc pd = parts[cl.pidx];
      const int r0 = cl.kb, r1 = min(pd.b, r0 + kQScatterRows);
      const T *mat = F + pd.f_off;
      const int64_t cnt = (int64_t)(r1 - r0) * pd.s;
      for (int64_t e = tid; e < cnt; e += blockDim.x) {
        const int i = r0 + (int)(e / pd.s), j = (int)(e % pd.s);
        D[(pd.row_base + i) * ldD + st2ed[pd.start + j]] = __ldcg(mat + (int64_t)i * pd.ldf + j);
      }
    } else if constexpr (WITH_MP) {
      const PartDesc pd = parts[cl.pidx];
      const MPWork wk{cl.pidx, cl.m0};
      ok = minplus_part_tile<T, 0>(pd, wk, cl.t, n, F, D, ldD, graph_id, ed2st, &mapA, &mapD, pk, sm,
                                       fq_smem_raw);
    }
    // this item's writes: visible to the async proxy, then to other CTAs,
    // before it counts as done
    fence_proxy_async_all();
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        set_status(status, kDevTmaTimeout);
        atomicExch(q.cnt + (int64_t)q.nparts * q.stride, 1);
      }
      break;
    }
    if (tid == 0 && kind > 0) {
      int32_t *cn = q.cnt + (int64_t)cl.pidx * q.stride;
      const int half = (q.stride - 2) / 2;
      int32_t *done = kind == kQFloyd1                           ? cn
                      : (kind == kQFloyd2 || kind == kQFloyd2S) ? cn + 2 + cl.kb
                      : (kind == kQFloyd3 || kind == kQFloyd3S) ? cn + 2 + half + cl.kb
                                                                : cn + 1;
      __threadfence();
      atomicAdd(done, 1);
    }
  }
}

template <typename T>
cudaError_t launch_floyd_queue(const PartDesc *parts, int nparts, T *F, int64_t ldf, const FloydQueue &q,
                               const MPWork *work, int n, T *D, int64_t ldD, int64_t drows,
                               const int32_t *st2ed, const int32_t *graph_id, const int32_t *ed2st,
                               int *status, cudaStream_t stream, int64_t *launches, const Pack16 *pk) {
  if (nparts <= 0 || (q.nitems <= 0 && q.mp_work <= 0)) return cudaSuccess;
  using FC = FloydCfg<T, kFloydTile>;
  CUtensorMap mapA, mapB, mapD;
  cudaError_t e = make_arena_tmaps<T>(F, ldf, nparts, &mapA, &mapB);
  if (e == cudaSuccess)
    e = make_tmap_3d(&mapD, D, Dist<T>::kDtype == FAP_DTYPE_F32, ldD, std::max<int64_t>(drows, 1), 1,
                     FC::TC::BN, FC::TC::BK);
  if (e != cudaSuccess) return e;
  // (min-plus tiles in the queue run in int32: the packed form needs bounds
  // over the boundary rows that the queue itself scatters, so a batch that
  // uses the packed form keeps its min-plus in launch_minplus_parts)
  (void)pk;
  auto kern = q.mp_work > 0 ? floyd_queue_kernel<T, true> : floyd_queue_kernel<T, false>;
  const size_t smem = FC::SMEM_BYTES;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, FC::THREADS, smem);
  if (e != cudaSuccess) return e;
  const int64_t total = q.nitems + (int64_t)q.mp_work * (ldD / kMinplusBN);
  const int grid =
      (int)std::max<int64_t>(1, std::min<int64_t>(total, (int64_t)std::max(per_sm, 1) * device_sm_count()));
  Pack16 none{};
  kern<<<grid, FC::THREADS, smem, stream>>>(parts, F, q, work, n, D, ldD, st2ed, graph_id, ed2st, mapA, mapB, mapD,
                                            status, none);
  *launches += 1;
  return cudaGetLastError();
}

// Thin-K variant (b <= kThinK): the product is store-bound, not
// relaxation-bound, so the kernel is shaped around the stores.  A CTA owns a
// strip of kThinCols columns of one part and walks all of the part's inner
// rows.  Each thread owns two groups of 4 columns, kThinCols/2 apart, so
// that every warp-wide 16-byte store covers 512 contiguous bytes (whole
// sectors; a half-written sector would be read back from DRAM).  The part's
// b boundary rows of the strip stay in registers for the whole CTA; each
// block of kMinplusBM rows stages its A values and its own-part (decode)
// values in shared memory.  The relaxation loop is instantiated for every
// exact b (a uniform switch per CTA), so no relaxation or branch is spent on
// padding.
constexpr int kThinK = kThinBoundary;
constexpr int kThinThreads = 256;
constexpr int kThinCols = 8 * kThinThreads;
constexpr int kThinHalf = kThinCols / 2;
constexpr int kThinOwnMax = 64;

template <typename T>
struct ThinShared {
  __align__(16) T As[kMinplusBM][kThinK];
  T Own[kMinplusBM][kThinOwnMax];
  int32_t own_col[kThinOwnMax];
  int nown;
};

// Rows [0, M) of the part's inner block for the thread's columns
// c0 + {0..3} (g = 0) and c0 + kThinHalf + {0..3} (g = 1); B relaxations per
// output.  G = 1 handles only group g0.
template <typename T, int B, int G>
__device__ __forceinline__ void thin_rows(ThinShared<T> &sh, const PartDesc &pd, int mb, int me, int64_t c0,
                                          const T *__restrict__ F, T *D, int64_t ldD, const int (&own)[8], bool any_own,
                                          int g0, const bool (&live)[2]) {
  using V = typename Vec4<T>::type;
  const T inf = Dist<T>::inf();
  T sv[B > 0 ? B : 1][4 * G];
#pragma unroll
  for (int k = 0; k < B; k++)
#pragma unroll
    for (int g = 0; g < G; g++) {
      const int gg = g0 + g;
      V v;
      if (live[gg]) v = __ldg(reinterpret_cast<const V *>(D + (pd.row_base + k) * ldD + c0 + gg * kThinHalf));
      else v.x = v.y = v.z = v.w = inf;
      sv[k][4 * g + 0] = v.x; sv[k][4 * g + 1] = v.y; sv[k][4 * g + 2] = v.z; sv[k][4 * g + 3] = v.w;
    }
  const T *Fp = F + pd.f_off;
  // Own-part columns (the decode): staged slot per column, or -1.  Own
  // columns are scattered over the strip, so the replacement is done with
  // selects (no divergent branch per row) whenever any lane of the warp has
  // one; a column whose value was not staged (more own columns than
  // kThinOwnMax in the strip) takes the rare global-load path.
  const bool warp_own = __any_sync(0xffffffffu, any_own);
  const bool cta_unstaged = sh.nown > kThinOwnMax;  // same in every thread
  for (int m0 = mb; m0 < me; m0 += kMinplusBM) {
    const int rows = min(kMinplusBM, me - m0);
    const T *Fr = Fp + (int64_t)(pd.b + m0) * pd.ldf;
    // stage this block's A values and own-part values
    __syncthreads();
    for (int t = threadIdx.x; t < kMinplusBM * kThinK; t += blockDim.x) {
      const int r = t / kThinK, k = t % kThinK;
      sh.As[r][k] = (r < rows && k < B) ? __ldg(Fr + (int64_t)r * pd.ldf + k) : inf;
    }
    const int nown = min(sh.nown, kThinOwnMax);
    for (int t = threadIdx.x; t < rows * nown; t += blockDim.x) {
      const int r = t / nown, o = t % nown;
      sh.Own[r][o] = __ldg(Fr + (int64_t)r * pd.ldf + sh.own_col[o]);
    }
    __syncthreads();
    T *Cm = D + (pd.row_base + pd.b + m0) * ldD + c0;
#pragma unroll 2
    for (int r = 0; r < rows; r++) {
      T acc[4 * G];
#pragma unroll
      for (int q = 0; q < 4 * G; q++) acc[q] = inf;
#pragma unroll
      for (int k4 = 0; k4 < (B + 3) / 4; k4++) {
        const V a4 = *reinterpret_cast<const V *>(&sh.As[r][4 * k4]);
        const T av[4] = {a4.x, a4.y, a4.z, a4.w};
#pragma unroll
        for (int kk = 0; kk < 4; kk++)
          if (4 * k4 + kk < B) {
#pragma unroll
            for (int q = 0; q < 4 * G; q++)
              acc[q] = Dist<T>::relax(av[kk], sv[4 * k4 + kk][q], acc[q]);
          }
      }
      if (warp_own) {
#pragma unroll
        for (int q = 0; q < 4 * G; q++) {
          const int o = own[4 * g0 + q];  // -1, or (part-local column << 7) | (slot + 1)
          const int sl = o >= 0 ? (o & 127) - 1 : -1;
          const T st = sh.Own[r][sl >= 0 ? sl : 0];
          acc[q] = sl >= 0 ? st : acc[q];
        }
        if (cta_unstaged) {
#pragma unroll
          for (int q = 0; q < 4 * G; q++) {
            const int o = own[4 * g0 + q];
            if (o >= 0 && (o & 127) == 0) acc[q] = Fr[(int64_t)r * pd.ldf + (o >> 7)];
          }
        }
      }
#pragma unroll
      for (int g = 0; g < G; g++) {
        const int gg = g0 + g;
        if (live[gg]) {
          V v;
          v.x = acc[4 * g + 0]; v.y = acc[4 * g + 1]; v.z = acc[4 * g + 2]; v.w = acc[4 * g + 3];
          __stcs(reinterpret_cast<V *>(Cm + (int64_t)r * ldD + gg * kThinHalf), v);
        }
      }
    }
  }
}

template <typename T, int B>
__device__ __forceinline__ void thin_dispatch(ThinShared<T> &sh, const PartDesc &pd, int mb, int me,
                                              int64_t c0, const T *F, T *D, int64_t ldD,
                                              const int (&own)[8], bool any_own,
                                              const bool (&live)[2]) {
  if (B <= 6) {
    thin_rows<T, B, 2>(sh, pd, mb, me, c0, F, D, ldD, own, any_own, 0, live);
  } else {
    // the two column groups in two passes keep the boundary strip in registers
    thin_rows<T, B, 1>(sh, pd, mb, me, c0, F, D, ldD, own, any_own, 0, live);
    thin_rows<T, B, 1>(sh, pd, mb, me, c0, F, D, ldD, own, any_own, 1, live);
  }
}

// grid (ceil(ldD / kThinCols), number of thin parts, row chunks);
// blockIdx.y indexes thin_parts (batch indices), blockIdx.z the chunk of
// row_chunk inner rows (a multiple of kMinplusBM) the CTA walks, so that a
// batch of few parts still spreads over every SM.
template <typename T>
__global__ void __launch_bounds__(kThinThreads, 2)
    minplus_thin_kernel(const PartDesc *__restrict__ parts, const int32_t *__restrict__ thin_parts,
                        int n, const T *__restrict__ F, T *D, int64_t ldD,
                        const int32_t *__restrict__ graph_id, const int32_t *__restrict__ ed2st,
                        int row_chunk) {
  __shared__ ThinShared<T> sh;
  const PartDesc pd = parts[thin_parts[blockIdx.y]];
  const int M = pd.s - pd.b;
  const int mb = blockIdx.z * row_chunk;
  const int me = min(M, mb + row_chunk);
  if (mb >= me) return;
  if (threadIdx.x == 0) sh.nown = 0;
  const int64_t c0 = (int64_t)blockIdx.x * kThinCols + 4 * threadIdx.x;
  const bool live[2] = {c0 < ldD, c0 + kThinHalf < ldD};  // ldD is a multiple of 4
  int own[8];
  bool any_own = false;
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 8; q++) {
    const int64_t c = c0 + (q >> 2) * kThinHalf + (q & 3);
    own[q] = -1;
    if (live[q >> 2] && c < n && __ldg(graph_id + c) == pd.part) {
      const int j = __ldg(ed2st + c) - pd.start;
      const int sl = atomicAdd(&sh.nown, 1);
      int staged = 0;
      if (sl < kThinOwnMax) {
        sh.own_col[sl] = j;
        staged = sl + 1;
      }
      own[q] = (j << 7) | staged;
      any_own = true;
    }
  }
  switch (pd.b) {
#define FAPB_THIN_CASE(NB) \
  case NB: thin_dispatch<T, NB>(sh, pd, mb, me, c0, F, D, ldD, own, any_own, live); break;
    FAPB_THIN_CASE(0) FAPB_THIN_CASE(1) FAPB_THIN_CASE(2) FAPB_THIN_CASE(3) FAPB_THIN_CASE(4)
    FAPB_THIN_CASE(5) FAPB_THIN_CASE(6) FAPB_THIN_CASE(7) FAPB_THIN_CASE(8) FAPB_THIN_CASE(9)
    FAPB_THIN_CASE(10) FAPB_THIN_CASE(11) FAPB_THIN_CASE(12) FAPB_THIN_CASE(13)
    FAPB_THIN_CASE(14) FAPB_THIN_CASE(15) FAPB_THIN_CASE(16)
#undef FAPB_THIN_CASE
    default: break;
  }
}

template <typename T>
cudaError_t launch_minplus_parts(const PartDesc *parts, int nparts, const MPWork *work, int nwork, int n,
                                 const T *F, int64_t ldf, T *D, int64_t ldD, int64_t drows,
                                 const int32_t *graph_id, const int32_t *ed2st, int *status,
                                 cudaStream_t stream, int64_t *launches, const Pack16 *pk) {
  if (nwork <= 0) return cudaSuccess;
  using C = MPCfg<T>;
  using TC = typename FloydCfg<T, kFloydTile>::TC;
  const bool f = Dist<T>::kDtype == FAP_DTYPE_F32;
  CUtensorMap mapF, mapD;
  cudaError_t e = make_tmap_3d(&mapF, F, f, ldf, ldf, nparts, TC::BK, TC::BM);
  if (e == cudaSuccess) e = make_tmap_3d(&mapD, D, f, ldD, drows, 1, TC::BN, TC::BK);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)(ldD / C::BN), (unsigned)nwork);
  Pack16 none{};
  bool done = false;
  if constexpr (std::is_same<T, int32_t>::value) {
    if (pk != nullptr) {
      // bounds of the packed form for the work's parts, then the merge
      if (pk->ntiles < (int)(ldD / C::BN)) return cudaErrorInvalidValue;
      pack16_cols_kernel<<<grid, kMinplusBN, 0, stream>>>(parts, work, n, D, ldD, *pk);
      pack16_maxa_kernel<<<(unsigned)nwork, 256, 0, stream>>>(parts, work, F, *pk);
      *launches += 2;
      if (pk->s16 != nullptr) {
        // operands packed beforehand: the boundary rows (above) and the
        // inner-to-boundary distances, then tiles without conversion
        if (pk->at == nullptr || pk->krow == nullptr || pk->at_ld % 4 != 0 || pk->prows <= 0 || pk->max_b <= 0)
          return cudaErrorInvalidValue;
        CUtensorMap mapAT, mapS;
        e = make_tmap_3d_dt(&mapAT, pk->at, CU_TENSOR_MAP_DATA_TYPE_UINT32, 4, pk->at_ld, pk->prows, 1, TC::BM,
                            TC::BK);
        if (e == cudaSuccess)
          e = make_tmap_3d_dt(&mapS, pk->s16, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, ldD, pk->prows, 1, TC::BN,
                              TC::BK);
        if (e != cudaSuccess) return e;
        pack16_at_kernel<<<dim3((unsigned)ceil_div(pk->max_b, 32), (unsigned)nwork), 256, 0, stream>>>(parts, work,
                                                                                                     F, *pk);
        *launches += 1;
        const size_t smem = TC::SMEM_BYTES;
        auto kern = minplus_part_kernel<T, 2>;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, C::THREADS, smem, stream>>>(parts, work, n, F, D, ldD, graph_id, ed2st, mapF, mapD, mapAT,
                                                 mapS, status, *pk);
      } else {
        using P = Pack16Cfg<TC>;
        const size_t smem = P::SMEM_BYTES;
        auto kern = minplus_part_kernel<T, 1>;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, C::THREADS, smem, stream>>>(parts, work, n, F, D, ldD, graph_id, ed2st, mapF, mapD, mapF,
                                                 mapD, status, *pk);
      }
      done = true;
    }
  }
  if (!done) {
    const size_t smem = TC::SMEM_BYTES;
    auto kern = minplus_part_kernel<T, 0>;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, C::THREADS, smem, stream>>>(parts, work, n, F, D, ldD, graph_id, ed2st, mapF, mapD, mapF, mapD,
                                             status, none);
  }
  *launches += 1;
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_minplus_thin(const PartDesc *parts, const int32_t *thin_parts, int nthin, int max_m,
                                int n, const T *F, T *D, int64_t ldD, const int32_t *graph_id,
                                const int32_t *ed2st, cudaStream_t stream, int64_t *launches) {
  if (nthin <= 0 || max_m <= 0) return cudaSuccess;
  // Enough CTAs for about four per SM: split the parts' inner rows into
  // chunks of whole kMinplusBM blocks when the column strips alone are few.
  const int64_t col_ctas = ceil_div(ldD, kThinCols) * (int64_t)nthin;
  const int64_t blocks = ceil_div(max_m, kMinplusBM);
  const int64_t want = 4 * (int64_t)device_sm_count();
  const int64_t zc = std::min<int64_t>(blocks, std::max<int64_t>(1, ceil_div(want, col_ctas)));
  const int row_chunk = (int)(ceil_div(blocks, zc) * kMinplusBM);
  const unsigned gz = (unsigned)ceil_div(max_m, row_chunk);
  dim3 grid((unsigned)ceil_div(ldD, kThinCols), (unsigned)nthin, gz);
  minplus_thin_kernel<T><<<grid, kThinThreads, 0, stream>>>(parts, thin_parts, n, F, D, ldD,
                                                            graph_id, ed2st, row_chunk);
  *launches += 1;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Predecessor (path) matrices
// ---------------------------------------------------------------------------
// P[row][j] for the batch's output rows: the in-neighbour u of j with the
// least D[row][u] + w(u, j), the smallest u among equal sums; the row's own
// vertex maps to itself and unreachable entries to -1.  That is the Bellman
// condition on the final distances, so with positive weights following P
// from any reachable j walks a shortest path back to the source.  The
// reference keeps whichever predecessor its Dijkstra / Floyd / min-plus
// evaluation order finds (fap/kernel/batch_sssp.h:108-110,
// fap/kernel/floyd.h:38-49, fap/kernel/minplus.h:51-65); both agree wherever
// the predecessor is unique.
// grid (column chunks, batch parts, row chunks of kPredRows): consecutive
// CTAs share their rows, which stay in L2 for the gathers D[row][u]; the
// in-edge list of a column is read once per CTA for all of its rows.
constexpr int kPredRows = 32;
constexpr int kPredThreads = 256;
constexpr int kPredDeg = 4;  // in-edges kept in registers (more are read in a loop)

// A candidate predecessor as one 64-bit key: the sum dist(u) + w in the
// high word (non-negative int32 and float32 values order like their bit
// patterns), u in the low word, so that the least key is the least sum and,
// among equal sums, the smallest u.  Unreachable u: the largest key.
template <typename T>
__device__ __forceinline__ uint64_t pred_key(T du, int u, T w, T inf) {
  const T v = du + w;
  uint32_t bits;
  if constexpr (sizeof(T) == 4 && Dist<T>::kDtype == FAP_DTYPE_F32) bits = __float_as_uint((float)v);
  else bits = (uint32_t)v;
  return du < inf ? ((uint64_t)bits << 32) | (uint32_t)u : ~0ull;
}

// Rows are taken kPredUnroll at a time, and every load of a group (the
// entry itself and the gathers of its in-neighbours' distances) is issued
// before any is used, so a thread keeps up to kPredUnroll * (kPredDeg + 1)
// loads in flight instead of waiting on each row in turn.
constexpr int kPredUnroll = 4;

template <typename T>
__global__ void __launch_bounds__(kPredThreads)
    pred_kernel(const PartDesc *__restrict__ parts, const T *__restrict__ D, int32_t *__restrict__ P,
                int64_t ldD, int n, const int32_t *__restrict__ tro, const int32_t *__restrict__ tcol,
                const T *__restrict__ tw, const int32_t *__restrict__ st2ed, int mode) {
  __shared__ int32_t src_s[kPredRows];
  const PartDesc pd = parts[blockIdx.y];
  // rows and columns this launch covers (PredMode)
  const bool thin = pd.b <= kPredThinB;
  int rlo = 0, rhi = pd.s;
  if (mode == kPredBoundaryRows) rhi = pd.b;
  if (mode == kPredOwnColumns && !thin) return;
  if (mode == kPredThickInner) {
    if (thin) return;
    rlo = pd.b;
  }
  const int r0 = rlo + blockIdx.z * kPredRows;
  if (r0 >= rhi) return;
  const int rows = min(kPredRows, rhi - r0);
  if (threadIdx.x < rows) src_s[threadIdx.x] = __ldg(st2ed + pd.start + r0 + threadIdx.x);
  __syncthreads();
  const T inf = Dist<T>::inf();
  const int jj = blockIdx.x * kPredThreads + threadIdx.x;
  int j = jj;
  if (mode == kPredOwnColumns) {
    if (jj >= pd.s) return;
    j = __ldg(st2ed + pd.start + jj);
  }
  if (j >= n) return;
  // the column's in-edges, read once for all of the CTA's rows
  const int e0 = __ldg(tro + j), e1 = __ldg(tro + j + 1);
  const int dk = min(e1 - e0, kPredDeg);
  int us[kPredDeg];
  T ws[kPredDeg];
#pragma unroll
  for (int k = 0; k < kPredDeg; k++) {
    us[k] = k < dk ? __ldg(tcol + e0 + k) : j;
    ws[k] = k < dk ? __ldg(tw + e0 + k) : T(0);
  }
  const T *Dr = D + (pd.row_base + r0) * ldD;
  int32_t *Pr = P + (pd.row_base + r0) * ldD + j;
  for (int rr = 0; rr < rows; rr += kPredUnroll, Dr += kPredUnroll * ldD, Pr += kPredUnroll * ldD) {
    T dj[kPredUnroll], g[kPredUnroll][kPredDeg];
#pragma unroll
    for (int q = 0; q < kPredUnroll; q++) {
      const bool live = rr + q < rows;
      const T *Dq = Dr + (int64_t)q * ldD;
      dj[q] = live ? __ldg(Dq + j) : inf;
#pragma unroll
      for (int k = 0; k < kPredDeg; k++) g[q][k] = (live && k < dk) ? __ldg(Dq + us[k]) : inf;
    }
#pragma unroll
    for (int q = 0; q < kPredUnroll; q++) {
      if (rr + q >= rows) break;
      const int src = src_s[rr + q];
      uint64_t best = ~0ull;
#pragma unroll
      for (int k = 0; k < kPredDeg; k++)
        if (k < dk) best = min(best, pred_key<T>(g[q][k], us[k], ws[k], inf));
      if (e1 - e0 > kPredDeg) {
        const T *Dq = Dr + (int64_t)q * ldD;
        for (int e = e0 + kPredDeg; e < e1; e++) {
          const int u = __ldg(tcol + e);
          best = min(best, pred_key<T>(__ldg(Dq + u), u, __ldg(tw + e), inf));
        }
      }
      int pred = best == ~0ull ? -1 : (int)(uint32_t)best;
      if (dj[q] >= inf) pred = -1;
      if (j == src) pred = src;
      Pr[(int64_t)q * ldD] = pred;
    }
  }
}

// Inner rows of parts with b <= kPredThinB, all columns: the predecessor of
// j on the path through the boundary vertex k* that the min-plus merge
// chose (the first k with the least F[i][k] + D[k][j]) is the predecessor
// on k*'s row: P[i][j] = P[k*][j] (-1 where unreachable).  A CTA owns a
// strip of kPredStrip columns of one part and a block of up to 128 inner
// rows: the strip of the b boundary rows sits in registers (distances) and
// shared memory (predecessors), the rows' F values in shared memory; every
// warp stores 512 contiguous bytes per row.  Own-part columns are left for
// the own-column pass (their decode is the closure, not a min-plus).
constexpr int kPredStrip = 4 * kPredThreads;

template <typename T, int B>
__device__ __forceinline__ void pred_thin_rows(const PartDesc &pd, const T *D, int32_t *P, int64_t ldD,
                                               int64_t c0, bool live, int m0, int rows,
                                               const T (*As)[kPredThinB], const int32_t (*Ps)[kPredStrip]) {
  using V = typename Vec4<T>::type;
  const T inf = Dist<T>::inf();
  T sv[B > 0 ? B : 1][4];
#pragma unroll
  for (int k = 0; k < B; k++) {
    V v;
    if (live) v = __ldg(reinterpret_cast<const V *>(D + (pd.row_base + k) * ldD + c0));
    else v.x = v.y = v.z = v.w = inf;
    sv[k][0] = v.x; sv[k][1] = v.y; sv[k][2] = v.z; sv[k][3] = v.w;
  }
  const int cl = 4 * threadIdx.x;
  for (int r = 0; r < rows; r++) {
    T best[4];
    int arg[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      best[q] = inf;
      arg[q] = -1;
    }
#pragma unroll
    for (int k = 0; k < B; k++) {
      const T a = As[r][k];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const T v = a + sv[k][q];
        if (v < best[q]) {
          best[q] = v;
          arg[q] = k;
        }
      }
    }
    int4 out;
    out.x = arg[0] >= 0 ? Ps[arg[0] > 0 ? arg[0] : 0][cl + 0] : -1;
    out.y = arg[1] >= 0 ? Ps[arg[1] > 0 ? arg[1] : 0][cl + 1] : -1;
    out.z = arg[2] >= 0 ? Ps[arg[2] > 0 ? arg[2] : 0][cl + 2] : -1;
    out.w = arg[3] >= 0 ? Ps[arg[3] > 0 ? arg[3] : 0][cl + 3] : -1;
    if (live) __stcs(reinterpret_cast<int4 *>(P + (pd.row_base + pd.b + m0 + r) * ldD + c0), out);
  }
}

template <typename T>
__global__ void __launch_bounds__(kPredThreads)
    pred_thin_kernel(const PartDesc *__restrict__ parts, const T *__restrict__ F, const T *D, int32_t *P,
                     int64_t ldD) {
  extern __shared__ __align__(16) unsigned char pt_smem_raw[];
  int32_t (*Ps)[kPredStrip] = reinterpret_cast<int32_t (*)[kPredStrip]>(pt_smem_raw);
  T (*As)[kPredThinB] =
      reinterpret_cast<T (*)[kPredThinB]>(pt_smem_raw + sizeof(int32_t) * kPredThinB * kPredStrip);
  const PartDesc pd = parts[blockIdx.y];
  if (pd.b > kPredThinB) return;
  const int m0 = blockIdx.z * 128;
  const int M = pd.s - pd.b;
  if (m0 >= M) return;
  const int rows = min(128, M - m0);
  const int64_t c0 = (int64_t)blockIdx.x * kPredStrip + 4 * threadIdx.x;
  const bool live = c0 < ldD;  // ldD is a multiple of 4
  for (int t = threadIdx.x; t < 128 * kPredThinB; t += blockDim.x) {
    const int r = t / kPredThinB, k = t % kPredThinB;
    As[r][k] = (r < rows && k < pd.b) ? __ldg(F + pd.f_off + (int64_t)(pd.b + m0 + r) * pd.ldf + k)
                                      : Dist<T>::inf();
  }
  for (int k = 0; k < pd.b; k++) {
    int4 v = make_int4(-1, -1, -1, -1);
    if (live) v = *reinterpret_cast<const int4 *>(P + (pd.row_base + k) * ldD + c0);
    *reinterpret_cast<int4 *>(&Ps[k][4 * threadIdx.x]) = v;
  }
  __syncthreads();
  switch (pd.b) {
#define FAPB_PRED_CASE(NB) \
  case NB: pred_thin_rows<T, NB>(pd, D, P, ldD, c0, live, m0, rows, As, Ps); break;
    FAPB_PRED_CASE(0) FAPB_PRED_CASE(1) FAPB_PRED_CASE(2) FAPB_PRED_CASE(3) FAPB_PRED_CASE(4)
    FAPB_PRED_CASE(5) FAPB_PRED_CASE(6) FAPB_PRED_CASE(7) FAPB_PRED_CASE(8) FAPB_PRED_CASE(9)
    FAPB_PRED_CASE(10) FAPB_PRED_CASE(11) FAPB_PRED_CASE(12)
#undef FAPB_PRED_CASE
    default: break;
  }
}

template <typename T>
cudaError_t launch_pred(const PartDesc *parts, int nparts, int max_s, const T *D, int32_t *P,
                        int64_t ldD, int n, const int32_t *tro, const int32_t *tcol, const T *tw,
                        const int32_t *st2ed, const T *F, cudaStream_t stream, int64_t *launches) {
  if (nparts <= 0 || max_s <= 0 || n <= 0) return cudaSuccess;
  const unsigned gz = (unsigned)ceil_div(max_s, kPredRows);
  // 1. boundary rows, all columns (the gather rule)
  pred_kernel<T><<<dim3((unsigned)ceil_div(n, kPredThreads), nparts, gz), kPredThreads, 0, stream>>>(
      parts, D, P, ldD, n, tro, tcol, tw, st2ed, kPredBoundaryRows);
  // 2. inner rows of thin parts from the min-plus argmin (own columns redone by 3)
  const size_t smem = sizeof(int32_t) * kPredThinB * kPredStrip + sizeof(T) * 128 * kPredThinB;
  cudaError_t e =
      cudaFuncSetAttribute(pred_thin_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  pred_thin_kernel<T><<<dim3((unsigned)ceil_div(ldD, kPredStrip), nparts, (unsigned)ceil_div(max_s, 128)),
                        kPredThreads, smem, stream>>>(parts, F, D, P, ldD);
  // 3. own-part columns of thin parts (the gather rule)
  pred_kernel<T><<<dim3((unsigned)ceil_div(max_s, kPredThreads), nparts, gz), kPredThreads, 0, stream>>>(
      parts, D, P, ldD, n, tro, tcol, tw, st2ed, kPredOwnColumns);
  // 4. inner rows of the other parts (the gather rule)
  pred_kernel<T><<<dim3((unsigned)ceil_div(n, kPredThreads), nparts, gz), kPredThreads, 0, stream>>>(
      parts, D, P, ldD, n, tro, tcol, tw, st2ed, kPredThickInner);
  *launches += 4;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Boundary-graph form of stage 1
// ---------------------------------------------------------------------------
// Every shortest path between boundary vertices is a chain of segments
// inside one part (between two of its boundary vertices: the local closure)
// and cross-part arcs (both ends are boundary vertices by construction,
// fap/utils/util_preprocess.h:32-58).  dB closed by Floyd is therefore exact;
// a path from a boundary vertex into part q last enters q at one of q's
// boundary vertices b' and stays in q, so D[g][v] = min_b' dB[g][b'] +
// F_q[b'][v] is the exact shortest distance.
template <typename T>
__global__ void bgraph_local_kernel(const PartDesc *__restrict__ parts, const T *__restrict__ F, T *dB,
                                    int64_t ldB) {
  const PartDesc pd = parts[blockIdx.y];
  const int i = blockIdx.x;
  if (i >= pd.b) return;
  const T *Fi = F + pd.f_off + (int64_t)i * pd.ldf;
  T *Bi = dB + ((int64_t)pd.bd_row + i) * ldB + pd.bd_row;
  for (int k = threadIdx.x; k < pd.b; k += blockDim.x) Bi[k] = Fi[k];
}

template <typename T>
__global__ void bgraph_cross_kernel(const int32_t *__restrict__ row_offset, const int32_t *__restrict__ col,
                                    const T *__restrict__ w, int n, const int32_t *__restrict__ graph_id,
                                    const int32_t *__restrict__ ed2st, const BPart *__restrict__ bpart,
                                    T *dB, int64_t ldB) {
  for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    const int pu = __ldg(graph_id + u);
    const int e0 = __ldg(row_offset + u), e1 = __ldg(row_offset + u + 1);
    int gu = -1;
    for (int e = e0; e < e1; e++) {
      const int v = __ldg(col + e);
      const int pv = __ldg(graph_id + v);
      if (pv == pu) continue;
      if (gu < 0) {
        const BPart P = bpart[pu];
        const int lu = __ldg(ed2st + u) - P.voff;
        if (lu < 0 || lu >= P.b) break;  // not a boundary vertex: cannot happen
        gu = P.boff + lu;
      }
      const BPart Q = bpart[pv];
      const int lv = __ldg(ed2st + v) - Q.voff;
      if (lv < 0 || lv >= Q.b) continue;
      Dist<T>::atomic_min(dB + (int64_t)gu * ldB + Q.boff + lv, __ldg(w + e));
    }
  }
}

template <typename T>
cudaError_t launch_bgraph(const PartDesc *parts, int nparts, int max_b, const T *F, T *dB, int64_t ldB,
                          const int32_t *row_offset, const int32_t *col, const T *w, int n,
                          const int32_t *graph_id, const int32_t *ed2st, const BPart *bpart,
                          cudaStream_t stream, int64_t *launches) {
  cudaError_t e = launch_fill<T>(dB, ldB, ldB, ldB, Dist<T>::inf(), stream, launches);
  if (e != cudaSuccess) return e;
  if (nparts > 0 && max_b > 0) {
    bgraph_local_kernel<T><<<dim3(max_b, nparts), 128, 0, stream>>>(parts, F, dB, ldB);
    *launches += 1;
  }
  const int blocks = (int)std::min<int64_t>(ceil_div(n, 256), device_sm_count() * 8);
  bgraph_cross_kernel<T><<<blocks, 256, 0, stream>>>(row_offset, col, w, n, graph_id, ed2st, bpart, dB, ldB);
  *launches += 1;
  return cudaGetLastError();
}

// Column table of the expansion: Tc[k][v] = F_q[k][j] for the column's part
// q (local index j) and k < b_q, the sentinel for b_q <= k < maxb, so that
// the expansion reads a column's boundary entries with coalesced loads (the
// F arena itself is ordered by part, the output by original vertex id).
// One read of every part's boundary rows per solve.
template <typename T>
__global__ void bdy_coltable_kernel(const BPart *__restrict__ bpart, const int32_t *__restrict__ graph_id,
                                    const int32_t *__restrict__ ed2st, int n, const T *__restrict__ F, int maxb,
                                    T *Tc, int64_t ldT) {
  const T inf = Dist<T>::inf();
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < ldT; v += (int64_t)gridDim.x * blockDim.x) {
    int qb = 0;
    const T *Fq = nullptr;
    int64_t ldq = 0;
    if (v < n) {
      const BPart Q = bpart[__ldg(graph_id + v)];
      qb = Q.b;
      Fq = F + Q.f_off + (__ldg(ed2st + v) - Q.voff);
      ldq = Q.ldf;
    }
    for (int k = 0; k < maxb; k++) Tc[k * ldT + v] = k < qb ? __ldg(Fq + k * ldq) : inf;
  }
}

// grid (column chunks, groups of kExpandRows listed rows); the rows' dB
// entries sit in shared memory; a thread computes whole output columns
// (coalesced stores in original column order) from the boundary rows of the
// column's part, read once for all of the CTA's rows (from the column table
// Tc when it is given, else from the F arena).  Own-part entries are
// also written to FB[g][j] (the exact distances from boundary vertex g to
// its part's vertices, for the local-closure fix-up).  RG rows per CTA:
// 32 where their dB entries fit in shared memory (each scattered F load
// then serves 32 rows), else 8.
constexpr int kExpandRows = 8;
constexpr int kExpandRowsWide = 32;

template <typename T, int RG>
__global__ void __launch_bounds__(256)
    bdy_expand_kernel(const int64_t *__restrict__ rows, int nrows, const BPart *__restrict__ bpart,
                      const int32_t *__restrict__ graph_id, const int32_t *__restrict__ ed2st, int n,
                      const T *__restrict__ dB, int64_t ldB, int nbB, const T *__restrict__ F, T *D,
                      int64_t ldD, T *FB, int64_t ldFB, const T *__restrict__ Tc) {
  extern __shared__ __align__(16) unsigned char bx_smem_raw[];
  // rows of RG x nbB dB entries, each padded to a multiple of 4 so that they
  // are staged with 16-byte loads, eight in flight per thread (dB rows start
  // on 512-byte boundaries and hold ldB >= that many entries)
  using V = typename Vec4<T>::type;
  const int nbs = (nbB + 3) & ~3, nvr = nbs / 4;
  T *drow = reinterpret_cast<T *>(bx_smem_raw);  // RG x nbs
  const int r0 = blockIdx.y * RG;
  const int nr = min(RG, nrows - r0);
  int64_t g[RG], dr[RG];
#pragma unroll
  for (int q = 0; q < RG; q++) {
    g[q] = q < nr ? rows[2 * (r0 + q)] : 0;
    dr[q] = q < nr ? rows[2 * (r0 + q) + 1] : 0;
  }
  for (int t0 = threadIdx.x; t0 < nr * nvr; t0 += 8 * blockDim.x) {
    V tmp[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int t = t0 + u * blockDim.x;
      if (t < nr * nvr)
        tmp[u] = __ldg(reinterpret_cast<const V *>(dB + rows[2 * (r0 + t / nvr)] * ldB) + t % nvr);
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int t = t0 + u * blockDim.x;
      if (t < nr * nvr) reinterpret_cast<V *>(drow)[t] = tmp[u];
    }
  }
  __syncthreads();
  const T inf = Dist<T>::inf();
  // (the next column's part and local index are loaded while this one's
  // minima run)
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int gv = v < n ? __ldg(graph_id + v) : 0, ev = v < n ? __ldg(ed2st + v) : 0;
  for (; v < ldD; v += stride) {
    const int64_t vn = v + stride;
    const int gn = vn < n ? __ldg(graph_id + vn) : 0, en = vn < n ? __ldg(ed2st + vn) : 0;
    T acc[RG];
#pragma unroll
    for (int q = 0; q < RG; q++) acc[q] = inf;
    int j = -1, qb = 0, qoff = 0;
    if (v < n) {
      const BPart Q = bpart[gv];
      j = ev - Q.voff;
      qb = Q.b;
      qoff = Q.boff;
      const T *Fq = Tc ? Tc + v : F + Q.f_off + j;
      const int64_t ldq = Tc ? ldD : Q.ldf;
      for (int k = 0; k < Q.b; k++) {
        const T f = __ldg(Fq + (int64_t)k * ldq);
#pragma unroll
        for (int q = 0; q < RG; q++) acc[q] = Dist<T>::relax(drow[q * nbs + Q.boff + k], f, acc[q]);
      }
    }
    gv = gn;
    ev = en;
#pragma unroll
    for (int q = 0; q < RG; q++) {
      if (q >= nr) break;
      D[dr[q] * ldD + v] = acc[q];
      if (j >= 0 && g[q] >= qoff && g[q] < qoff + qb) FB[g[q] * ldFB + j] = acc[q];
    }
  }
}

template <typename T, int RG>
cudaError_t launch_bdy_expand_rg(const int64_t *rows, int nrows, const BPart *bpart, const int32_t *graph_id,
                                 const int32_t *ed2st, int n, const T *dB, int64_t ldB, int nbB, const T *F,
                                 T *D, int64_t ldD, T *FB, int64_t ldFB, const T *Tc, cudaStream_t stream,
                                 int64_t *launches) {
  const size_t smem = (size_t)RG * round_up(std::max(nbB, 1), 4) * sizeof(T);
  if (ldB < round_up(std::max(nbB, 1), 4) || ldB % 4 != 0) return cudaErrorInvalidValue;
  auto kern = bdy_expand_kernel<T, RG>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  // Enough CTAs for about 16 per SM, each looping over columns so that the
  // rows' dB entries are staged only once per CTA.
  const int64_t ny = ceil_div(nrows, RG);
  const int bx = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(ldD, 256), ceil_div((int64_t)device_sm_count() * 16, ny)));
  kern<<<dim3(bx, (unsigned)ny), 256, smem, stream>>>(
      rows, nrows, bpart, graph_id, ed2st, n, dB, ldB, nbB, F, D, ldD, FB, ldFB, Tc);
  *launches += 1;
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_bdy_expand(const int64_t *rows, int nrows, const BPart *bpart, const int32_t *graph_id,
                              const int32_t *ed2st, int n, const T *dB, int64_t ldB, int nbB, const T *F,
                              T *D, int64_t ldD, T *FB, int64_t ldFB, T *Tc, int maxb, cudaStream_t stream,
                              int64_t *launches) {
  if (nrows <= 0) return cudaSuccess;
  if (Tc) {
    const int blocks = (int)std::min<int64_t>(ceil_div(ldD, 256), (int64_t)device_sm_count() * 8);
    bdy_coltable_kernel<T><<<blocks, 256, 0, stream>>>(bpart, graph_id, ed2st, n, F, maxb, Tc, ldD);
    *launches += 1;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if ((size_t)kExpandRowsWide * round_up(std::max(nbB, 1), 4) * sizeof(T) <= 160 * 1024)
    return launch_bdy_expand_rg<T, kExpandRowsWide>(rows, nrows, bpart, graph_id, ed2st, n, dB, ldB, nbB, F, D,
                                                     ldD, FB, ldFB, Tc, stream, launches);
  return launch_bdy_expand_rg<T, kExpandRows>(rows, nrows, bpart, graph_id, ed2st, n, dB, ldB, nbB, F, D, ldD,
                                              FB, ldFB, Tc, stream, launches);
}

// Boundary graph closed by Bellman-Ford in alternating steps (large
// boundary sets).  A shortest path between boundary vertices alternates
// segments inside one part (their lengths are the local closure F_p, already
// transitive) and cross-part arcs, so for kMsbfS sources at a time (tile
// Dt[g][s], boundary index g):
//   local step, per part p whose rows changed in the last cross step:
//     Dt[c][s] = min(Dt[c][s], min_a Dt[a][s] + F_p[a][c])
//   over the rows a that the cross step changed (the others were closed
//   before, and F_p is transitive): a min-plus product run from shared
//   memory, 128 sources x 64 columns per CTA, K = the changed rows; rows
//   that improve are stamped for the cross step;
//   cross step: every head of a cross-part arc whose tail row changed since
//   the last cross step (a work list) pulls over its cross-part in-arcs (one
//   warp per head row, plain stores); heads that improve put their own
//   arcs' heads on the next list and stamp their parts for the next local
//   step.
// Stamps are iteration numbers (per boundary vertex: cact, the list its
// out-arcs' heads last went to from a local step or the seed (several
// threads of a local step may change one row); hact, the list it last
// joined as a head;
// lact, the iteration whose local step takes it as a changed row; per part:
// pact, the local step to run), so nothing is cleared between iterations or
// tiles.  The work list of iteration t (entries z * nb + g) is filled by the
// cross step t - 1 and the local step t and read by the cross step t; lists
// alternate between two buffers by parity, and the local step t empties the
// list t + 1 before the cross step t fills it.  Values only decrease
// and each is a path length, so the fixed point (no cross-step improvement)
// is the exact closure whatever the order of the updates.
template <typename T>
using LStepCfg = TileCfg<T, kMsbfS, 64, 16, 8, 4>;

constexpr int kLStepList = 2048;  // changed rows listed per part (larger parts take all rows)

// Several tiles run side by side (blockIdx.z / the item range): tile z has
// its own Dt, xact, lact (nb each) and pact (K + 1) at offset z; its sources
// are s0 + z * kMsbfS + s for s < kMsbfS and below nb.
// Reserves one slot of a work list whose length is *count: the lanes of a
// warp that call it together share one atomicAdd (a busy iteration appends
// hundreds of thousands of heads to the same counter).
__device__ __forceinline__ int wl_append(int *count) {
  const cg::coalesced_group g = cg::coalesced_threads();
  int base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(count, (int)g.size());
  return g.shfl(base, 0) + (int)g.thread_rank();
}

// Row g of tile z changed: the heads of g's cross-part out-arcs join the
// work list of iteration `stamp` (each row's heads once per list, each head
// once per list).  cact/hact point at tile z's stamps.
__device__ __forceinline__ void bgraph_mark_heads(int g, int64_t znb, int *cact, int *hact, int stamp,
                                                  const int32_t *__restrict__ otro,
                                                  const int32_t *__restrict__ otcol, int *wl, int *wl_count) {
  if (atomicExch(cact + g, stamp) == stamp) return;
  const int e1 = __ldg(otro + g + 1);
  for (int e = __ldg(otro + g); e < e1; e++) {
    const int h = __ldg(otcol + e);
    if (atomicExch(hact + h, stamp) != stamp)
      wl[(stamp & 1) * (int64_t)wl_count[2] + wl_append(wl_count + (stamp & 1))] = (int)(znb + h);
  }
}

template <typename T>
__global__ void bgraph_seed_kernel(T *Dt, int s0, int nb, int K1, const int32_t *__restrict__ gpart, int *cact,
                                   int *hact, int *lact, int *pact, int stamp, const int32_t *__restrict__ otro,
                                   const int32_t *__restrict__ otcol, int *wl, int *wl_count) {
  const int z = blockIdx.y, s = threadIdx.x;
  const int g = s0 + z * kMsbfS + s;
  if (g >= nb) return;
  const int64_t znb = (int64_t)z * nb;
  Dt[(znb + g) * kMsbfS + s] = T(0);
  bgraph_mark_heads(g, znb, cact + znb, hact + znb, stamp, otro, otcol, wl, wl_count);  // its cross arcs
  lact[znb + g] = stamp;  // and its part's rows
  pact[(int64_t)z * K1 + __ldg(gpart + g)] = stamp;
}

template <typename T>
__global__ void __launch_bounds__(LStepCfg<T>::THREADS)
    bgraph_lstep_kernel(const PartDesc *__restrict__ parts, const T *__restrict__ F, T *Dt, int nb, int K1,
                        const int *__restrict__ pact, const int *__restrict__ lact, int stamp, int *cact, int *hact,
                        const int32_t *__restrict__ otro, const int32_t *__restrict__ otcol, int *wl,
                        int *wl_count) {
  using C = LStepCfg<T>;
  using V = typename Vec4<T>::type;
  if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0) wl_count[(stamp + 1) & 1] = 0;
  const PartDesc pd = parts[blockIdx.y];
  const int c0 = blockIdx.x * C::BN;
  const int64_t z = blockIdx.z;
  if (c0 >= pd.b || __ldcg(pact + z * K1 + pd.part) != stamp) return;
  Dt += z * nb * kMsbfS;
  lact += z * nb;
  cact += z * nb;
  hact += z * nb;
  __shared__ __align__(16) T smem[C::SMEM_ELEMS];
  __shared__ int klist[kLStepList];
  __shared__ int kcount;
  const T inf = Dist<T>::inf();
  const int tid = threadIdx.x, ty = tid / C::TX, tx = tid % C::TX;
  const T *Dp = Dt + (int64_t)pd.bd_row * kMsbfS;  // rows a of the part: A^T (k = a, i = s)
  const T *Fp = F + pd.f_off + c0;                  // rows a, columns c0..: B (k = a, j = c)
  // the rows the last cross step (or the seed) changed
  const bool listed = pd.b <= kLStepList;
  if (tid == 0) kcount = 0;
  __syncthreads();
  if (listed)
    for (int a = tid; a < pd.b; a += C::THREADS)
      if (__ldcg(lact + pd.bd_row + a) == stamp) klist[atomicAdd(&kcount, 1)] = a;
  __syncthreads();
  const int K = listed ? kcount : pd.b;
  if (K == 0) return;
  auto krow = [&](int k) { return listed ? klist[k] : k; };
  constexpr int A4 = C::BK * C::BM / 4 / C::THREADS;  // 16-byte loads per thread and chunk
  constexpr int B4 = C::BK * C::BN / 4 / C::THREADS;
  static_assert(A4 * 4 * C::THREADS == C::BK * C::BM && B4 * 4 * C::THREADS == C::BK * C::BN, "even");
  V ra[A4], rb[B4];
  auto load = [&](int k0) {
#pragma unroll
    for (int r = 0; r < A4; r++) {
      const int idx = tid + r * C::THREADS, k = idx / (C::BM / 4), i4 = (idx % (C::BM / 4)) * 4;
      if (k0 + k < K) ra[r] = __ldcg(reinterpret_cast<const V *>(Dp + (int64_t)krow(k0 + k) * kMsbfS + i4));
      else ra[r] = V{inf, inf, inf, inf};
    }
#pragma unroll
    for (int r = 0; r < B4; r++) {
      const int idx = tid + r * C::THREADS, k = idx / (C::BN / 4), j4 = (idx % (C::BN / 4)) * 4;
      if (k0 + k < K) rb[r] = __ldg(reinterpret_cast<const V *>(Fp + (int64_t)krow(k0 + k) * pd.ldf + j4));
      else rb[r] = V{inf, inf, inf, inf};
    }
  };
  auto store = [&](T *As, T *Bs) {
#pragma unroll
    for (int r = 0; r < A4; r++) {
      const int idx = tid + r * C::THREADS, k = idx / (C::BM / 4), i4 = (idx % (C::BM / 4)) * 4;
      *reinterpret_cast<V *>(As + k * C::AP + i4) = ra[r];
    }
#pragma unroll
    for (int r = 0; r < B4; r++) {
      const int idx = tid + r * C::THREADS, k = idx / (C::BN / 4), j4 = (idx % (C::BN / 4)) * 4;
      *reinterpret_cast<V *>(Bs + k * C::BN + j4) = rb[r];
    }
  };
  T acc[C::TM][C::TN];
  acc_fill<T, C>(acc, inf);
  T *const As0 = smem;
  T *const Bs0 = smem + 2 * C::A_ELEMS;
  const int nchunks = (int)ceil_div(K, C::BK);
  load(0);
  store(As0, Bs0);
  __syncthreads();
  for (int c = 0; c < nchunks; c++) {
    const int cur = c & 1;
    if (c + 1 < nchunks) load((c + 1) * C::BK);
    mma_chunk<T, C>(As0 + cur * C::A_ELEMS, Bs0 + cur * C::B_ELEMS, acc, ty, tx, min(C::BK, K - c * C::BK));
    if (c + 1 < nchunks) store(As0 + (cur ^ 1) * C::A_ELEMS, Bs0 + (cur ^ 1) * C::B_ELEMS);
    __syncthreads();
  }
  // Rows c of the part: lower the thread's 4 consecutive sources per group.
#pragma unroll
  for (int gj = 0; gj < C::GN; gj++)
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int c = c0 + tile_col<C>(tx, gj, q);
      if (c >= pd.b) continue;
      T *row = Dt + ((int64_t)pd.bd_row + c) * kMsbfS;
      bool imp = false;
#pragma unroll
      for (int gi = 0; gi < C::GM; gi++) {
        const int s = tile_row<C>(ty, gi, 0);
        V cur = __ldcg(reinterpret_cast<const V *>(row + s));
        const T n0 = acc[4 * gi + 0][4 * gj + q], n1 = acc[4 * gi + 1][4 * gj + q];
        const T n2 = acc[4 * gi + 2][4 * gj + q], n3 = acc[4 * gi + 3][4 * gj + q];
        if (n0 < cur.x || n1 < cur.y || n2 < cur.z || n3 < cur.w) {
          imp = true;
          cur.x = min(cur.x, n0);
          cur.y = min(cur.y, n1);
          cur.z = min(cur.z, n2);
          cur.w = min(cur.w, n3);
          __stcg(reinterpret_cast<V *>(row + s), cur);
        }
      }
      if (imp) bgraph_mark_heads(pd.bd_row + c, z * nb, cact, hact, stamp, otro, otcol, wl, wl_count);
    }
}

template <typename T>
__global__ void __launch_bounds__(256)
    bgraph_xstep_kernel(T *Dt, int nb, int K1, const int32_t *__restrict__ itro, const int32_t *__restrict__ itcol,
                        const T *__restrict__ itw, const int32_t *__restrict__ otro,
                        const int32_t *__restrict__ otcol, int *cact, int *hact, int *lact, int stamp,
                        const int32_t *__restrict__ gpart, int *pact, int *wl, int *wl_count, int *changed) {
  using V = typename Vec4<T>::type;
  const T inf = Dist<T>::inf();
  // one head per half-warp (two heads in flight per warp), 8 sources a lane
  const int lane = threadIdx.x & 31, half = lane >> 4, hl = lane & 15;
  const int nwarps = gridDim.x * (blockDim.x >> 5);
  const int count = __ldcg(wl_count + (stamp & 1));
  const int *list = wl + (stamp & 1) * (int64_t)wl_count[2];
  const int t1 = stamp + 1;
  bool any_change = false;
  for (int base = 2 * (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)); base < count; base += 2 * nwarps) {
    const int it = base + half;
    const bool live = it < count;
    const int entry = live ? __ldcg(list + it) : 0;
    const int64_t z = entry / nb;
    const int v = entry - (int)(z * nb);
    T *Dz = Dt + z * nb * kMsbfS;
    T acc[8];
#pragma unroll
    for (int q = 0; q < 8; q++) acc[q] = inf;
    const int e0 = live ? __ldg(itro + v) : 0, e1 = live ? __ldg(itro + v + 1) : 0;
    for (int e = e0; e < e1; e += 4) {  // four tail rows in flight
      V d[4][2];
      T w[4];
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (e + q < e1) {
          const V *r = reinterpret_cast<const V *>(Dz + (int64_t)__ldg(itcol + e + q) * kMsbfS) + 2 * hl;
          d[q][0] = __ldcg(r);
          d[q][1] = __ldcg(r + 1);
          w[q] = __ldg(itw + e + q);
        }
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (e + q < e1)
#pragma unroll
          for (int h = 0; h < 2; h++) {
            acc[4 * h + 0] = Dist<T>::relax(d[q][h].x, w[q], acc[4 * h + 0]);
            acc[4 * h + 1] = Dist<T>::relax(d[q][h].y, w[q], acc[4 * h + 1]);
            acc[4 * h + 2] = Dist<T>::relax(d[q][h].z, w[q], acc[4 * h + 2]);
            acc[4 * h + 3] = Dist<T>::relax(d[q][h].w, w[q], acc[4 * h + 3]);
          }
    }
    bool imp = false;
    if (live) {  // this half-warp is the row's only writer in this step
      V *row = reinterpret_cast<V *>(Dz + (int64_t)v * kMsbfS) + 2 * hl;
#pragma unroll
      for (int h = 0; h < 2; h++) {
        V cur = __ldcg(row + h);
        if (acc[4 * h] < cur.x || acc[4 * h + 1] < cur.y || acc[4 * h + 2] < cur.z || acc[4 * h + 3] < cur.w) {
          imp = true;
          cur.x = min(cur.x, acc[4 * h]);
          cur.y = min(cur.y, acc[4 * h + 1]);
          cur.z = min(cur.z, acc[4 * h + 2]);
          cur.w = min(cur.w, acc[4 * h + 3]);
          __stcg(row + h, cur);
        }
      }
    }
    const unsigned bal = __ballot_sync(0xffffffffu, imp);
    if ((bal >> (16 * half)) & 0xffffu) {
      // the heads of v's out-arcs join the next list, one lane per arc
      const int f1 = __ldg(otro + v + 1);
      for (int e = __ldg(otro + v) + hl; e < f1; e += 16) {
        const int h = __ldg(otcol + e);
        if (atomicExch(hact + z * nb + h, t1) != t1)
          wl[(t1 & 1) * (int64_t)wl_count[2] + wl_append(wl_count + (t1 & 1))] = (int)(z * nb + h);
      }
      if (hl == 0) {
        lact[z * nb + v] = t1;
        pact[z * K1 + __ldg(gpart + v)] = t1;
      }
      any_change = true;
    }
  }
  // one store per warp that changed a row (the loop is warp-uniform)
  if (__any_sync(0xffffffffu, any_change) && lane == 0) *changed = 1;
}

template <typename T>
cudaError_t launch_bgraph_bf(const PartDesc *parts, int nparts, int max_b, const T *F, const int32_t *itro,
                             const int32_t *itcol, const T *itw, const int32_t *otro, const int32_t *otcol,
                             const int32_t *gpart, const int32_t *pcol, int nb, int K, int ztiles, T *dB,
                             int64_t ldB, T *Dt, int *act, int *pact, int *wl, int *wl_count, int *changed,
                             int *host_changed, int64_t max_rounds, int *status, cudaStream_t stream,
                             int64_t *launches) {
  using C = LStepCfg<T>;
  if (nb <= 0 || nparts <= 0) return cudaSuccess;
  if (nparts > 65535 || ztiles < 1 || ztiles > 64) return cudaErrorInvalidConfiguration;
  const int K1 = K + 1;
  int *cact = act, *hact = act + (int64_t)ztiles * nb, *lact = act + (int64_t)2 * ztiles * nb;
  if ((int64_t)ztiles * nb >= INT32_MAX) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(act, 0xff, (size_t)3 * ztiles * nb * sizeof(int), stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(pact, 0xff, (size_t)ztiles * K1 * sizeof(int), stream);
  // wl_count: the two lists' lengths and the capacity of each list
  const int counts[3] = {0, 0, ztiles * nb};
  if (e == cudaSuccess) e = cudaMemcpyAsync(wl_count, counts, sizeof(counts), cudaMemcpyHostToDevice, stream);
  if (e != cudaSuccess) return e;
  constexpr int kChunk = 4;  // iterations between convergence checks
  int stamp = 0;
  for (int s0 = 0; s0 < nb; s0 += ztiles * kMsbfS) {
    const int z = (int)std::min<int64_t>(ztiles, ceil_div(nb - s0, kMsbfS));  // tiles side by side
    const dim3 lgrid((unsigned)ceil_div(std::max(max_b, 1), C::BN), (unsigned)nparts, (unsigned)z);
    const int xblocks = device_sm_count() * 5;  // about the resident limit at 256 threads
    e = launch_fill<T>(Dt, (int64_t)z * nb, kMsbfS, kMsbfS, Dist<T>::inf(), stream, launches);
    if (e == cudaSuccess) e = cudaMemsetAsync(wl_count, 0, 2 * sizeof(int), stream);
    if (e != cudaSuccess) return e;
    bgraph_seed_kernel<T><<<dim3(1, z), kMsbfS, 0, stream>>>(Dt, s0, nb, K1, gpart, cact, hact, lact, pact, stamp,
                                                            otro, otcol, wl, wl_count);
    *launches += 1;
    bool done = false;
    for (int64_t round = 0; !done; round += kChunk) {
      if (round >= max_rounds) {
        e = cudaMemcpyAsync(status, &kMsbfRoundLimit, sizeof(int), cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return e;
        break;
      }
      e = cudaMemsetAsync(changed, 0, kChunk * sizeof(int), stream);
      if (e != cudaSuccess) return e;
      for (int c = 0; c < kChunk; c++, stamp++) {
        bgraph_lstep_kernel<T><<<lgrid, C::THREADS, 0, stream>>>(parts, F, Dt, nb, K1, pact, lact, stamp, cact, hact,
                                                                 otro, otcol, wl, wl_count);
        bgraph_xstep_kernel<T><<<xblocks, 256, 0, stream>>>(Dt, nb, K1, itro, itcol, itw, otro, otcol, cact, hact,
                                                            lact, stamp, gpart, pact, wl, wl_count, changed + c);
        *launches += 2;
      }
      e = cudaMemcpyAsync(host_changed, changed, kChunk * sizeof(int), cudaMemcpyDeviceToHost, stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
      if (e != cudaSuccess) return e;
      for (int c = 0; c < kChunk; c++) done |= host_changed[c] == 0;
    }
    for (int q = 0; q < z; q++) {
      const int sq = s0 + q * kMsbfS;
      msbf_store_kernel<T><<<(unsigned)ceil_div(nb, 32), 256, 0, stream>>>(Dt + (int64_t)q * nb * kMsbfS, nb, sq,
                                                                          std::min(kMsbfS, nb - sq), dB, ldB,
                                                                          nullptr, nb, pcol);
    }
    *launches += z;
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Expansion with TMA-fed tiles: A = dB rows m0.. at part q's padded
// boundary columns (bd_col.., a 16-byte start), B = q's local rows
// F_q[0..b_q) over columns n0.. (the arena map), K = b_q; the stores go to
// the columns' original ids (st2ed), own-part values also to FB.
// Packed-form bounds of the expansion (Expand16): grid (128-row tiles of dB,
// parts), warp w takes rows m0 + w, m0 + w + 8, ...; its lanes read the
// row's b_q entries of part q's boundary columns (coalesced).
__global__ void __launch_bounds__(256)
    expand16_rows_kernel(const PartDesc *__restrict__ parts, int nbB, const int32_t *__restrict__ dB,
                         int64_t ldB, Expand16 xk) {
  const PartDesc pd = parts[blockIdx.y];
  const int m0 = blockIdx.x * 128, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int32_t tile_range = 0;
  for (int r = warp; r < 128; r += 8) {
    const int g = m0 + r;
    if (g >= nbB) break;
    const int32_t *row = dB + (int64_t)g * ldB + pd.bd_col;
    int32_t lo = INT32_MAX, hi = 0;
    for (int k = lane; k < pd.b; k += 32) {
      const int32_t v = __ldg(row + k);
      if (v < kInfI32) {
        lo = min(lo, v);
        hi = max(hi, v);
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (lane == 0) {
      xk.off[(int64_t)blockIdx.y * nbB + g] = lo == INT32_MAX ? 0 : lo;
      tile_range = max(tile_range, lo == INT32_MAX ? 0 : hi - lo);
    }
  }
  __shared__ int32_t red[8];
  if (lane == 0) red[warp] = tile_range;
  __syncthreads();
  if (threadIdx.x == 0) {
    int32_t m = 0;
    for (int w = 0; w < 8; w++) m = max(m, red[w]);
    xk.range[(int64_t)blockIdx.y * xk.nrt + blockIdx.x] = m;
  }
}

// Largest finite F_q[b'][v] (b' < b_q, v < s_q) of every part (one CTA per
// part); a negative entry (never produced from non-negative weights) makes
// the part's tiles run in int32.
__global__ void __launch_bounds__(256)
    expand16_maxb_kernel(const PartDesc *__restrict__ parts, const int32_t *__restrict__ F, Expand16 xk) {
  const PartDesc pd = parts[blockIdx.x];
  const int64_t cnt = (int64_t)pd.b * pd.s;
  int32_t m = 0;
  for (int64_t e = threadIdx.x; e < cnt; e += blockDim.x) {
    const int32_t v = __ldg(F + pd.f_off + (e / pd.s) * pd.ldf + e % pd.s);
    if (v < 0) m = kPackCap;
    else if (v < kInfI32) m = max(m, v);
  }
  __shared__ int32_t red[8];
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    int32_t x = 0;
    for (int w = 0; w < 8; w++) x = max(x, red[w]);
    xk.maxB[blockIdx.x] = x;
  }
}

// Tiled expansion (any boundary count): grid (column tiles, 128-row tiles of
// dB, parts); a CTA is a min-plus tile dB[g][b'_q] (x) F_q[b'][j] written
// to D rows grow[g], columns st2ed[start_q + j] (and, for g of part q itself,
// to FB).  PACK (int32): a tile whose values provably fit (Expand16) runs
// the packed 16-bit engine with its rows shifted by their offsets.
template <typename T, int PACK>
__global__ void __launch_bounds__(FloydCfg<T, kFloydTile>::THREADS, 2)
    bdy_expand_tma_kernel(const PartDesc *__restrict__ parts, int nbB, const int64_t *__restrict__ grow,
                          const int32_t *__restrict__ st2ed, T *D, int64_t ldD, T *FB, int64_t ldFB,
                          const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                          int *status, Expand16 xk, const __grid_constant__ CUtensorMap mapAP,
                          const __grid_constant__ CUtensorMap mapBD) {
  using TC = typename FloydCfg<T, kFloydTile>::TC;
  extern __shared__ __align__(128) unsigned char bxt_smem_raw[];
  const PartDesc pd = parts[blockIdx.z];
  // column tiles vary fastest: consecutive CTAs share their A tile (dB rows
  // of part q's boundary columns) in L2; q's B tiles are small enough to stay
  const int n0 = blockIdx.x * TC::BN, m0 = blockIdx.y * TC::BM;
  if (n0 >= pd.s) return;
  auto sm = tma_smem_init<T, TC>(bxt_smem_raw);
  T acc[8][8];
  const int fz = (int)(pd.f_off / ((int64_t)pd.ldf * pd.ldf));
  bool packed = false;
  if constexpr (PACK != 0) {
    packed = __ldg(xk.range + (int64_t)blockIdx.z * xk.nrt + blockIdx.y) + __ldg(xk.maxB + blockIdx.z) < kPackCap;
    if (threadIdx.x == 0) {
      atomicAdd(xk.tiles + 1, 1ull);
      if (packed) atomicAdd(xk.tiles, 1ull);
    }
  }
  if (packed) {
    if constexpr (PACK != 0) {
      using P = Pack16Cfg<TC>;
      // row offsets: after the packed buffers (PACK 1), after the packed
      // ring in the int32 ring's memory (PACK 2)
      int32_t *roff =
          PACK == 1 ? reinterpret_cast<int32_t *>(reinterpret_cast<uint32_t *>(smem_align128(bxt_smem_raw) +
                                                                               P::BUF_OFFSET) +
                                                  2 * P::BUF_ELEMS) +
                          TC::BN
                    : reinterpret_cast<int32_t *>(reinterpret_cast<unsigned char *>(sm.ring) +
                                                  Pack16qCfg<TC>::STAGE_WORDS * 4 * TC::STAGES);
      for (int r = threadIdx.x; r < TC::BM; r += blockDim.x)
        roff[r] = m0 + r < nbB ? __ldg(xk.off + (int64_t)blockIdx.z * nbB + m0 + r) : 0;
      uint32_t a16[4][8];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) a16[i][j] = kPackInit;
      // (the engine's first barrier orders the row offsets before use)
      bool ok;
      if constexpr (PACK == 1) {
        uint32_t *pbuf = reinterpret_cast<uint32_t *>(smem_align128(bxt_smem_raw) + P::BUF_OFFSET);
        ok = tma_minplus_tile16<TC>(&mapA, pd.bd_col, m0, 0, &mapB, n0, 0, fz, pd.b, a16, sm, pbuf, roff, nullptr,
                                    nbB - m0);
      } else {
        ok = tma_minplus_tile16q<TC>(&mapAP, m0 / 2, &mapBD, n0, pd.bd_row, pd.b, a16, sm, nbB - m0);
      }
      if (!ok) {
        if (threadIdx.x == 0) set_status(status, kDevTmaTimeout);
        return;
      }
      const int ty = threadIdx.x / TC::TX;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        // pair i = 2g + h holds rows 4g + 2h and 4g + 2h + 1 of the thread
        const int r0 = 4 * (i / 2) + 2 * (i % 2);
        const int tr = (i / 2) * (TC::BM / 2) + ty * 4 + 2 * (i % 2);   // tile row of the pair's first
        const int32_t o0 = roff[tr], o1 = roff[tr + 1];
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const int32_t lo = (int32_t)(int16_t)(a16[i][j] & 0xffffu);
          const int32_t hi = (int32_t)(int16_t)(a16[i][j] >> 16);
          acc[r0][j] = lo < kPackCap ? lo + o0 : Dist<T>::inf();
          acc[r0 + 1][j] = hi < kPackCap ? hi + o1 : Dist<T>::inf();
        }
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
      for (int j = 0; j < 8; j++) acc[i][j] = Dist<T>::inf();
    if (!tma_minplus_tile<T, TC>(&mapA, pd.bd_col, m0, 0, &mapB, n0, 0, fz, pd.b, acc, sm)) {
      if (threadIdx.x == 0) set_status(status, kDevTmaTimeout);
      return;
    }
  }
  const int tid = threadIdx.x, ty = tid / TC::TX, tx = tid % TC::TX;
  int col[8];
#pragma unroll
  for (int g = 0; g < 2; g++)
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int j = n0 + g * (TC::BN / 2) + tx * 4 + q;
      col[4 * g + q] = j < pd.s ? __ldg(st2ed + pd.start + j) : -1;
    }
#pragma unroll
  for (int gi = 0; gi < 2; gi++)
#pragma unroll
    for (int l = 0; l < 4; l++) {
      const int r = m0 + gi * (TC::BM / 2) + ty * 4 + l;
      if (r >= nbB) continue;
      T *dst = D + __ldg(grow + r) * ldD;
      const bool own = r >= pd.bd_row && r < pd.bd_row + pd.b;
      T *fb = FB + (int64_t)r * ldFB + n0;
#pragma unroll
      for (int g = 0; g < 2; g++)
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int c = col[4 * g + q];
          if (c < 0) continue;
          const T v = acc[4 * gi + l][4 * g + q];
          __stcs(dst + c, v);
          if (own) fb[g * (TC::BN / 2) + tx * 4 + q] = v;
        }
    }
}

// Pre-packed A operand of the packed expansion tiles (Expand16::ap): CTA
// (x, y, q) packs dB rows 128x .. 128x+127 at part q's boundary columns
// bd_col + 32y .. +31 through a shared-memory transpose: reads along k,
// writes along the row pairs.  Rows past nbB read as having no finite entry.
__global__ void __launch_bounds__(256)
    expand16_pack_a_kernel(const PartDesc *__restrict__ parts, int nbB, const int32_t *__restrict__ dB,
                           int64_t ldB, Expand16 xk) {
  const PartDesc pd = parts[blockIdx.z];
  const int g0 = blockIdx.x * 128, k0 = blockIdx.y * 32;
  if (k0 >= pd.b) return;
  __shared__ uint16_t t[32][130];
  const int tid = threadIdx.x;
  const int32_t *off = xk.off + (int64_t)blockIdx.z * nbB;
#pragma unroll 4
  for (int q = 0; q < 16; q++) {
    const int r = tid / 32 + 8 * q, k = tid % 32;
    const int g = g0 + r;
    int32_t v = kPackCap;
    if (g < nbB && k0 + k < pd.b) v = pack_clamp(__ldg(dB + (int64_t)g * ldB + pd.bd_col + k0 + k), __ldg(off + g));
    t[k][r] = (uint16_t)v;
  }
  __syncthreads();
#pragma unroll 4
  for (int q = 0; q < 8; q++) {
    const int p = tid % 64, k = tid / 64 + 4 * q;
    const int gp = g0 / 2 + p;
    if (k0 + k < pd.b && gp < xk.ap_ld)
      xk.ap[(int64_t)(pd.bd_row + k0 + k) * xk.ap_ld + gp] = (uint32_t)t[k][2 * p] | ((uint32_t)t[k][2 * p + 1] << 16);
  }
}

// Pre-packed B operand (Expand16::bd): row bd_row + k of part q holds
// F_q[k][v] clamped at kPackCap in both halves (kPackCap past s_q).
__global__ void __launch_bounds__(256)
    expand16_pack_b_kernel(const PartDesc *__restrict__ parts, const int32_t *__restrict__ F, Expand16 xk) {
  const PartDesc pd = parts[blockIdx.z];
  const int k = blockIdx.y;
  if (k >= pd.b) return;
  const int v = blockIdx.x * 256 + threadIdx.x;
  if (v >= xk.bd_ld) return;
  const int32_t x = v < pd.s ? min(__ldg(F + pd.f_off + (int64_t)k * pd.ldf + v), kPackCap) : kPackCap;
  xk.bd[(int64_t)(pd.bd_row + k) * xk.bd_ld + v] = pack_pair(x, x);
}

template <typename T>
cudaError_t launch_bdy_expand_tma(const PartDesc *parts, int nparts, int max_s, int nbB, const int64_t *grow,
                                  const int32_t *st2ed, const T *dB, int64_t ldB, const T *F, int64_t ldf,
                                  int nparts_f, T *D, int64_t ldD, T *FB, int64_t ldFB, int *status,
                                  cudaStream_t stream, int64_t *launches, const Expand16 *xk) {
  using TC = typename FloydCfg<T, kFloydTile>::TC;
  if (nparts <= 0 || max_s <= 0 || nbB <= 0) return cudaSuccess;
  if (nparts > 65535 || ceil_div(nbB, TC::BM) > 65535) return cudaErrorInvalidConfiguration;
  CUtensorMap mapA, mapB, unused;
  cudaError_t e = make_tmap_3d(&mapA, dB, Dist<T>::kDtype == FAP_DTYPE_F32, ldB, nbB, 1, TC::BK, TC::BM);
  if (e == cudaSuccess) e = make_arena_tmaps<T>(F, ldf, nparts_f, &unused, &mapB);
  if (e != cudaSuccess) return e;
  const dim3 grid((unsigned)ceil_div(max_s, TC::BN), (unsigned)ceil_div(nbB, TC::BM), nparts);
  Expand16 none{};
  if constexpr (std::is_same<T, int32_t>::value) {
    if (xk != nullptr) {
      if (xk->nrt < (int)ceil_div(nbB, TC::BM)) return cudaErrorInvalidValue;
      expand16_rows_kernel<<<dim3((unsigned)ceil_div(nbB, 128), (unsigned)nparts), 256, 0, stream>>>(
          parts, nbB, dB, ldB, *xk);
      expand16_maxb_kernel<<<(unsigned)nparts, 256, 0, stream>>>(parts, F, *xk);
      *launches += 2;
      if (xk->ap != nullptr) {
        // operands packed beforehand, then tiles without conversion
        if (xk->bd == nullptr || xk->ap_ld % 4 != 0 || xk->bd_ld % 4 != 0 || xk->rows <= 0 || xk->max_b <= 0 ||
            xk->ap_ld < (int)ceil_div(nbB, 2) || xk->bd_ld < max_s)
          return cudaErrorInvalidValue;
        CUtensorMap mapAP, mapBD;
        e = make_tmap_3d_dt(&mapAP, xk->ap, CU_TENSOR_MAP_DATA_TYPE_UINT32, 4, xk->ap_ld, xk->rows, 1, TC::BM / 2,
                            TC::BK);
        if (e == cudaSuccess)
          e = make_tmap_3d_dt(&mapBD, xk->bd, CU_TENSOR_MAP_DATA_TYPE_UINT32, 4, xk->bd_ld, xk->rows, 1, TC::BN,
                              TC::BK);
        if (e != cudaSuccess) return e;
        expand16_pack_a_kernel<<<dim3((unsigned)ceil_div(nbB, 128), (unsigned)ceil_div(xk->max_b, 32),
                                      (unsigned)nparts),
                                 256, 0, stream>>>(parts, nbB, dB, ldB, *xk);
        expand16_pack_b_kernel<<<dim3((unsigned)ceil_div(xk->bd_ld, 256), (unsigned)xk->max_b, (unsigned)nparts),
                                 256, 0, stream>>>(parts, F, *xk);
        *launches += 2;
        const size_t smem = TC::SMEM_BYTES;
        auto kern = bdy_expand_tma_kernel<T, 2>;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, TC::THREADS, smem, stream>>>(parts, nbB, grow, st2ed, D, ldD, FB, ldFB, mapA, mapB, status,
                                                  *xk, mapAP, mapBD);
        *launches += 1;
        return cudaGetLastError();
      }
      const size_t smem = Pack16Cfg<TC>::SMEM_BYTES;
      auto kern = bdy_expand_tma_kernel<T, 1>;
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      kern<<<grid, TC::THREADS, smem, stream>>>(parts, nbB, grow, st2ed, D, ldD, FB, ldFB, mapA, mapB, status,
                                                *xk, mapA, mapB);
      *launches += 1;
      return cudaGetLastError();
    }
  }
  const size_t smem = TC::SMEM_BYTES;
  auto kern = bdy_expand_tma_kernel<T, 0>;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<grid, TC::THREADS, smem, stream>>>(parts, nbB, grow, st2ed, D, ldD, FB, ldFB, mapA, mapB, status, none,
                                            mapA, mapB);
  *launches += 1;
  return cudaGetLastError();
}

// Expansion as one min-plus tile per CTA: rows m0.. of dB (boundary indices)
// restricted to part q's boundary columns, times q's local rows F_q[0..b_q)
// over its columns n0..; the register-tiled engine streams K = b_q through
// shared memory.  Stores go to the columns' original ids (st2ed).
template <typename T>
__global__ void __launch_bounds__(MPCfg<T>::THREADS, 2)
    bdy_expand_tiled_kernel(const PartDesc *__restrict__ parts, int nbB, const int64_t *__restrict__ grow,
                            const int32_t *__restrict__ st2ed, const T *__restrict__ dB, int64_t ldB,
                            const T *__restrict__ F, T *D, int64_t ldD, T *FB, int64_t ldFB) {
  using C = MPCfg<T>;
  __shared__ __align__(16) T smem[C::SMEM_ELEMS];
  const PartDesc pd = parts[blockIdx.z];
  const int n0 = blockIdx.y * C::BN;
  if (n0 >= pd.s) return;
  const int m0 = blockIdx.x * C::BM;
  T acc[C::TM][C::TN];
  acc_fill<T, C>(acc, Dist<T>::inf());
  minplus_tile<T, C, true, true>(dB + pd.bd_row, ldB, F + pd.f_off, pd.ldf, m0, n0, nbB, pd.s, pd.b, acc,
                                 smem);
  const int tid = threadIdx.x, ty = tid / C::TX, tx = tid % C::TX;
  int col[C::TN];
#pragma unroll
  for (int gj = 0; gj < C::GN; gj++)
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int j = n0 + tile_col<C>(tx, gj, q);
      col[4 * gj + q] = j < pd.s ? __ldg(st2ed + pd.start + j) : -1;
    }
#pragma unroll
  for (int gi = 0; gi < C::GM; gi++)
#pragma unroll
    for (int l = 0; l < 4; l++) {
      const int r = m0 + tile_row<C>(ty, gi, l);
      if (r >= nbB) continue;
      T *dst = D + __ldg(grow + r) * ldD;
      const bool own = r >= pd.bd_row && r < pd.bd_row + pd.b;
      T *fb = FB + (int64_t)r * ldFB + n0;
#pragma unroll
      for (int gj = 0; gj < C::GN; gj++)
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int c = col[4 * gj + q];
          if (c < 0) continue;
          const T v = acc[4 * gi + l][4 * gj + q];
          __stcs(dst + c, v);
          if (own) fb[tile_col<C>(tx, gj, q)] = v;
        }
    }
}

template <typename T>
cudaError_t launch_bdy_expand_tiled(const PartDesc *parts, int nparts, int max_s, int nbB, const int64_t *grow,
                                    const int32_t *st2ed, const T *dB, int64_t ldB, const T *F, T *D,
                                    int64_t ldD, T *FB, int64_t ldFB, cudaStream_t stream, int64_t *launches) {
  using C = MPCfg<T>;
  if (nparts <= 0 || max_s <= 0 || nbB <= 0) return cudaSuccess;
  if (nparts > 65535 || ceil_div(max_s, C::BN) > 65535) return cudaErrorInvalidConfiguration;
  bdy_expand_tiled_kernel<T><<<dim3((unsigned)ceil_div(nbB, C::BM), (unsigned)ceil_div(max_s, C::BN), nparts),
                               C::THREADS, 0, stream>>>(parts, nbB, grow, st2ed, dB, ldB, F, D, ldD, FB, ldFB);
  *launches += 1;
  return cudaGetLastError();
}

// Local closure -> exact closure of each part, in place: for inner rows i,
//   F[i][j] = min(F[i][j], min_{k<b} F[i][k] + FB[k][j])
// (a path from i to j either stays in the part or leaves it through a
// boundary vertex k first, after which FB holds the exact rest).  The
// boundary rows of F take FB's values.  Two launches, so that every row
// reads its local values F[i][0..b) before they change:
//   1. columns j >= b of the inner rows, one min-plus tile (A = F[i][k],
//      B = FB[k][j]) per CTA, grid (column tiles, row tiles, parts);
//   2. columns j < b of the inner rows (each CTA stages its rows' local
//      values first) and the boundary rows, grid (parts, row chunks of 32).
constexpr int kFixRows = 32;

constexpr int kFixStage = 4096;  // staged values per CTA: rows x boundary count

template <typename T>
__global__ void __launch_bounds__(MPCfg<T>::THREADS, 2)
    local_fixup_tile_kernel(const PartDesc *__restrict__ parts, T *F, const T *__restrict__ FB, int64_t ldFB) {
  using C = MPCfg<T>;
  __shared__ __align__(16) T smem[C::SMEM_ELEMS];
  const PartDesc pd = parts[blockIdx.z];
  const int n0 = blockIdx.x * C::BN, m0 = blockIdx.y * C::BM;
  const int M = pd.s - pd.b;
  if (n0 + C::BN <= pd.b || n0 >= pd.s || m0 >= M || pd.b == 0) return;
  T *Fi = F + pd.f_off + (int64_t)pd.b * pd.ldf;  // inner rows
  T acc[C::TM][C::TN];
  acc_load<T, C, false>(acc, Fi, pd.ldf, m0, n0, M, pd.s);
  minplus_tile<T, C, true, true>(Fi, pd.ldf, FB + (int64_t)pd.bd_row * ldFB, ldFB, m0, n0, M, pd.s, pd.b, acc,
                                 smem);
  const int tid = threadIdx.x, ty = tid / C::TX, tx = tid % C::TX;
#pragma unroll
  for (int gi = 0; gi < C::GM; gi++)
#pragma unroll
    for (int l = 0; l < 4; l++) {
      const int r = m0 + tile_row<C>(ty, gi, l);
      if (r >= M) continue;
#pragma unroll
      for (int gj = 0; gj < C::GN; gj++)
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int c = n0 + tile_col<C>(tx, gj, q);
          if (c >= pd.b && c < pd.s) Fi[(int64_t)r * pd.ldf + c] = acc[4 * gi + l][4 * gj + q];
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(256)
    local_fixup_kernel(const PartDesc *__restrict__ parts, T *F, const T *__restrict__ FB, int64_t ldFB) {
  // the rows' local distances to their part's boundary vertices, before the update
  __shared__ T a_s[kFixStage];
  const PartDesc pd = parts[blockIdx.x];
  const int i0 = max(blockIdx.y * kFixRows, 0);
  if (i0 >= pd.s) return;
  const T *FBp = FB + (int64_t)pd.bd_row * ldFB;
  const int i1 = min(i0 + kFixRows, pd.s);
  const bool staged = (int64_t)kFixRows * pd.b <= kFixStage;
  if (staged) {
    for (int t = threadIdx.x; t < (i1 - i0) * pd.b; t += blockDim.x) {
      const int r = t / pd.b, k = t % pd.b;
      a_s[t] = F[pd.f_off + (int64_t)(i0 + r) * pd.ldf + k];
    }
  }
  __syncthreads();
  const bool row_staged = !staged && pd.b <= kFixStage;  // one row at a time
  for (int i = i0; i < i1; i++) {
    T *Fi = F + pd.f_off + (int64_t)i * pd.ldf;
    if (i < pd.b) {
      for (int j = threadIdx.x; j < pd.s; j += blockDim.x) Fi[j] = FBp[(int64_t)i * ldFB + j];
      continue;
    }
    // columns j < b only (the tile launch did the rest)
    if (row_staged) {
      __syncthreads();
      for (int k = threadIdx.x; k < pd.b; k += blockDim.x) a_s[k] = Fi[k];
      __syncthreads();
    }
    // (more than kFixStage boundary vertices: the row reads values that other
    // threads may already have lowered to the exact ones, which gives the
    // same minimum in int32)
    const T *ai = staged ? a_s + (int64_t)(i - i0) * pd.b : row_staged ? a_s : Fi;
    for (int j = threadIdx.x; j < pd.b; j += blockDim.x) {
      T acc = Fi[j];
      for (int k = 0; k < pd.b; k++) acc = Dist<T>::relax(ai[k], FBp[(int64_t)k * ldFB + j], acc);
      Fi[j] = acc;
    }
  }
}

template <typename T>
cudaError_t launch_local_fixup(const PartDesc *parts, int nparts, int max_s, T *F, const T *FB, int64_t ldFB,
                               cudaStream_t stream, int64_t *launches) {
  using C = MPCfg<T>;
  if (nparts <= 0 || max_s <= 0) return cudaSuccess;
  if (nparts > 65535) return cudaErrorInvalidConfiguration;
  local_fixup_tile_kernel<T><<<dim3((unsigned)ceil_div(max_s, C::BN), (unsigned)ceil_div(max_s, C::BM), nparts),
                               C::THREADS, 0, stream>>>(parts, F, FB, ldFB);
  local_fixup_kernel<T><<<dim3(nparts, (unsigned)ceil_div(max_s, kFixRows)), 256, 0, stream>>>(parts, F, FB,
                                                                                              ldFB);
  *launches += 2;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Resident cache kernels
// ---------------------------------------------------------------------------
template <typename T>
__global__ void bdy_copy_kernel(const PartDesc *__restrict__ parts, const T *__restrict__ Bd, T *D,
                                int64_t ldD) {
  const PartDesc pd = parts[blockIdx.y];
  const int i = blockIdx.x;
  if (i >= pd.b) return;
  using V = typename Vec4<T>::type;  // ldD is a multiple of 128: rows are 16-byte aligned
  const V *src = reinterpret_cast<const V *>(Bd + ((int64_t)pd.bd_row + i) * ldD);
  V *dst = reinterpret_cast<V *>(D + (pd.row_base + i) * ldD);
  for (int64_t j = threadIdx.x; j < ldD / 4; j += blockDim.x) dst[j] = __ldg(src + j);
}

template <typename T>
cudaError_t launch_bdy_copy(const PartDesc *parts, int nparts, int max_b, const T *Bd, T *D,
                            int64_t ldD, cudaStream_t stream, int64_t *launches) {
  if (nparts <= 0 || max_b <= 0) return cudaSuccess;
  bdy_copy_kernel<T><<<dim3(max_b, nparts), 256, 0, stream>>>(parts, Bd, D, ldD);
  *launches += 1;
  return cudaGetLastError();
}

template <typename T>
__global__ void row_gather_kernel(const T *__restrict__ src, int64_t ld_src,
                                  const int64_t *__restrict__ idx, int n, T *__restrict__ out,
                                  int64_t ld_out, const int64_t *__restrict__ out_rows) {
  const int64_t r = blockIdx.y;
  const T *s = src + idx[r] * ld_src;
  T *o = out + out_rows[r] * ld_out;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x)
    o[j] = __ldg(s + j);
}

template <typename T>
cudaError_t launch_row_gather(const T *src, int64_t ld_src, const int64_t *idx, int64_t rows, int n,
                              T *out, int64_t ld_out, const int64_t *out_rows, cudaStream_t stream,
                              int64_t *launches) {
  if (rows <= 0 || n <= 0) return cudaSuccess;
  const int bx = (int)std::min<int64_t>(ceil_div(n, 256), 16);
  row_gather_kernel<T><<<dim3(bx, (unsigned)rows), 256, 0, stream>>>(src, ld_src, idx, n, out, ld_out,
                                                                     out_rows);
  *launches += 1;
  return cudaGetLastError();
}

// grid (ngroups, column chunks of kRowsCols): consecutive CTAs take the
// groups of one column chunk, so a part's boundary-row chunk is read from
// DRAM once and from L2 by its other groups.  Each thread owns 4 columns
// (stride 256: coalesced loads of the boundary rows), each group up to
// kRowsGroup rows; the A values are staged in shared memory in chunks of
// kRowsKC boundary columns.
constexpr int kRowsThreads = 256;
constexpr int kRowsCols = 4 * kRowsThreads;
constexpr int kRowsKC = 256;

// Body for groups of at most RG rows (RG a compile-time bound, so that the
// accumulators of absent rows cost nothing).
template <typename T, int RG>
__device__ __forceinline__ void minplus_rows_body(const RowGroup &g, const PartDesc &pd,
                                                  const int64_t *__restrict__ out_row, int n,
                                                  const T *__restrict__ F, const T *__restrict__ Bd,
                                                  int64_t ldD, const int32_t *__restrict__ graph_id,
                                                  const int32_t *__restrict__ ed2st, T *__restrict__ out,
                                                  int64_t ld_out, T (&As)[kRowsGroup][kRowsKC],
                                                  const int32_t *rloc) {
  const int c0 = blockIdx.y * kRowsCols + threadIdx.x;
  const T inf = Dist<T>::inf();
  T acc[RG][4];
#pragma unroll
  for (int r = 0; r < RG; r++)
#pragma unroll
    for (int q = 0; q < 4; q++) acc[r][q] = inf;
  const T *Fp = F + pd.f_off;
  const T *Bp = Bd + (int64_t)pd.bd_row * ldD;
  for (int k0 = 0; k0 < pd.b; k0 += kRowsKC) {
    const int kc = min(kRowsKC, pd.b - k0);
    __syncthreads();
    for (int t = threadIdx.x; t < RG * kRowsKC; t += blockDim.x) {
      const int r = t / kRowsKC, k = t % kRowsKC;
      As[r][k] = (r < g.count && k < kc) ? __ldg(Fp + (int64_t)rloc[r] * pd.ldf + k0 + k) : inf;
    }
    __syncthreads();
#pragma unroll 4
    for (int k = 0; k < kc; k++) {
      const T *Bk = Bp + (int64_t)(k0 + k) * ldD;
      T v[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int c = c0 + q * kRowsThreads;
        v[q] = c < n ? __ldg(Bk + c) : inf;
      }
#pragma unroll
      for (int r = 0; r < RG; r++) {
        const T a = As[r][k];
#pragma unroll
        for (int q = 0; q < 4; q++) acc[r][q] = Dist<T>::relax(a, v[q], acc[r][q]);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int c = c0 + q * kRowsThreads;
    if (c >= n) continue;
    const int o = (__ldg(graph_id + c) == pd.part) ? __ldg(ed2st + c) - pd.start : -1;
#pragma unroll
    for (int r = 0; r < RG; r++) {
      if (r >= g.count) break;
      const T val = o >= 0 ? __ldg(Fp + (int64_t)rloc[r] * pd.ldf + o) : acc[r][q];
      out[out_row[g.first + r] * ld_out + c] = val;
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kRowsThreads, 2)
    minplus_rows_kernel(const PartDesc *__restrict__ parts, const RowGroup *__restrict__ groups,
                        const int32_t *__restrict__ loc, const int64_t *__restrict__ out_row, int n,
                        const T *__restrict__ F, const T *__restrict__ Bd, int64_t ldD,
                        const int32_t *__restrict__ graph_id, const int32_t *__restrict__ ed2st,
                        T *__restrict__ out, int64_t ld_out) {
  __shared__ T As[kRowsGroup][kRowsKC];
  __shared__ int32_t rloc[kRowsGroup];
  const RowGroup g = groups[blockIdx.x];
  const PartDesc pd = parts[g.pidx];
  if (threadIdx.x < kRowsGroup) rloc[threadIdx.x] = threadIdx.x < g.count ? loc[g.first + threadIdx.x] : 0;
  __syncthreads();
  if (g.count <= 1)
    minplus_rows_body<T, 1>(g, pd, out_row, n, F, Bd, ldD, graph_id, ed2st, out, ld_out, As, rloc);
  else if (g.count <= 4)
    minplus_rows_body<T, 4>(g, pd, out_row, n, F, Bd, ldD, graph_id, ed2st, out, ld_out, As, rloc);
  else
    minplus_rows_body<T, kRowsGroup>(g, pd, out_row, n, F, Bd, ldD, graph_id, ed2st, out, ld_out, As, rloc);
}

template <typename T>
cudaError_t launch_minplus_rows(const PartDesc *parts, const RowGroup *groups, int ngroups,
                                const int32_t *loc, const int64_t *out_row, int max_b, int n,
                                const T *F, const T *Bd, int64_t ldD, const int32_t *graph_id,
                                const int32_t *ed2st, T *out, int64_t ld_out, cudaStream_t stream,
                                int64_t *launches) {
  (void)max_b;
  if (ngroups <= 0 || n <= 0) return cudaSuccess;
  dim3 grid((unsigned)ngroups, (unsigned)ceil_div(n, kRowsCols));
  minplus_rows_kernel<T><<<grid, kRowsThreads, 0, stream>>>(parts, groups, loc, out_row, n, F, Bd,
                                                            ldD, graph_id, ed2st, out, ld_out);
  *launches += 1;
  return cudaGetLastError();
}

// Generic C = min(INF, A (x) B), any sizes and alignments.
template <typename T, bool VEC_B>
__global__ void __launch_bounds__(MPCfg<T>::THREADS)
    minplus_generic_kernel(int M, int N, int K, const T *__restrict__ A, int64_t lda,
                           const T *__restrict__ B, int64_t ldb, T *__restrict__ Cp, int64_t ldc) {
  using C = MPCfg<T>;
  extern __shared__ __align__(16) unsigned char mg_smem_raw[];
  T *smem = reinterpret_cast<T *>(mg_smem_raw);
  const int m0 = blockIdx.y * C::BM, n0 = blockIdx.x * C::BN;
  T acc[C::TM][C::TN];
  acc_fill<T, C>(acc, Dist<T>::inf());
  minplus_tile<T, C, VEC_B, true>(A, lda, B, ldb, m0, n0, M, N, K, acc, smem);
  acc_store<T, C, false>(acc, Cp, ldc, m0, n0, M, N);
}

template <typename T>
cudaError_t launch_minplus_generic(int M, int N, int K, const T *A, int64_t lda, const T *B,
                                   int64_t ldb, T *C, int64_t ldc, cudaStream_t stream,
                                   int64_t *launches) {
  if (M <= 0 || N <= 0) return cudaSuccess;
  using Cf = MPCfg<T>;
  const size_t smem = Cf::SMEM_ELEMS * sizeof(T);
  dim3 grid((unsigned)ceil_div(N, Cf::BN), (unsigned)ceil_div(M, Cf::BM));
  // Vector B loads need 16-byte rows and whole 4-vectors inside each row.
  const bool vec = (ldb % 4 == 0) && (N % 4 == 0) && ((uintptr_t)B % 16 == 0);
  if (vec)
    minplus_generic_kernel<T, true><<<grid, Cf::THREADS, smem, stream>>>(M, N, K, A, lda, B, ldb, C, ldc);
  else
    minplus_generic_kernel<T, false><<<grid, Cf::THREADS, smem, stream>>>(M, N, K, A, lda, B, ldb, C, ldc);
  *launches += 1;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Utilities
// ---------------------------------------------------------------------------
template <typename T>
__global__ void fill_kernel(T *p, int64_t rows, int64_t cols, int64_t ld, T v) {
  const int64_t total = rows * cols;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t / cols, c = t % cols;
    p[r * ld + c] = v;
  }
}

template <typename T>
cudaError_t launch_fill(T *p, int64_t rows, int64_t cols, int64_t ld, T v, cudaStream_t stream,
                        int64_t *launches) {
  if (rows <= 0 || cols <= 0) return cudaSuccess;
  const int64_t total = rows * cols;
  const int blocks = (int)std::min<int64_t>(ceil_div(total, 256), device_sm_count() * 32);
  fill_kernel<T><<<blocks, 256, 0, stream>>>(p, rows, cols, ld, v);
  *launches += 1;
  return cudaGetLastError();
}

// One CTA per row: sum over j of (uint32)D[r][j] * (2j + 1), mod 2^64.  Float
// input holds exact integers (int32 distances converted for output).
__device__ __forceinline__ uint32_t checksum_word(int32_t x) { return (uint32_t)x; }
__device__ __forceinline__ uint32_t checksum_word(float x) { return (uint32_t)(int32_t)x; }

template <typename T>
__global__ void row_checksum_kernel(const T *__restrict__ D, int64_t n, int64_t ld,
                                    uint64_t *__restrict__ out) {
  const int64_t r = blockIdx.x;
  const T *row = D + r * ld;
  uint64_t acc = 0;
  for (int64_t j = threadIdx.x; j < n; j += blockDim.x)
    acc += (uint64_t)checksum_word(__ldg(row + j)) * (uint64_t)(2 * j + 1);
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  __shared__ uint64_t part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    uint64_t v = (threadIdx.x < (blockDim.x >> 5)) ? part[threadIdx.x] : 0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) out[r] = v;
  }
}

cudaError_t launch_row_checksums(const int32_t *D, int64_t rows, int64_t n, int64_t ld,
                                 uint64_t *out, cudaStream_t stream, int64_t *launches) {
  if (rows <= 0) return cudaSuccess;
  row_checksum_kernel<int32_t><<<(unsigned)rows, 256, 0, stream>>>(D, n, ld, out);
  *launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_row_checksums(const float *D, int64_t rows, int64_t n, int64_t ld,
                                 uint64_t *out, cudaStream_t stream, int64_t *launches) {
  if (rows <= 0) return cudaSuccess;
  row_checksum_kernel<float><<<(unsigned)rows, 256, 0, stream>>>(D, n, ld, out);
  *launches += 1;
  return cudaGetLastError();
}

__global__ void i32_to_f32_kernel(const int32_t *__restrict__ src, int64_t rows, int64_t n,
                                  int64_t ld, float *__restrict__ dst) {
  const int64_t total = rows * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t / n, c = t % n;
    dst[t] = (float)src[r * ld + c];
  }
}

cudaError_t launch_i32_to_f32(const int32_t *src, int64_t rows, int64_t n, int64_t ld, float *dst,
                              cudaStream_t stream, int64_t *launches) {
  if (rows <= 0 || n <= 0) return cudaSuccess;
  const int blocks = (int)std::min<int64_t>(ceil_div(rows * n, 256), device_sm_count() * 32);
  i32_to_f32_kernel<<<blocks, 256, 0, stream>>>(src, rows, n, ld, dst);
  *launches += 1;
  return cudaGetLastError();
}

// Relaxation throughput: 64 independent-ish accumulators per thread, every
// relaxation's add input changes each iteration so nothing can be hoisted.
template <typename T>
__global__ void __launch_bounds__(256) relax_peak_kernel(T *sink, int iters, T seed) {
  T acc[8][8], b[8];
#pragma unroll
  for (int j = 0; j < 8; j++) b[j] = seed + T((threadIdx.x + j) & 7);
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) acc[i][j] = seed * T(i + 1) + T(j + threadIdx.x % 5);
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
      for (int j = 0; j < 8; j++) acc[i][j] = Dist<T>::relax(acc[i][j], b[j], acc[(i + 1) & 7][j]);
  }
  T s = T(0);
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) s = Dist<T>::min(s, acc[i][j]);
  if (s == T(-12345)) sink[0] = s;  // never true; keeps the loop live
  if (threadIdx.x == 0 && blockIdx.x == 0) sink[1] = s;
}

template <typename T>
cudaError_t launch_relax_peak(T *sink, int blocks, int iters, cudaStream_t stream,
                              double *relax_count) {
  relax_peak_kernel<T><<<blocks, 256, 0, stream>>>(sink, iters, T(3));
  *relax_count = (double)blocks * 256.0 * (double)iters * 64.0;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Explicit instantiations
// ---------------------------------------------------------------------------
#define FAPB_INSTANTIATE(T)                                                                       \
  template cudaError_t launch_sssp<T>(const int32_t *, const int32_t *, const T *, int,           \
                                      const int32_t *, const int64_t *, int, T *, int64_t,        \
                                      int64_t, const int32_t *, T *, T, int, int, int64_t, int *, \
                                      cudaStream_t, int64_t *);                                   \
  template cudaError_t launch_msbf<T>(const MsbfItem *, int, const int32_t *, const int32_t *,     \
                                      const T *, int, const int32_t *, const int32_t *,            \
                                      const int64_t *, int, T *, int64_t, int64_t, int, T *,       \
                                      uint32_t *, int *, int *, int64_t, int *, cudaStream_t,      \
                                      int64_t *); \
  template cudaError_t launch_gather<T>(const PartDesc *, int, int, const int32_t *,              \
                                        const int32_t *, const T *, const int32_t *,              \
                                        const int32_t *, const int32_t *, const T *, int64_t, T *, \
                                        cudaStream_t, int64_t *);                                 \
  template cudaError_t launch_floyd_parts<T>(const PartDesc *, int, T *, int64_t, T *, int64_t,   \
                                             const int32_t *, int *, cudaStream_t, int64_t *);    \
  template cudaError_t launch_floyd_matrix<T>(T *, int64_t, int, int *, cudaStream_t, int64_t *, int); \
  template cudaError_t launch_floyd_parts_multi<T>(const PartDesc *, int, int, T *, int64_t, int *, \
                                                   cudaStream_t, int64_t *);                      \
  template cudaError_t launch_floyd_queue<T>(const PartDesc *, int, T *, int64_t, const FloydQueue &, \
                                             const MPWork *, int, T *, int64_t, int64_t,          \
                                             const int32_t *, const int32_t *, const int32_t *,    \
                                             int *, cudaStream_t, int64_t *, const Pack16 *);     \
  template cudaError_t launch_bdy_scatter<T>(const PartDesc *, int, const T *, T *, int64_t,      \
                                             const int32_t *, int, int, cudaStream_t, int64_t *); \
  template cudaError_t launch_minplus_parts<T>(const PartDesc *, int, const MPWork *, int, int,   \
                                               const T *, int64_t, T *, int64_t, int64_t,         \
                                               const int32_t *, const int32_t *, int *,           \
                                               cudaStream_t, int64_t *, const Pack16 *);          \
  template cudaError_t launch_minplus_thin<T>(const PartDesc *, const int32_t *, int, int, int,   \
                                              const T *, T *, int64_t, const int32_t *,           \
                                              const int32_t *, cudaStream_t, int64_t *);          \
  template cudaError_t launch_minplus_generic<T>(int, int, int, const T *, int64_t, const T *,    \
                                                 int64_t, T *, int64_t, cudaStream_t, int64_t *); \
  template cudaError_t launch_fill<T>(T *, int64_t, int64_t, int64_t, T, cudaStream_t, int64_t *); \
  template cudaError_t launch_bgraph<T>(const PartDesc *, int, int, const T *, T *, int64_t,       \
                                        const int32_t *, const int32_t *, const T *, int,          \
                                        const int32_t *, const int32_t *, const BPart *,           \
                                        cudaStream_t, int64_t *);                                  \
  template cudaError_t launch_bdy_expand<T>(const int64_t *, int, const BPart *, const int32_t *,  \
                                            const int32_t *, int, const T *, int64_t, int,         \
                                            const T *, T *, int64_t, T *, int64_t, T *, int,       \
                                            cudaStream_t, int64_t *);                              \
  template cudaError_t launch_local_fixup<T>(const PartDesc *, int, int, T *, const T *, int64_t,  \
                                             cudaStream_t, int64_t *);                             \
  template cudaError_t launch_bgraph_bf<T>(const PartDesc *, int, int, const T *, const int32_t *,  \
                                           const int32_t *, const T *, const int32_t *,              \
                                           const int32_t *, const int32_t *, const int32_t *, int,   \
                                           int, int, T *, int64_t, T *, int *, int *, int *, int *,  \
                                           int *, int *, int64_t, int *, cudaStream_t, int64_t *);   \
  template cudaError_t launch_bdy_expand_tma<T>(const PartDesc *, int, int, int, const int64_t *,  \
                                                const int32_t *, const T *, int64_t, const T *,    \
                                                int64_t, int, T *, int64_t, T *, int64_t, int *,   \
                                                cudaStream_t, int64_t *, const Expand16 *);                          \
  template cudaError_t launch_bdy_expand_tiled<T>(const PartDesc *, int, int, int, const int64_t *, \
                                                  const int32_t *, const T *, int64_t, const T *,  \
                                                  T *, int64_t, T *, int64_t, cudaStream_t,        \
                                                  int64_t *);                                      \
  template cudaError_t launch_pred<T>(const PartDesc *, int, int, const T *, int32_t *, int64_t,  \
                                      int, const int32_t *, const int32_t *, const T *,            \
                                      const int32_t *, const T *, cudaStream_t, int64_t *);        \
  template cudaError_t launch_bdy_copy<T>(const PartDesc *, int, int, const T *, T *, int64_t,    \
                                          cudaStream_t, int64_t *);                               \
  template cudaError_t launch_row_gather<T>(const T *, int64_t, const int64_t *, int64_t, int, T *, \
                                            int64_t, const int64_t *, cudaStream_t, int64_t *);   \
  template cudaError_t launch_minplus_rows<T>(const PartDesc *, const RowGroup *, int,            \
                                              const int32_t *, const int64_t *, int, int,         \
                                              const T *, const T *, int64_t, const int32_t *,     \
                                              const int32_t *, T *, int64_t, cudaStream_t,        \
                                              int64_t *);                                         \
  template cudaError_t launch_relax_peak<T>(T *, int, int, cudaStream_t, double *);

FAPB_INSTANTIATE(int32_t)
FAPB_INSTANTIATE(float)

}  // namespace fapb
