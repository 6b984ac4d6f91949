// Stage 1: batched multi-source shortest paths from boundary vertices.
//
// Replaces handle_boundry_Nvidia_GPU / multi_source_Nvidia_sssp
// (fap/kernel/cuda/batch_sssp.cu:222-296), which ran one source at a time
// with a host round trip per Bellman-Ford iteration, and the CPU
// batched_sssp_path (fap/kernel/batch_sssp.h:232-252).
//
// Design: one CTA per source (grid-stride over sources), every source of
// every requested part in one launch.
//   - Work space: the CSR may be relabelled into partition order (sorted
//     positions), so that a frontier -- geometrically compact on road-like
//     graphs, and METIS parts are compact -- touches nearby addresses.  The
//     CTA then works on a scratch row and finally writes the output row in
//     original column order (out[v] = dist[ed2st[v]]).
//   - Frontier: a work queue in shared memory, deduplicated by one bitmap of
//     n bits ("queued").  A round processes the queue and pushes improved
//     vertices to the other queue, so its cost follows the frontier, not n.
//     When a queue overflows, the vertices stay marked in the bitmap and the
//     next round collects them with a block-wide scan of the bitmap instead.
//   - Expansion: a thread relaxes a light vertex's edges with all loads and
//     atomics of a 4-edge group in flight at once; vertices with more than
//     kHeavyDeg edges are expanded by a whole warp (lane-strided, coalesced
//     column/weight reads).
//   - Order: near/far (delta stepping).  A frontier vertex whose distance is
//     not below the threshold stays in the bitmap; when no near vertex is
//     left, the threshold moves to (smallest far distance + delta).
//     delta = INF gives plain frontier Bellman-Ford.
// Convergence needs no host round trip and no inter-CTA synchronisation.
// The number of rounds is bounded; a CTA that hits the bound records an
// error status and stops (it never spins).
#pragma once

#include "fap_common.cuh"

namespace fapb {

constexpr int kSsspThreads = 256;
constexpr int kSsspQueue = 2048;  // entries per frontier queue (two queues)
constexpr int kHeavyDeg = 32;     // vertices above this degree go to a warp
constexpr int kHeavyList = 256;

// Shared-memory bytes a CTA needs for n vertices (dynamic part).
inline size_t sssp_smem_bytes(int n) {
  return (size_t)ceil_div(n, 32) * sizeof(uint32_t) + (2 * kSsspQueue + kHeavyList) * sizeof(int32_t);
}

template <typename T>
__device__ __forceinline__ int32_t order_bits(T v);
template <>
__device__ __forceinline__ int32_t order_bits<int32_t>(int32_t v) { return v; }
template <>
__device__ __forceinline__ int32_t order_bits<float>(float v) { return __float_as_int(v); }
template <typename T>
__device__ __forceinline__ T from_order_bits(int32_t b);
template <>
__device__ __forceinline__ int32_t from_order_bits<int32_t>(int32_t b) { return b; }
template <>
__device__ __forceinline__ float from_order_bits<float>(int32_t b) { return __int_as_float(b); }

template <typename T>
__device__ __forceinline__ T ld_relaxed(const T *p) {
  return *reinterpret_cast<const volatile T *>(p);
}

// Block-wide exclusive scan of one int per thread (blockDim.x == kSsspThreads).
__device__ __forceinline__ int block_excl_scan(int x, int *warp_tmp, int *total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) warp_tmp[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    int s = (lane < kSsspThreads / 32) ? warp_tmp[lane] : 0;
    int si = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, si, o);
      if (lane >= o) si += y;
    }
    if (lane < kSsspThreads / 32) warp_tmp[lane] = si - s;
    if (lane == kSsspThreads / 32 - 1) *total = si;
  }
  __syncthreads();
  return warp_tmp[wid] + inc - x;
}

// Frontier push: marks v in the queued bitmap and, if it was not marked,
// appends it to the next queue (or flags an overflow, leaving it marked).
__device__ __forceinline__ void frontier_push(int v, uint32_t *queued, int32_t *nextq, int *ncount,
                                              int *novf) {
  const uint32_t bit = 1u << (v & 31);
  if (!(atomicOr(queued + (v >> 5), bit) & bit)) {
    const int p = atomicAdd(ncount, 1);
    if (p < kSsspQueue) nextq[p] = v;
    else *novf = 1;
  }
}

// Relaxes edges [e0, e1) (every stride-th) of a vertex at distance du with
// 4 loads and 4 atomics in flight; pushes every improved neighbour.  Returns
// whether anything improved.
template <typename T>
__device__ __forceinline__ bool relax_edges(const int32_t *__restrict__ col, const T *__restrict__ w,
                                            int e0, int e1, int stride, T du, T *dist,
                                            uint32_t *queued, int32_t *nextq, int *ncount, int *novf) {
  bool any = false;
  for (int e = e0; e < e1; e += 4 * stride) {
    int v[4];
    T nd[4], cur[4], old[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int ek = e + k * stride;
      v[k] = ek < e1 ? __ldg(col + ek) : -1;
      nd[k] = ek < e1 ? du + __ldg(w + ek) : du;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) cur[k] = v[k] >= 0 ? ld_relaxed(dist + v[k]) : du;
#pragma unroll
    for (int k = 0; k < 4; k++)
      old[k] = (v[k] >= 0 && nd[k] < cur[k]) ? Dist<T>::atomic_min(dist + v[k], nd[k]) : nd[k];
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (nd[k] < old[k]) {
        frontier_push(v[k], queued, nextq, ncount, novf);
        any = true;
      }
  }
  return any;
}

// sources / row_offset / col are in work space.  When perm_out is not null
// the work space is a relabelling: dist lives in scratch (one row of n per
// CTA) and out[v] = dist[perm_out[v]] is written at the end; otherwise dist is
// the output row itself.
template <typename T>
__global__ void __launch_bounds__(kSsspThreads, 4)
    sssp_frontier_kernel(const int32_t *__restrict__ row_offset, const int32_t *__restrict__ col,
                         const T *__restrict__ w, int n, const int32_t *__restrict__ sources,
                         const int64_t *__restrict__ out_rows, int num_sources, T *out, int64_t ld,
                         int64_t init_cols, const int32_t *__restrict__ perm_out, T *scratch,
                         T delta, int64_t max_rounds, int *status) {
  extern __shared__ uint32_t queued[];
  __shared__ int32_t s_minfar[3];
  __shared__ int s_warp[kSsspThreads / 32];
  __shared__ int s_total, s_nheavy;
  __shared__ int s_cnt[2], s_ovf[2];  // queue fill and overflow flag, by round parity
  const int nwords = (int)ceil_div(n, 32);
  int32_t *const qbase = reinterpret_cast<int32_t *>(queued + nwords);  // two queues
  int32_t *const heavy = qbase + 2 * kSsspQueue;
  const T inf = Dist<T>::inf();
  const int32_t inf_bits = order_bits<T>(inf + inf);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;

  for (int si = blockIdx.x; si < num_sources; si += gridDim.x) {
    const int src = sources[si];
    T *orow = out + (out_rows ? out_rows[si] : (int64_t)si) * ld;
    T *dist = perm_out ? scratch + (int64_t)blockIdx.x * n : orow;
    if (src < 0 || src >= n) {
      if (threadIdx.x == 0) set_status(status, kDevBadIndex);
      continue;
    }
    const int64_t init = perm_out ? n : init_cols;
    for (int64_t v = threadIdx.x; v < init; v += blockDim.x) dist[v] = inf;
    for (int i = threadIdx.x; i < nwords; i += blockDim.x) queued[i] = 0;
    if (threadIdx.x < 3) s_minfar[threadIdx.x] = inf_bits;
    __syncthreads();
    if (threadIdx.x == 0) {
      dist[src] = T(0);
      queued[src >> 5] = 1u << (src & 31);
      qbase[0] = src;
      s_cnt[0] = 1;
      s_ovf[0] = 0;
      s_cnt[1] = 0;
      s_ovf[1] = 0;
    }
    __syncthreads();
    T thresh = delta;  // identical in every thread
    for (int64_t round = 0;; round++) {
      if (round >= max_rounds) {
        if (threadIdx.x == 0) set_status(status, kDevSsspRoundLimit);
        break;
      }
      const int cur = (int)(round & 1), nxt = cur ^ 1;
      const int slot = (int)(round % 3);
      if (threadIdx.x == 0) s_minfar[(slot + 1) % 3] = inf_bits;
      const int cnt = s_cnt[cur];
      const bool scan = s_ovf[cur] != 0;
      int32_t *const list = qbase + cur * kSsspQueue;
      int32_t *const nextq = qbase + nxt * kSsspQueue;
      int any = 0, far = 0;
      int32_t minfar = inf_bits;
      // Expand one frontier vertex (its queued bit already cleared).
      auto expand = [&](int u) {
        const T du = ld_relaxed(dist + u);
        if (!(du < thresh)) {  // far: keep it for a later bucket
          frontier_push(u, queued, nextq, &s_cnt[nxt], &s_ovf[nxt]);
          minfar = min(minfar, order_bits<T>(du));
          far = 1;
          return;
        }
        const int e0 = __ldg(row_offset + u), e1 = __ldg(row_offset + u + 1);
        if (e1 - e0 > kHeavyDeg) {
          const int h = atomicAdd(&s_nheavy, 1);
          if (h < kHeavyList) {
            heavy[h] = u;
            return;
          }
        }
        any |= relax_edges<T>(col, w, e0, e1, 1, du, dist, queued, nextq, &s_cnt[nxt], &s_ovf[nxt]);
      };
      auto heavy_pass = [&]() {
        const int nh = min(s_nheavy, kHeavyList);
        for (int h = wid; h < nh; h += kSsspThreads / 32) {
          const int u = heavy[h];
          const T du = ld_relaxed(dist + u);
          const int e0 = __ldg(row_offset + u), e1 = __ldg(row_offset + u + 1);
          any |= relax_edges<T>(col, w, e0 + lane, e1, 32, du, dist, queued, nextq, &s_cnt[nxt],
                                &s_ovf[nxt]);
        }
      };
      if (!scan) {
        // Queue round: the frontier is list[0, cnt).
        if (threadIdx.x == 0) s_nheavy = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
          const int u = list[i];
          atomicAnd(queued + (u >> 5), ~(1u << (u & 31)));
          expand(u);
        }
        __syncthreads();
        // every thread has read s_cnt[cur]: reset it for the round after next
        if (threadIdx.x == 0) {
          s_cnt[cur] = 0;
          s_ovf[cur] = 0;
        }
        heavy_pass();
      } else {
        // Overflow round: collect every marked vertex from the bitmap, in
        // passes of at most kSsspQueue (the current queue is reused as the
        // list; nothing pushes into it this round).
        for (;;) {
          int c = 0;
          for (int wi = threadIdx.x; wi < nwords; wi += blockDim.x) c += __popc(queued[wi]);
          const int off = block_excl_scan(c, s_warp, &s_total);
          const int total = s_total;
          if (total == 0) break;
          if (threadIdx.x == 0) s_nheavy = 0;
          int pos = off;
          for (int wi = threadIdx.x; wi < nwords && pos < kSsspQueue; wi += blockDim.x) {
            uint32_t m = queued[wi];
            if (!m) continue;
            uint32_t taken = 0;
            while (m && pos < kSsspQueue) {
              const int b = __ffs(m) - 1;
              m &= m - 1;
              list[pos++] = (wi << 5) + b;
              taken |= 1u << b;
            }
            queued[wi] &= ~taken;  // no pushes run during collection
          }
          __syncthreads();
          const int take = min(total, kSsspQueue);
          for (int i = threadIdx.x; i < take; i += blockDim.x) expand(list[i]);
          __syncthreads();
          heavy_pass();
          __syncthreads();
          // Vertices pushed during this pass are marked again; the next
          // round picks them up (from the queue, or by another scan).
          if (total <= kSsspQueue) break;
          // more marked vertices than one pass: the pushes of this pass are in
          // the bitmap as well, so keep collecting from it
        }
        if (threadIdx.x == 0) {
          s_cnt[cur] = 0;
          s_ovf[cur] = 0;
        }
      }
      if (far) atomicMin(&s_minfar[slot], minfar);
      const int active = __syncthreads_or(any);
      const int farany = __syncthreads_or(far);
      if (!active) {
        if (!farany) break;
        // Only far vertices remain: open the bucket of the nearest one.
        const T mf = from_order_bits<T>(s_minfar[slot]);
        thresh = (mf >= inf - delta) ? inf + inf : mf + delta;
      }
    }
    __syncthreads();
    if (perm_out) {
      for (int64_t v = threadIdx.x; v < init_cols; v += blockDim.x)
        orow[v] = v < n ? dist[__ldg(perm_out + v)] : inf;
      __syncthreads();
    }
  }
}

}  // namespace fapb
