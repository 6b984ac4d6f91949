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
//   - Frontier: a pair of bitmaps in shared memory (n bits each); dedup is
//     free.  Each round compacts the set bits into a shared list with a block
//     scan, so active vertices are spread evenly over the threads.
//   - Expansion: a thread relaxes a light vertex's edges with all loads and
//     atomics of a 4-edge group in flight at once; vertices with more than
//     kHeavyDeg edges are expanded by a whole warp (lane-strided, coalesced
//     column/weight reads).
//   - Relaxation: a plain read of dist[v] first skips the atomic when it
//     cannot improve (fewer atomics) at the price of one more dependent
//     access; `precheck` selects it.
//   - Chains: a thread that improves a near neighbour expands it at once
//     (up to `chain` hops per round) instead of leaving it for the next
//     round, so a hop along a path costs one load + atomic latency rather
//     than a whole round.
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
constexpr int kSsspList = 2048;   // compacted frontier entries per pass
constexpr int kHeavyDeg = 32;     // vertices above this degree go to a warp
constexpr int kHeavyList = 256;

// Shared-memory bytes a CTA needs for n vertices (dynamic part).
inline size_t sssp_smem_bytes(int n) {
  return 2 * (size_t)ceil_div(n, 32) * sizeof(uint32_t) + (kSsspList + kHeavyList) * sizeof(int32_t);
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

// Relaxes edges [e0, e1) of a light vertex at distance du.  One improved
// neighbour inside the current bucket may be handed back in *next / *dnext
// (chain-following: the caller expands it at once instead of a round later);
// every other improved neighbour gets its frontier bit.  Returns whether a bit
// was set.
template <typename T>
__device__ __forceinline__ bool relax_edges_chain(const int32_t *__restrict__ col,
                                                  const T *__restrict__ w, int e0, int e1, T du,
                                                  T *dist, uint32_t *nb, T thresh, bool may_chain,
                                                  bool precheck, int *next, T *dnext) {
  bool any = false;
  *next = -1;
  for (int e = e0; e < e1; e += 4) {
    int v[4];
    T nd[4], cur[4], old[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int ek = e + k;
      v[k] = ek < e1 ? __ldg(col + ek) : -1;
      nd[k] = ek < e1 ? du + __ldg(w + ek) : du;
    }
#pragma unroll
    for (int k = 0; k < 4; k++)
      cur[k] = v[k] < 0 ? du : precheck ? ld_relaxed(dist + v[k]) : Dist<T>::inf() + Dist<T>::inf();
#pragma unroll
    for (int k = 0; k < 4; k++)
      old[k] = (v[k] >= 0 && nd[k] < cur[k]) ? Dist<T>::atomic_min(dist + v[k], nd[k]) : nd[k];
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (nd[k] < old[k]) {
        if (may_chain && *next < 0 && nd[k] < thresh) {
          *next = v[k];
          *dnext = nd[k];
        } else {
          atomicOr(nb + (v[k] >> 5), 1u << (v[k] & 31));
          any = true;
        }
      }
  }
  return any;
}

// Relaxes edges [e0, e1) of a vertex at distance du; sets the frontier bit
// of every improved neighbour.  Returns whether anything improved.
template <typename T>
__device__ __forceinline__ bool relax_edges(const int32_t *__restrict__ col, const T *__restrict__ w,
                                            int e0, int e1, int stride, T du, T *dist,
                                            uint32_t *nb, bool precheck) {
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
    for (int k = 0; k < 4; k++)
      cur[k] = v[k] < 0 ? du : precheck ? ld_relaxed(dist + v[k]) : Dist<T>::inf() + Dist<T>::inf();
#pragma unroll
    for (int k = 0; k < 4; k++)
      old[k] = (v[k] >= 0 && nd[k] < cur[k]) ? Dist<T>::atomic_min(dist + v[k], nd[k]) : nd[k];
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (nd[k] < old[k]) {
        atomicOr(nb + (v[k] >> 5), 1u << (v[k] & 31));
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
__global__ void __launch_bounds__(kSsspThreads)
    sssp_frontier_kernel(const int32_t *__restrict__ row_offset, const int32_t *__restrict__ col,
                         const T *__restrict__ w, int n, const int32_t *__restrict__ sources,
                         const int64_t *__restrict__ out_rows, int num_sources, T *out, int64_t ld,
                         int64_t init_cols, const int32_t *__restrict__ perm_out, T *scratch,
                         T delta, int chain, int precheck, int64_t max_rounds, int *status) {
  extern __shared__ uint32_t sm_bits[];
  __shared__ int32_t s_minfar[3];
  __shared__ int s_warp[kSsspThreads / 32];
  __shared__ int s_total, s_nheavy;
  const int nwords = (int)ceil_div(n, 32);
  int32_t *act = reinterpret_cast<int32_t *>(sm_bits + 2 * nwords);
  int32_t *heavy = act + kSsspList;
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
    for (int i = threadIdx.x; i < 2 * nwords; i += blockDim.x) sm_bits[i] = 0;
    if (threadIdx.x < 3) s_minfar[threadIdx.x] = inf_bits;
    __syncthreads();
    if (threadIdx.x == 0) {
      dist[src] = T(0);
      sm_bits[src >> 5] = 1u << (src & 31);
    }
    __syncthreads();
    T thresh = delta;  // identical in every thread
    int cur = 0;
    for (int64_t round = 0;; round++) {
      if (round >= max_rounds) {
        if (threadIdx.x == 0) set_status(status, kDevSsspRoundLimit);
        break;
      }
      const int slot = (int)(round % 3);
      if (threadIdx.x == 0) s_minfar[(slot + 1) % 3] = inf_bits;
      uint32_t *cb = sm_bits + cur * nwords, *nb = sm_bits + (cur ^ 1) * nwords;
      int any = 0, far = 0;
      int32_t minfar = inf_bits;
      // Passes of at most kSsspList frontier vertices each.
      for (;;) {
        int cnt = 0;
        for (int wi = threadIdx.x; wi < nwords; wi += blockDim.x) cnt += __popc(cb[wi]);
        const int off = block_excl_scan(cnt, s_warp, &s_total);
        const int total = s_total;
        if (total == 0) break;
        if (threadIdx.x == 0) s_nheavy = 0;
        // Move the first kSsspList set bits (in thread order) to the list.
        int pos = off;
        for (int wi = threadIdx.x; wi < nwords && pos < kSsspList; wi += blockDim.x) {
          uint32_t m = cb[wi];
          if (!m) continue;
          uint32_t taken = 0;
          while (m && pos < kSsspList) {
            const int b = __ffs(m) - 1;
            m &= m - 1;
            act[pos++] = (wi << 5) + b;
            taken |= 1u << b;
          }
          cb[wi] &= ~taken;
        }
        __syncthreads();
        const int take = min(total, kSsspList);
        for (int i = threadIdx.x; i < take; i += blockDim.x) {
          const int u = act[i];
          // The distance and the edge range are independent loads: issue
          // them together (one latency instead of two).
          const T du = ld_relaxed(dist + u);
          const int u0 = __ldg(row_offset + u), u1 = __ldg(row_offset + u + 1);
          if (!(du < thresh)) {  // far: expand in a later bucket
            atomicOr(nb + (u >> 5), 1u << (u & 31));
            minfar = min(minfar, order_bits<T>(du));
            far = 1;
            continue;
          }
          // Expand u, then follow improved near neighbours in this thread.
          int x = u;
          T dx = du;
          for (int hop = 0;; hop++) {
            const int e0 = hop == 0 ? u0 : __ldg(row_offset + x);
            const int e1 = hop == 0 ? u1 : __ldg(row_offset + x + 1);
            if (e1 - e0 > kHeavyDeg) {
              const int h = atomicAdd(&s_nheavy, 1);
              if (h < kHeavyList) {
                heavy[h] = x;
                break;
              }
            }
            int nx;
            T dn;
            any |= relax_edges_chain<T>(col, w, e0, e1, dx, dist, nb, thresh, hop < chain, precheck != 0,
                                        &nx, &dn);
            if (nx < 0) break;
            x = nx;
            dx = dn;
          }
        }
        __syncthreads();
        // Heavy vertices: one warp each, lanes stride over the edges.
        const int nh = min(s_nheavy, kHeavyList);
        for (int h = wid; h < nh; h += kSsspThreads / 32) {
          const int u = heavy[h];
          const T du = ld_relaxed(dist + u);
          const int e0 = __ldg(row_offset + u), e1 = __ldg(row_offset + u + 1);
          any |= relax_edges<T>(col, w, e0 + lane, e1, 32, du, dist, nb, precheck != 0);
        }
        __syncthreads();
        if (total <= kSsspList) break;
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
      cur ^= 1;
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
