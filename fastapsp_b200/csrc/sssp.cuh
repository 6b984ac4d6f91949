// Stage 1: batched multi-source shortest paths from boundary vertices.
//
// Replaces handle_boundry_Nvidia_GPU / multi_source_Nvidia_sssp
// (fap/kernel/cuda/batch_sssp.cu:222-296), which ran one source at a time
// with a host round trip per Bellman-Ford iteration, and the CPU
// batched_sssp_path (fap/kernel/batch_sssp.h:232-252).
//
// Design: one CTA per source, all sources of all requested parts in one
// launch.  The distance row lives in the output matrix (global memory,
// relaxed with atomicMin); the frontier is a pair of bitmaps in shared
// memory (n bits each), so frontier dedup is free and a round costs one
// shared-memory scan plus the edge relaxations of the active vertices.
// Vertices are expanded in near/far order (delta stepping): a frontier
// vertex whose distance is not below the current threshold stays in the
// bitmap for a later bucket; when no near vertex is left the threshold moves
// to (smallest far distance + delta).  delta = INF gives plain frontier
// Bellman-Ford.  Convergence needs no host round trip and no inter-CTA
// synchronisation; the number of rounds is bounded and a CTA that hits the
// bound records an error status and stops (it never spins).
#pragma once

#include "fap_common.cuh"

namespace fapb {

constexpr int kSsspThreads = 256;

// Shared-memory bytes a CTA needs for n vertices.
inline size_t sssp_smem_bytes(int n) { return 2 * (size_t)ceil_div(n, 32) * sizeof(uint32_t); }

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
__global__ void __launch_bounds__(kSsspThreads)
    sssp_bitmap_kernel(const int32_t *__restrict__ row_offset, const int32_t *__restrict__ col,
                       const T *__restrict__ w, int n, const int32_t *__restrict__ sources,
                       const int64_t *__restrict__ out_rows, int num_sources, T *out, int64_t ld,
                       int64_t init_cols, T delta, int64_t max_rounds, int *status) {
  extern __shared__ uint32_t sm_bits[];
  __shared__ int32_t s_minfar[3];
  const int nwords = (int)ceil_div(n, 32);
  const T inf = Dist<T>::inf();
  const int32_t inf_bits = order_bits<T>(inf + inf);

  for (int si = blockIdx.x; si < num_sources; si += gridDim.x) {
    const int src = sources[si];
    T *dist = out + (out_rows ? out_rows[si] : (int64_t)si) * ld;
    if (src < 0 || src >= n) {
      if (threadIdx.x == 0) set_status(status, kDevBadIndex);
      continue;
    }
    for (int64_t v = threadIdx.x; v < init_cols; v += blockDim.x) dist[v] = inf;
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
      // Reset the slot used two rounds from now; its last readers finished
      // before the previous round's barrier.
      if (threadIdx.x == 0) s_minfar[(slot + 1) % 3] = inf_bits;
      uint32_t *cb = sm_bits + cur * nwords, *nb = sm_bits + (cur ^ 1) * nwords;
      int any = 0, far = 0;
      int32_t minfar = inf_bits;
      for (int wi = threadIdx.x; wi < nwords; wi += blockDim.x) {
        uint32_t m = cb[wi];
        if (!m) continue;
        cb[wi] = 0;
        uint32_t keep = 0;
        while (m) {
          const int b = __ffs(m) - 1;
          m &= m - 1;
          const int u = (wi << 5) + b;
          const T du = *((volatile T *)(dist + u));
          if (!(du < thresh)) {  // far: expand in a later bucket
            keep |= 1u << b;
            minfar = min(minfar, order_bits<T>(du));
            continue;
          }
          const int e0 = __ldg(row_offset + u), e1 = __ldg(row_offset + u + 1);
          for (int e = e0; e < e1; e++) {
            const int v = __ldg(col + e);
            const T nd = du + __ldg(w + e);
            if (nd < *((volatile T *)(dist + v))) {
              const T old = Dist<T>::atomic_min(dist + v, nd);
              if (nd < old) {
                atomicOr(nb + (v >> 5), 1u << (v & 31));
                any = 1;
              }
            }
          }
        }
        if (keep) {
          atomicOr(nb + wi, keep);
          far = 1;
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
      cur ^= 1;
    }
    __syncthreads();
  }
}

}  // namespace fapb
