// TMA-fed register-tiled min-plus engine (sm_100a):
//
//   acc[i][j] = min(acc[i][j], min_k A[i][k] + B[k][j])
//
// over a BM x BN tile.  One thread streams the K dimension in chunks of BK
// through a ring of STAGES shared-memory buffers with tiled TMA loads (A box
// BM x BK, B box BK x BN, both row-major as in global memory); the other
// threads only compute.  Completion of each stage is counted on its own
// mbarrier; a stage is refilled once every thread has passed the barrier that
// ends its use.  No register staging of loads, so the 8 x 8 accumulator tile
// fits two CTAs per SM.  Waits are bounded: on a timeout the engine drains
// the copies it still has in flight (bounded too) and reports failure
// uniformly to the whole CTA.
#pragma once

#include <cuda.h>

#include "minplus_tile.cuh"
#include "tma.cuh"

namespace fapb {

template <typename T, int BM_, int BN_, int BK_, int STAGES_>
struct TmaTileCfg {
  static constexpr int BM = BM_, BN = BN_, BK = BK_, STAGES = STAGES_;
  static constexpr int TM = 8, TN = 8, GM = 2, GN = 2;
  static constexpr int TY = BM / TM, TX = BN / TN;
  static constexpr int THREADS = TY * TX;
  static constexpr int A_ELEMS = BM * BK;
  static constexpr int B_ELEMS = BK * BN;
  static constexpr int STAGE_ELEMS = A_ELEMS + B_ELEMS;
  static constexpr uint32_t TX_BYTES = STAGE_ELEMS * sizeof(T);
  static constexpr int RING_BYTES = STAGES * STAGE_ELEMS * (int)sizeof(T);
  // ring + mbarriers + slack for 128-byte alignment of the ring
  static constexpr int SMEM_BYTES = RING_BYTES + STAGES * 8 + 128;
  static_assert(BK % 16 == 0, "A boxes start on 16-element (64-byte) boundaries");
  static_assert((A_ELEMS * sizeof(T)) % 128 == 0 && (B_ELEMS * sizeof(T)) % 128 == 0, "aligned boxes");
};

// Carved dynamic shared memory of a TMA tile CTA.
template <typename T, class C>
struct TmaSmem {
  T *ring;
  uint64_t *bars;
  uint32_t phase;  // bit s = parity of stage s's next completion (same in all threads)
};

template <typename T, class C>
__device__ __forceinline__ TmaSmem<T, C> tma_smem_init(unsigned char *raw) {
  TmaSmem<T, C> s;
  const uintptr_t a = (reinterpret_cast<uintptr_t>(raw) + 127) & ~uintptr_t(127);
  s.ring = reinterpret_cast<T *>(a);
  s.bars = reinterpret_cast<uint64_t *>(a + C::RING_BYTES);
  s.phase = 0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < C::STAGES; i++) mbar_init(&s.bars[i], 1);
    fence_mbar_init();
  }
  __syncthreads();
  return s;
}

// One chunk of K from shared memory: As is BM x BK, Bs is BK x BN.  Per k:
// the thread's 8 A values are 8 broadcast loads (each address is shared by
// the 16 threads of a half-warp), its 8 B values two conflict-free 16-byte
// loads, then 64 relaxations.  GI / GJ: the thread's row / column groups
// computed (1 skips the second group, rows or columns BM/2.. or BN/2..,
// when they are all padding).
template <typename T, class C, int GI = 2, int GJ = 2>
__device__ __forceinline__ void tma_chunk_compute(const T *As, const T *Bs, T (&acc)[8][8], int ty,
                                                  int tx, int kc) {
  using V = typename Vec4<T>::type;
  const T *Arow = As + (ty * 4) * C::BK;
#pragma unroll 4
  for (int k = 0; k < kc; k++) {
    T a[8], b[8];
#pragma unroll
    for (int g = 0; g < GI; g++)
#pragma unroll
      for (int l = 0; l < 4; l++) a[4 * g + l] = Arow[(g * (C::BM / 2) + l) * C::BK + k];
#pragma unroll
    for (int g = 0; g < GJ; g++) {
      const V v = *reinterpret_cast<const V *>(Bs + k * C::BN + g * (C::BN / 2) + tx * 4);
      b[4 * g + 0] = v.x; b[4 * g + 1] = v.y; b[4 * g + 2] = v.z; b[4 * g + 3] = v.w;
    }
#pragma unroll
    for (int i = 0; i < 4 * GI; i++)
#pragma unroll
      for (int j = 0; j < 4 * GJ; j++) acc[i][j] = Dist<T>::relax(a[i], b[j], acc[i][j]);
  }
}

// acc <- min(acc, A (x) B) for K elements of the inner dimension, A boxes at
// (ax + c*BK, ay, az) of mapA and B boxes at (bx, by + c*BK, bz) of mapB.
// Block-wide.  Returns false (in every thread) if a stage never completed.
// mvalid / nvalid: rows / columns of the tile that are not padding (the
// second half of the thread's rows or columns is skipped when they are all
// padding; the caller's padding then keeps its values).
// (PAD: the caller may pass tiles with padding; otherwise the full-tile
// compute is the only one compiled.)
template <typename T, class C, bool PAD = false>
__device__ __forceinline__ bool tma_minplus_tile(const CUtensorMap *mapA, int ax, int ay, int az,
                                                 const CUtensorMap *mapB, int bx, int by, int bz,
                                                 int K, T (&acc)[8][8], TmaSmem<T, C> &sm,
                                                 int mvalid = C::BM, int nvalid = C::BN) {
  const bool rhi = !PAD || mvalid > C::BM / 2, chi = !PAD || nvalid > C::BN / 2;
  const int tid = threadIdx.x, ty = tid / C::TX, tx = tid % C::TX;
  const int n = (int)ceil_div(K, C::BK);
  if (n == 0) return true;
  auto issue = [&](int c, int s) {
    T *As = sm.ring + s * C::STAGE_ELEMS;
    T *Bs = As + C::A_ELEMS;
    mbar_arrive_expect_tx(&sm.bars[s], C::TX_BYTES);
    tma_load_3d(As, mapA, ax + c * C::BK, ay, az, &sm.bars[s]);
    tma_load_3d(Bs, mapB, bx, by + c * C::BK, bz, &sm.bars[s]);
  };
  // every thread's earlier accesses to the ring (and to the tiles about to be
  // loaded) come before the first copies
  fence_proxy_async_all();
  __syncthreads();
  if (tid == 0)
    for (int c = 0; c < n && c < C::STAGES; c++) issue(c, c);
  for (int c = 0; c < n; c++) {
    const int s = c % C::STAGES;
    const bool got = mbar_wait_bounded(&sm.bars[s], (sm.phase >> s) & 1u);
    sm.phase ^= 1u << s;
    if (got) {
      const T *As = sm.ring + s * C::STAGE_ELEMS;
      const int kc = min(C::BK, K - c * C::BK);
      if (!PAD || (rhi && chi)) tma_chunk_compute<T, C, 2, 2>(As, As + C::A_ELEMS, acc, ty, tx, kc);
      else if (rhi) tma_chunk_compute<T, C, 2, 1>(As, As + C::A_ELEMS, acc, ty, tx, kc);
      else if (chi) tma_chunk_compute<T, C, 1, 2>(As, As + C::A_ELEMS, acc, ty, tx, kc);
      else tma_chunk_compute<T, C, 1, 1>(As, As + C::A_ELEMS, acc, ty, tx, kc);
    }
    fence_proxy_async_smem();  // this thread's reads of stage s precede its refill
    if (__syncthreads_or(!got)) {
      // drain the stages still in flight, then give up
      for (int c2 = c + 1; c2 < n && c2 < c + C::STAGES; c2++) {
        const int s2 = c2 % C::STAGES;
        if (tid == 0) mbar_wait_bounded(&sm.bars[s2], (sm.phase >> s2) & 1u);
        sm.phase ^= 1u << s2;
      }
      __syncthreads();
      return false;
    }
    if (tid == 0 && c + C::STAGES < n) issue(c + C::STAGES, s);
  }
  return true;
}

}  // namespace fapb
