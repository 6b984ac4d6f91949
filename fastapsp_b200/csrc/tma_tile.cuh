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

// The first 128-byte boundary at or after raw (dynamic shared memory).  The
// pointer is formed by arithmetic on raw itself, not through an integer, so
// that the compiler still knows it points to shared memory and accesses
// through it become shared-memory loads and stores with immediate offsets.
__device__ __forceinline__ unsigned char *smem_align128(unsigned char *raw) {
  return raw + ((128u - (smem_u32(raw) & 127u)) & 127u);
}

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
  unsigned char *a = smem_align128(raw);
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
template <typename T, class C, int GI, int GJ>
__device__ __forceinline__ void tma_k_step(const T *Arow, const T *Bs, T (&acc)[8][8], int tx, int k) {
  using V = typename Vec4<T>::type;
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

// (a full chunk runs with k unrolled: constant shared-memory offsets and no
// loop counter; a partial last chunk runs the rolled loop)
template <typename T, class C, int GI = 2, int GJ = 2>
__device__ __forceinline__ void tma_chunk_compute(const T *As, const T *Bs, T (&acc)[8][8], int ty,
                                                  int tx, int kc) {
  const T *Arow = As + (ty * 4) * C::BK;
  if (kc == C::BK) {
#pragma unroll
    for (int k = 0; k < C::BK; k++) tma_k_step<T, C, GI, GJ>(Arow, Bs, acc, tx, k);
  } else {
#pragma unroll 1
    for (int k = 0; k < kc; k++) tma_k_step<T, C, GI, GJ>(Arow, Bs, acc, tx, k);
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
  const int tid = threadIdx.x, ty = tid / C::TX, tx = tid % C::TX;
  // Rows are skipped per warp: a warp holds rows 8w..8w+7 of each row group
  // (two values of ty), so whether any of them is real is warp-uniform.
  // Columns span every warp, so they are skipped per tile half only.
  static_assert(C::TX == 16, "a warp holds two row quads of each group");
  const int w8 = (tid / 32) * 8;
  const bool rlo = !PAD || w8 < mvalid, rhi = !PAD || C::BM / 2 + w8 < mvalid;
  const bool chi = !PAD || nvalid > C::BN / 2;
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
      else if (rlo && chi) tma_chunk_compute<T, C, 1, 2>(As, As + C::A_ELEMS, acc, ty, tx, kc);
      else if (rlo) tma_chunk_compute<T, C, 1, 1>(As, As + C::A_ELEMS, acc, ty, tx, kc);
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

// ---------------------------------------------------------------------------
// Packed 16-bit form (int32 distances that provably fit in 14 bits after a
// per-column shift): one __viaddmin_s16x2 relaxes two outputs, the same
// column of two rows.  Stages arrive as int32 tiles through the same TMA
// ring; the CTA converts each stage into packed shared buffers:
//   PA[k][p]  = (A[2p][k], A[2p+1][k])            row pairs, k-major
//   PB[k][c]  = (B'[k][c], B'[k][c])              B' = B[k][c] - off[c]
// with every entry clamped to kPackCap (the sentinel and anything at least
// as large become kPackCap).  The caller guarantees, per tile, that every
// finite A is >= 0, every finite B' is in [0, range] and
// maxA + range < kPackCap: then every sum of finite entries is below
// kPackCap, every sum with a clamped entry is at least kPackCap, no sum
// exceeds 2 * kPackCap < 2^15, and a packed result r < kPackCap is exactly
// min_k A[i][k] + B[k][c] - off[c] (r >= kPackCap: no finite path).
// ---------------------------------------------------------------------------
constexpr int32_t kPackCap = 16383;
constexpr uint32_t kPackInit = 0x7FFE7FFEu;   // 32766 in both halves

template <class C>
struct Pack16Cfg {
  static constexpr int PA_LD = C::BM / 2 + 2;      // padded k-row of PA (conflict-free stores)
  static constexpr int PA_ELEMS = C::BK * PA_LD;
  static constexpr int PB_ELEMS = C::BK * C::BN;
  static constexpr int BUF_ELEMS = PA_ELEMS + PB_ELEMS;   // one buffer (two are used)
  // after the ring (128-byte aligned) and its mbarriers (64 bytes): the two
  // packed buffers, then the tile's column offsets, then its row offsets
  static constexpr int BUF_OFFSET = C::RING_BYTES + 64;
  static constexpr int SMEM_BYTES = 128 + BUF_OFFSET + 2 * BUF_ELEMS * 4 + C::BN * 4 + C::BM * 4;
  static_assert(C::STAGES * 8 <= 64, "mbarriers fit before the packed buffers");
  static_assert((PA_ELEMS * 4) % 16 == 0 && (BUF_ELEMS * 4) % 16 == 0, "16-byte aligned buffers");
  static_assert(C::BM == 128 && C::BN == 128 && C::THREADS == 256, "thread mapping below");
  static_assert((C::BK * C::BM / 2) % C::THREADS == 0 && (C::BK * C::BN) % C::THREADS == 0, "even split");
};

__device__ __forceinline__ uint32_t pack_pair(int32_t lo, int32_t hi) {
  return (uint32_t)(lo & 0xffff) | ((uint32_t)hi << 16);
}

// An entry shifted by its offset and clamped: the sentinel (and anything at
// least kPackCap above the offset) becomes kPackCap.
__device__ __forceinline__ int32_t pack_clamp(int32_t v, int32_t off) {
  return v >= kInfI32 ? kPackCap : min(v - off, kPackCap);
}

// Converts ring stage (As, Bs) (kc valid k of BK) into PA / PB.  roff: the
// tile's BM row offsets of A, coff: its BN column offsets of B, in shared
// memory (either may be null: no shift).
template <class C>
__device__ __forceinline__ void pack16_convert(const int32_t *As, const int32_t *Bs, uint32_t *PA,
                                               uint32_t *PB, const int32_t *roff, const int32_t *coff) {
  using P = Pack16Cfg<C>;
  const int tid = threadIdx.x;
  // A: BK x BM/2 pairs; thread -> (k = tid % BK, p = tid / BK + q * THREADS / BK)
#pragma unroll
  for (int q = 0; q < (C::BK * C::BM / 2) / C::THREADS; q++) {
    const int k = tid % C::BK, p = tid / C::BK + q * (C::THREADS / C::BK);
    const int32_t a0 = pack_clamp(As[(2 * p) * C::BK + k], roff ? roff[2 * p] : 0);
    const int32_t a1 = pack_clamp(As[(2 * p + 1) * C::BK + k], roff ? roff[2 * p + 1] : 0);
    PA[k * P::PA_LD + p] = pack_pair(a0, a1);
  }
  // B: BK x BN, column fastest
#pragma unroll
  for (int q = 0; q < (C::BK * C::BN) / C::THREADS; q++) {
    const int e = tid + q * C::THREADS;
    const int32_t v = pack_clamp(Bs[e], coff ? coff[e % C::BN] : 0);
    PB[e] = pack_pair(v, v);
  }
}

// One converted chunk: per k, the thread's 4 row pairs (two 8-byte loads)
// and 8 columns (two 16-byte loads), then 32 packed relaxations.
template <class C, int GI>
__device__ __forceinline__ void pack16_k_step(const uint32_t *PA, const uint32_t *PB, uint32_t (&acc)[4][8],
                                              int ty, int tx, int k) {
  using P = Pack16Cfg<C>;
  uint32_t a[4], b[8];
#pragma unroll
  for (int g = 0; g < GI; g++) {
    const uint2 v = *reinterpret_cast<const uint2 *>(PA + k * P::PA_LD + g * (C::BM / 4) + ty * 2);
    a[2 * g] = v.x;
    a[2 * g + 1] = v.y;
  }
#pragma unroll
  for (int g = 0; g < 2; g++) {
    const uint4 v = *reinterpret_cast<const uint4 *>(PB + k * C::BN + g * (C::BN / 2) + tx * 4);
    b[4 * g + 0] = v.x; b[4 * g + 1] = v.y; b[4 * g + 2] = v.z; b[4 * g + 3] = v.w;
  }
#pragma unroll
  for (int i = 0; i < 2 * GI; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) acc[i][j] = __viaddmin_s16x2(a[i], b[j], acc[i][j]);
}

template <class C, int GI = 2>
__device__ __forceinline__ void pack16_chunk_compute(const uint32_t *PA, const uint32_t *PB,
                                                     uint32_t (&acc)[4][8], int ty, int tx, int kc) {
  if (kc == C::BK) {
#pragma unroll
    for (int k = 0; k < C::BK; k++) pack16_k_step<C, GI>(PA, PB, acc, ty, tx, k);
  } else {
#pragma unroll 1
    for (int k = 0; k < kc; k++) pack16_k_step<C, GI>(PA, PB, acc, ty, tx, k);
  }
}

// The packed form of tma_minplus_tile (same boxes, same bounded waits).
// pbuf: 2 * BUF_ELEMS words of shared memory; roff / coff: BM row offsets of
// A / BN column offsets of B in shared memory (null: no shift), written
// before the call (the first barrier below orders them before their use).
template <class C>
__device__ __forceinline__ bool tma_minplus_tile16(const CUtensorMap *mapA, int ax, int ay, int az,
                                                   const CUtensorMap *mapB, int bx, int by, int bz,
                                                   int K, uint32_t (&acc)[4][8], TmaSmem<int32_t, C> &sm,
                                                   uint32_t *pbuf, const int32_t *roff, const int32_t *coff,
                                                   int mvalid = C::BM) {
  using P = Pack16Cfg<C>;
  const int tid = threadIdx.x, ty = tid / C::TX, tx = tid % C::TX;
  // rows skipped per warp as in tma_minplus_tile (row pairs of a warp lie
  // in its rows 8w..8w+7 of each group)
  const int w8 = (tid / 32) * 8;
  const bool rlo = w8 < mvalid, rhi = C::BM / 2 + w8 < mvalid;
  const int n = (int)ceil_div(K, C::BK);
  if (n == 0) return true;
  auto issue = [&](int c, int s) {
    int32_t *As = sm.ring + s * C::STAGE_ELEMS;
    int32_t *Bs = As + C::A_ELEMS;
    mbar_arrive_expect_tx(&sm.bars[s], C::TX_BYTES);
    tma_load_3d(As, mapA, ax + c * C::BK, ay, az, &sm.bars[s]);
    tma_load_3d(Bs, mapB, bx, by + c * C::BK, bz, &sm.bars[s]);
  };
  fence_proxy_async_all();
  __syncthreads();
  if (tid == 0)
    for (int c = 0; c < n && c < C::STAGES; c++) issue(c, c);
  for (int c = 0; c < n; c++) {
    const int s = c % C::STAGES;
    const bool got = mbar_wait_bounded(&sm.bars[s], (sm.phase >> s) & 1u);
    sm.phase ^= 1u << s;
    uint32_t *PA = pbuf + (c & 1) * P::BUF_ELEMS;
    uint32_t *PB = PA + P::PA_ELEMS;
    if (got) {
      const int32_t *As = sm.ring + s * C::STAGE_ELEMS;
      pack16_convert<C>(As, As + C::A_ELEMS, PA, PB, roff, coff);
    }
    fence_proxy_async_smem();  // this thread's reads of stage s precede its refill
    // One barrier per chunk: after it the stage may be refilled (every
    // thread has converted it) and the packed buffer read; the other packed
    // buffer was last read in the previous chunk, before this barrier.
    if (__syncthreads_or(!got)) {
      for (int c2 = c + 1; c2 < n && c2 < c + C::STAGES; c2++) {
        const int s2 = c2 % C::STAGES;
        if (tid == 0) mbar_wait_bounded(&sm.bars[s2], (sm.phase >> s2) & 1u);
        sm.phase ^= 1u << s2;
      }
      __syncthreads();
      return false;
    }
    if (tid == 0 && c + C::STAGES < n) issue(c + C::STAGES, s);
    if (rhi) pack16_chunk_compute<C, 2>(PA, PB, acc, ty, tx, min(C::BK, K - c * C::BK));
    else if (rlo) pack16_chunk_compute<C, 1>(PA, PB, acc, ty, tx, min(C::BK, K - c * C::BK));
  }
  return true;
}

// ---------------------------------------------------------------------------
// Packed 16-bit form on operands packed in global memory beforehand, so that
// the stages arrive ready for the relaxations (no conversion, no second
// barrier per chunk).  One __viaddmin_s16x2 relaxes one row against two
// adjacent columns:
//   AT[k][i] = (A'[i][k], A'[i][k])     uint32, k-major (i fastest)
//   S[k][c]  = B'[k][c]                 uint16, so a uint32 holds columns
//                                       (c, c+1) of row k
// with the clamping and bounds of the in-kernel form above (the caller
// packs both arrays; A' = min(A, kPackCap), B' = min(B - off[c], kPackCap)).
// A stage is the AT box (x = rows ax.., y = k) and the S box (x = columns
// bx.., y = k), both at y = ky + c * BK.  acc[i][p]: row tile_row(i), columns
// tile_col(2p mod 4 ..) as in Pack16pCfg below.
// ---------------------------------------------------------------------------
template <class C>
struct Pack16pCfg {
  static constexpr int A_WORDS = C::BK * C::BM;        // AT box: BK rows of BM uint32
  static constexpr int B_WORDS = C::BK * C::BN / 2;    // S box: BK rows of BN uint16
  static constexpr int STAGE_WORDS = A_WORDS + B_WORDS;
  static constexpr uint32_t TX_BYTES = STAGE_WORDS * 4;
  static_assert(C::STAGES * STAGE_WORDS * 4 <= C::RING_BYTES, "the packed ring fits in the int32 ring");
  static_assert((A_WORDS * 4) % 128 == 0 && (STAGE_WORDS * 4) % 128 == 0, "128-byte aligned boxes");
  static_assert(C::BM == 128 && C::BN == 128 && C::THREADS == 256 && C::TX == 16, "thread mapping below");
};

// One chunk: per k, the thread's 8 rows (two 16-byte loads: rows ty*4..+3 of
// each row group, duplicated halves) and 4 column pairs (two 8-byte loads:
// columns tx*4..+3 of each column group), then 32 packed relaxations.
template <class C, int GI>
__device__ __forceinline__ void pack16p_k_step(const uint32_t *As, const uint32_t *Bs, uint32_t (&acc)[8][4],
                                               int ty, int tx, int k) {
  uint32_t a[8], b[4];
#pragma unroll
  for (int g = 0; g < GI; g++) {
    const uint4 v = *reinterpret_cast<const uint4 *>(As + k * C::BM + g * (C::BM / 2) + ty * 4);
    a[4 * g + 0] = v.x; a[4 * g + 1] = v.y; a[4 * g + 2] = v.z; a[4 * g + 3] = v.w;
  }
#pragma unroll
  for (int g = 0; g < 2; g++) {
    const uint2 v = *reinterpret_cast<const uint2 *>(Bs + k * (C::BN / 2) + g * (C::BN / 4) + tx * 2);
    b[2 * g + 0] = v.x; b[2 * g + 1] = v.y;
  }
#pragma unroll
  for (int i = 0; i < 4 * GI; i++)
#pragma unroll
    for (int p = 0; p < 4; p++) acc[i][p] = __viaddmin_s16x2(a[i], b[p], acc[i][p]);
}

template <class C, int GI = 2>
__device__ __forceinline__ void pack16p_chunk_compute(const uint32_t *As, const uint32_t *Bs,
                                                      uint32_t (&acc)[8][4], int ty, int tx, int kc) {
  if (kc == C::BK) {
#pragma unroll
    for (int k = 0; k < C::BK; k++) pack16p_k_step<C, GI>(As, Bs, acc, ty, tx, k);
  } else {
#pragma unroll 1
    for (int k = 0; k < kc; k++) pack16p_k_step<C, GI>(As, Bs, acc, ty, tx, k);
  }
}

// The pre-packed form of tma_minplus_tile16: the same ring protocol as
// tma_minplus_tile (one barrier per chunk, bounded waits, drain on a
// timeout) over the int32 ring's memory and mbarriers.  mvalid: rows of the
// tile that are not padding (warps holding none of them skip the work).
template <class C>
__device__ __forceinline__ bool tma_minplus_tile16p(const CUtensorMap *mapA, int ax, const CUtensorMap *mapB,
                                                    int bx, int ky, int K, uint32_t (&acc)[8][4],
                                                    TmaSmem<int32_t, C> &sm, int mvalid = C::BM) {
  using P = Pack16pCfg<C>;
  const int tid = threadIdx.x, ty = tid / C::TX, tx = tid % C::TX;
  const int w8 = (tid / 32) * 8;
  const bool rlo = w8 < mvalid, rhi = C::BM / 2 + w8 < mvalid;
  const int n = (int)ceil_div(K, C::BK);
  if (n == 0) return true;
  uint32_t *ring = reinterpret_cast<uint32_t *>(sm.ring);
  auto issue = [&](int c, int s) {
    uint32_t *As = ring + s * P::STAGE_WORDS;
    mbar_arrive_expect_tx(&sm.bars[s], P::TX_BYTES);
    tma_load_3d(As, mapA, ax, ky + c * C::BK, 0, &sm.bars[s]);
    tma_load_3d(As + P::A_WORDS, mapB, bx, ky + c * C::BK, 0, &sm.bars[s]);
  };
  fence_proxy_async_all();
  __syncthreads();
  if (tid == 0)
    for (int c = 0; c < n && c < C::STAGES; c++) issue(c, c);
  for (int c = 0; c < n; c++) {
    const int s = c % C::STAGES;
    const bool got = mbar_wait_bounded(&sm.bars[s], (sm.phase >> s) & 1u);
    sm.phase ^= 1u << s;
    if (got) {
      const uint32_t *As = ring + s * P::STAGE_WORDS;
      const int kc = min(C::BK, K - c * C::BK);
      if (rhi) pack16p_chunk_compute<C, 2>(As, As + P::A_WORDS, acc, ty, tx, kc);
      else if (rlo) pack16p_chunk_compute<C, 1>(As, As + P::A_WORDS, acc, ty, tx, kc);
    }
    fence_proxy_async_smem();  // this thread's reads of stage s precede its refill
    if (__syncthreads_or(!got)) {
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

// ---------------------------------------------------------------------------
// Packed 16-bit form on row pairs packed beforehand: the A box holds BK rows
// (k) of BM/2 words, each word two rows of A (row 2p in the low half), and
// the B box BK rows of BN words with both halves equal; one
// __viaddmin_s16x2 relaxes two rows against one column, as in
// tma_minplus_tile16 (acc[i][j]: pair i = 2g + h, rows 4g + 2h and the next
// of the thread, column j), without the conversion.
// ---------------------------------------------------------------------------
template <class C>
struct Pack16qCfg {
  static constexpr int A_WORDS = C::BK * C::BM / 2;
  static constexpr int B_WORDS = C::BK * C::BN;
  static constexpr int STAGE_WORDS = A_WORDS + B_WORDS;
  static constexpr uint32_t TX_BYTES = STAGE_WORDS * 4;
  static_assert(C::STAGES * STAGE_WORDS * 4 <= C::RING_BYTES, "the packed ring fits in the int32 ring");
  static_assert((A_WORDS * 4) % 128 == 0 && (STAGE_WORDS * 4) % 128 == 0, "128-byte aligned boxes");
  static_assert(C::BM == 128 && C::BN == 128 && C::THREADS == 256 && C::TX == 16, "thread mapping below");
};

template <class C, int GI>
__device__ __forceinline__ void pack16q_k_step(const uint32_t *PA, const uint32_t *PB, uint32_t (&acc)[4][8],
                                               int ty, int tx, int k) {
  uint32_t a[4], b[8];
#pragma unroll
  for (int g = 0; g < GI; g++) {
    const uint2 v = *reinterpret_cast<const uint2 *>(PA + k * (C::BM / 2) + g * (C::BM / 4) + ty * 2);
    a[2 * g] = v.x;
    a[2 * g + 1] = v.y;
  }
#pragma unroll
  for (int g = 0; g < 2; g++) {
    const uint4 v = *reinterpret_cast<const uint4 *>(PB + k * C::BN + g * (C::BN / 2) + tx * 4);
    b[4 * g + 0] = v.x; b[4 * g + 1] = v.y; b[4 * g + 2] = v.z; b[4 * g + 3] = v.w;
  }
#pragma unroll
  for (int i = 0; i < 2 * GI; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) acc[i][j] = __viaddmin_s16x2(a[i], b[j], acc[i][j]);
}

template <class C, int GI>
__device__ __forceinline__ void pack16q_chunk_compute(const uint32_t *PA, const uint32_t *PB,
                                                      uint32_t (&acc)[4][8], int ty, int tx, int kc) {
  if (kc == C::BK) {
#pragma unroll
    for (int k = 0; k < C::BK; k++) pack16q_k_step<C, GI>(PA, PB, acc, ty, tx, k);
  } else {
#pragma unroll 1
    for (int k = 0; k < kc; k++) pack16q_k_step<C, GI>(PA, PB, acc, ty, tx, k);
  }
}

// A boxes at (ax, ky + c*BK) of mapA (ax: the tile's first row pair), B
// boxes at (bx, ky + c*BK) of mapB; the same ring protocol as
// tma_minplus_tile.  mvalid: rows of the tile that are not padding.
template <class C>
__device__ __forceinline__ bool tma_minplus_tile16q(const CUtensorMap *mapA, int ax, const CUtensorMap *mapB,
                                                    int bx, int ky, int K, uint32_t (&acc)[4][8],
                                                    TmaSmem<int32_t, C> &sm, int mvalid = C::BM) {
  using P = Pack16qCfg<C>;
  const int tid = threadIdx.x, ty = tid / C::TX, tx = tid % C::TX;
  const int w8 = (tid / 32) * 8;
  const bool rlo = w8 < mvalid, rhi = C::BM / 2 + w8 < mvalid;
  const int n = (int)ceil_div(K, C::BK);
  if (n == 0) return true;
  uint32_t *ring = reinterpret_cast<uint32_t *>(sm.ring);
  auto issue = [&](int c, int s) {
    uint32_t *As = ring + s * P::STAGE_WORDS;
    mbar_arrive_expect_tx(&sm.bars[s], P::TX_BYTES);
    tma_load_3d(As, mapA, ax, ky + c * C::BK, 0, &sm.bars[s]);
    tma_load_3d(As + P::A_WORDS, mapB, bx, ky + c * C::BK, 0, &sm.bars[s]);
  };
  fence_proxy_async_all();
  __syncthreads();
  if (tid == 0)
    for (int c = 0; c < n && c < C::STAGES; c++) issue(c, c);
  for (int c = 0; c < n; c++) {
    const int s = c % C::STAGES;
    const bool got = mbar_wait_bounded(&sm.bars[s], (sm.phase >> s) & 1u);
    sm.phase ^= 1u << s;
    if (got) {
      const uint32_t *As = ring + s * P::STAGE_WORDS;
      const int kc = min(C::BK, K - c * C::BK);
      if (rhi) pack16q_chunk_compute<C, 2>(As, As + P::A_WORDS, acc, ty, tx, kc);
      else if (rlo) pack16q_chunk_compute<C, 1>(As, As + P::A_WORDS, acc, ty, tx, kc);
    }
    fence_proxy_async_smem();  // this thread's reads of stage s precede its refill
    if (__syncthreads_or(!got)) {
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
