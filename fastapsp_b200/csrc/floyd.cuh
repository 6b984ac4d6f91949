// Stage 2: blocked Floyd-Warshall closure of each part's s x s matrix.
//
// Replaces floyd_GPU_Nvidia_path (fap/kernel/cuda/floyd.cu:284-348: one
// 32x32 tile per CTA, one element per thread, 2 launches per pivot) and the
// CPU floyd_CPU_path (fap/kernel/floyd.h:38-49).
//
// The matrices live in an arena of equal-sized padded squares (leading
// dimension ld, a multiple of TILE, part z at offset z * ld * ld), padded with
// the sentinel (padding never improves a real entry), so no tile needs bounds
// checks and one 3-D tensor map (column, row, part) describes every part.
// Per pivot block kb:
//   phase 1  close the diagonal tile D[kb][kb] with TILE sequential steps;
//            each thread keeps its TMxTN entries in registers and only the
//            pivot row/column of a step go through shared memory.
//   phase 2  row panel    D[kb][J] = min(D[kb][J], D*[kb][kb] (x) D[kb][J])
//            column panel D[I][kb] = min(D[I][kb], D[I][kb] (x) D*[kb][kb])
//            Because D*[kb][kb] is closed, one min-plus product gives what
//            TILE sequential pivot steps give.
//   phase 3  D[I][J] = min(D[I][J], D[I][kb] (x) D[kb][J])
// Phases 2 and 3 run on the TMA-fed tile engine (tma_tile.cuh).
//
// Drivers:
//   floyd_close_cta      one CTA closes one part's whole matrix;
//   floyd_*_phase kernels one launch per phase, tiles across the GPU.
#pragma once

#include "minplus_tile.cuh"
#include "tma_tile.cuh"

namespace fapb {

constexpr int kFloydStages = 4;

template <typename T, int TILE>
struct FloydCfg {
  using C = TileCfg<T, TILE, TILE, 16, 8, 8>;                 // register layout
  using TC = TmaTileCfg<T, TILE, TILE, 16, kFloydStages>;      // phase 2/3 engine
  static constexpr int THREADS = C::THREADS;
  static_assert(TC::THREADS == C::THREADS, "same thread layout");
  static constexpr int P1_BYTES = 4 * TILE * (int)sizeof(T);
  static constexpr int SMEM_BYTES = TC::SMEM_BYTES;
  static_assert(P1_BYTES <= TC::RING_BYTES, "phase-1 buffers fit in the ring");
};

// Phase 1 on the tile at (r0, r0) of a padded matrix.  Block-wide; `buf`
// holds 4*TILE elements of shared memory.  Pivots past kvalid (padding, the
// sentinel) change nothing and are skipped.
template <typename T, int TILE>
__device__ __forceinline__ void floyd_diag_close(T *mat, int64_t ld, int r0, T *buf, int kvalid = TILE) {
  using C = typename FloydCfg<T, TILE>::C;
  const int tid = threadIdx.x, ty = tid / C::TX, tx = tid % C::TX;
  T acc[C::TM][C::TN];
  acc_load<T, C, true>(acc, mat, ld, r0, r0, 0, 0);
  for (int k = 0; k < kvalid; k++) {
    T *rowbuf0 = buf + (k & 1) * TILE;
    T *colbuf0 = buf + 2 * TILE + (k & 1) * TILE;
    // publish the current pivot row k and pivot column k (all register
    // indices compile-time; the owner test selects the live copy)
    const int kg = k / (TILE / C::GM), kl = k % 4, kt = (k % (TILE / C::GM)) / 4;
    if (ty == kt) {
#pragma unroll
      for (int gi = 0; gi < C::GM; gi++)
#pragma unroll
        for (int l = 0; l < 4; l++)
          if (gi == kg && l == kl) {
#pragma unroll
            for (int g = 0; g < C::GN; g++)
#pragma unroll
              for (int q = 0; q < 4; q++)
                rowbuf0[tile_col<C>(tx, g, q)] = acc[4 * gi + l][4 * g + q];
          }
    }
    const int cg = k / (TILE / C::GN), cl = k % 4, ct = (k % (TILE / C::GN)) / 4;
    if (tx == ct) {
#pragma unroll
      for (int gj = 0; gj < C::GN; gj++)
#pragma unroll
        for (int l = 0; l < 4; l++)
          if (gj == cg && l == cl) {
#pragma unroll
            for (int g = 0; g < C::GM; g++)
#pragma unroll
              for (int q = 0; q < 4; q++)
                colbuf0[tile_row<C>(ty, g, q)] = acc[4 * g + q][4 * gj + l];
          }
    }
    __syncthreads();
    T a[C::TM], bb[C::TN];
#pragma unroll
    for (int g = 0; g < C::GM; g++)
#pragma unroll
      for (int q = 0; q < 4; q++) a[4 * g + q] = colbuf0[tile_row<C>(ty, g, q)];
#pragma unroll
    for (int g = 0; g < C::GN; g++)
#pragma unroll
      for (int q = 0; q < 4; q++) bb[4 * g + q] = rowbuf0[tile_col<C>(tx, g, q)];
#pragma unroll
    for (int i = 0; i < C::TM; i++)
#pragma unroll
      for (int j = 0; j < C::TN; j++) acc[i][j] = Dist<T>::relax(a[i], bb[j], acc[i][j]);
  }
  acc_store<T, C, true>(acc, mat, ld, r0, r0, 0, 0);
  __syncthreads();
}

// Phase 2/3 on one tile of part z: D[ti][tj] = min(D[ti][tj], D[ti][tk] (x)
// D[tk][tj]).  mat is the part's matrix (ld = arena leading dimension);
// mapA/mapB describe the arena with TILE x 16 and 16 x TILE boxes; only the
// first kvalid pivots of block tk, mvalid rows of block ti and nvalid columns
// of block tj are real (the rest is padding, the sentinel, left as it is).
// Block-wide; false if a TMA stage never completed.
template <typename T, int TILE>
__device__ __forceinline__ bool floyd_tile_update(const CUtensorMap *mapA, const CUtensorMap *mapB,
                                                  int z, T *mat, int64_t ld, int ti, int tj, int tk,
                                                  TmaSmem<T, typename FloydCfg<T, TILE>::TC> &sm,
                                                  int kvalid = TILE, int mvalid = TILE, int nvalid = TILE) {
  using C = typename FloydCfg<T, TILE>::C;
  using TC = typename FloydCfg<T, TILE>::TC;
  T acc[C::TM][C::TN];
  const int64_t r0 = (int64_t)ti * TILE, c0 = (int64_t)tj * TILE;
  acc_load<T, C, true>(acc, mat + r0 * ld + c0, ld, 0, 0, 0, 0);
  const bool ok = tma_minplus_tile<T, TC, true>(mapA, tk * TILE, ti * TILE, z, mapB, tj * TILE, tk * TILE,
                                                z, kvalid, acc, sm, mvalid, nvalid);
  if (ok) acc_store<T, C, true>(acc, mat + r0 * ld + c0, ld, 0, 0, 0, 0);
  return ok;
}

// floyd_tile_update, and for a symmetric matrix (transpose, ti != tj) also
// the transpose of the updated tile stored into (tj, ti), which then needs no
// update of its own.  Each thread's 4 consecutive rows of a column
// are 4 consecutive columns of the transposed tile: one 16-byte store, and
// the two row quads of a warp fill whole 32-byte sectors.
template <typename T, int TILE>
__device__ __forceinline__ bool floyd_tile_update_sym(const CUtensorMap *mapA, const CUtensorMap *mapB,
                                                      int z, T *mat, int64_t ld, int ti, int tj, int tk,
                                                      TmaSmem<T, typename FloydCfg<T, TILE>::TC> &sm,
                                                      int kvalid, int mvalid, int nvalid, bool transpose) {
  using C = typename FloydCfg<T, TILE>::C;
  using TC = typename FloydCfg<T, TILE>::TC;
  using V = typename Vec4<T>::type;
  T acc[C::TM][C::TN];
  const int64_t r0 = (int64_t)ti * TILE, c0 = (int64_t)tj * TILE;
  acc_load<T, C, true>(acc, mat + r0 * ld + c0, ld, 0, 0, 0, 0);
  const bool ok = tma_minplus_tile<T, TC, true>(mapA, tk * TILE, ti * TILE, z, mapB, tj * TILE, tk * TILE,
                                                z, kvalid, acc, sm, mvalid, nvalid);
  if (!ok) return false;
  acc_store<T, C, true>(acc, mat + r0 * ld + c0, ld, 0, 0, 0, 0);
  if (transpose && ti != tj) {
    const int tid = threadIdx.x, ty = tid / C::TX, tx = tid % C::TX;
#pragma unroll
    for (int gj = 0; gj < C::GN; gj++)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int c = tile_col<C>(tx, gj, q);   // row of the transposed tile
#pragma unroll
        for (int gi = 0; gi < C::GM; gi++) {
          V v;
          v.x = acc[4 * gi + 0][4 * gj + q];
          v.y = acc[4 * gi + 1][4 * gj + q];
          v.z = acc[4 * gi + 2][4 * gj + q];
          v.w = acc[4 * gi + 3][4 * gj + q];
          *reinterpret_cast<V *>(mat + (c0 + c) * ld + r0 + tile_row<C>(ty, gi, 0)) = v;
        }
      }
  }
  return true;
}

// Closes one padded matrix (nb x nb tiles, s real rows) of part z with the
// calling CTA.
template <typename T, int TILE>
__device__ bool floyd_close_cta(const CUtensorMap *mapA, const CUtensorMap *mapB, int z, T *mat,
                                int64_t ld, int nb, int s, TmaSmem<T, typename FloydCfg<T, TILE>::TC> &sm) {
  bool ok = true;
  for (int kb = 0; kb < nb && ok; kb++) {
    const int kv = min(TILE, s - kb * TILE);
    floyd_diag_close<T, TILE>(mat, ld, kb * TILE, sm.ring, kv);
    auto valid = [&](int t) { return min(TILE, s - t * TILE); };
    for (int j = 0; j < nb && ok; j++)
      if (j != kb) ok = floyd_tile_update<T, TILE>(mapA, mapB, z, mat, ld, kb, j, kb, sm, kv, kv, valid(j));
    for (int i = 0; i < nb && ok; i++)
      if (i != kb) ok = floyd_tile_update<T, TILE>(mapA, mapB, z, mat, ld, i, kb, kb, sm, kv, valid(i), kv);
    __syncthreads();
    for (int i = 0; i < nb && ok; i++) {
      if (i == kb) continue;
      for (int j = 0; j < nb && ok; j++)
        if (j != kb)
          ok = floyd_tile_update<T, TILE>(mapA, mapB, z, mat, ld, i, j, kb, sm, kv, valid(i), valid(j));
    }
    __syncthreads();
  }
  return ok;
}

}  // namespace fapb
