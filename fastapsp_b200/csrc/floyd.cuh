// Stage 2: blocked Floyd-Warshall closure of each part's s x s matrix.
//
// Replaces floyd_GPU_Nvidia_path (fap/kernel/cuda/floyd.cu:284-348: one
// 32x32 tile per CTA, one element per thread, 2 launches per pivot) and the
// CPU floyd_CPU_path (fap/kernel/floyd.h:38-49).
//
// The matrix is padded to a multiple of TILE in both dimensions with the
// sentinel (padding never improves a real entry), so no tile needs bounds
// checks.  Per pivot block kb:
//   phase 1  close the diagonal tile D[kb][kb] with TILE sequential steps;
//            each thread keeps its TMxTN entries in registers and only the
//            pivot row/column of a step go through shared memory.
//   phase 2  row panel    D[kb][J] = min(D[kb][J], D*[kb][kb] (x) D[kb][J])
//            column panel D[I][kb] = min(D[I][kb], D[I][kb] (x) D*[kb][kb])
//            Because D*[kb][kb] is closed, one min-plus product gives what
//            TILE sequential pivot steps give.
//   phase 3  D[I][J] = min(D[I][J], D[I][kb] (x) D[kb][J])
// Phases 2 and 3 run on the register-tiled min-plus engine.
//
// Two drivers use the same phases:
//   floyd_part_kernel   one CTA closes one part's whole matrix (every part of
//                       a batch in one launch, no inter-CTA synchronisation);
//   floyd_*_phase       one launch per phase, tiles spread over the GPU (one
//                       matrix at a time: the plain form and fap_op_floyd).
#pragma once

#include "minplus_tile.cuh"

namespace fapb {

template <typename T, int TILE>
struct FloydCfg {
  using C = TileCfg<T, TILE, TILE, 16, 8, 8>;
  static constexpr int THREADS = C::THREADS;
  // phase-1 pivot row/column buffers (double-buffered) + min-plus staging
  static constexpr int P1_ELEMS = 4 * TILE;
  static constexpr int SMEM_ELEMS = (C::SMEM_ELEMS > P1_ELEMS ? C::SMEM_ELEMS : P1_ELEMS);
};

// Phase 1 on the tile at (r0, r0) of a padded matrix.  Block-wide; all
// threads of the CTA must call it.
template <typename T, int TILE>
__device__ __forceinline__ void floyd_diag_close(T *mat, int64_t ld, int r0, T *smem) {
  using C = typename FloydCfg<T, TILE>::C;
  const int tid = threadIdx.x, ty = tid / C::TX, tx = tid % C::TX;
  T acc[C::TM][C::TN];
  acc_load<T, C, true>(acc, mat, ld, r0, r0, 0, 0);
  for (int k = 0; k < TILE; k++) {
    T *rowbuf0 = smem + (k & 1) * TILE;
    T *colbuf0 = smem + 2 * TILE + (k & 1) * TILE;
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

// Phase 2/3 on one tile: D[ti][tj] = min(D[ti][tj], D[ti][tk] (x) D[tk][tj]).
// Tile coordinates are in units of TILE.  Block-wide.
template <typename T, int TILE>
__device__ __forceinline__ void floyd_tile_update(T *mat, int64_t ld, int ti, int tj, int tk,
                                                  T *smem) {
  using C = typename FloydCfg<T, TILE>::C;
  T acc[C::TM][C::TN];
  const int64_t r0 = (int64_t)ti * TILE, c0 = (int64_t)tj * TILE, k0 = (int64_t)tk * TILE;
  acc_load<T, C, true>(acc, mat + r0 * ld + c0, ld, 0, 0, 0, 0);
  minplus_tile<T, C, true, false>(mat + r0 * ld + k0, ld, mat + k0 * ld + c0, ld, 0, 0, TILE, TILE,
                           TILE, acc, smem);
  acc_store<T, C, true>(acc, mat + r0 * ld + c0, ld, 0, 0, 0, 0);
}

// Closes one padded matrix (nb x nb tiles) with the calling CTA.
template <typename T, int TILE>
__device__ void floyd_close_cta(T *mat, int64_t ld, int nb, T *smem) {
  for (int kb = 0; kb < nb; kb++) {
    floyd_diag_close<T, TILE>(mat, ld, kb * TILE, smem);
    for (int j = 0; j < nb; j++)
      if (j != kb) floyd_tile_update<T, TILE>(mat, ld, kb, j, kb, smem);
    for (int i = 0; i < nb; i++)
      if (i != kb) floyd_tile_update<T, TILE>(mat, ld, i, kb, kb, smem);
    __syncthreads();
    for (int i = 0; i < nb; i++) {
      if (i == kb) continue;
      for (int j = 0; j < nb; j++)
        if (j != kb) floyd_tile_update<T, TILE>(mat, ld, i, j, kb, smem);
    }
    __syncthreads();
  }
}

// ---- multi-launch form: one matrix, tiles across the GPU ----

template <typename T, int TILE>
__global__ void __launch_bounds__(FloydCfg<T, TILE>::THREADS)
    floyd_phase1_kernel(T *mat, int64_t ld, int kb) {
  extern __shared__ __align__(16) unsigned char fl_smem_raw[];
  T *smem = reinterpret_cast<T *>(fl_smem_raw);
  floyd_diag_close<T, TILE>(mat, ld, kb * TILE, smem);
}

// blockIdx.x in [0, 2*(nb-1)): first nb-1 are row-panel tiles, rest column.
template <typename T, int TILE>
__global__ void __launch_bounds__(FloydCfg<T, TILE>::THREADS)
    floyd_phase2_kernel(T *mat, int64_t ld, int kb, int nb) {
  extern __shared__ __align__(16) unsigned char fl_smem_raw[];
  T *smem = reinterpret_cast<T *>(fl_smem_raw);
  int t = blockIdx.x;
  if (t < nb - 1) {
    const int j = t < kb ? t : t + 1;
    floyd_tile_update<T, TILE>(mat, ld, kb, j, kb, smem);
  } else {
    t -= nb - 1;
    const int i = t < kb ? t : t + 1;
    floyd_tile_update<T, TILE>(mat, ld, i, kb, kb, smem);
  }
}

// blockIdx.x over the (nb-1)^2 remainder tiles.
template <typename T, int TILE>
__global__ void __launch_bounds__(FloydCfg<T, TILE>::THREADS)
    floyd_phase3_kernel(T *mat, int64_t ld, int kb, int nb) {
  extern __shared__ __align__(16) unsigned char fl_smem_raw[];
  T *smem = reinterpret_cast<T *>(fl_smem_raw);
  const int t = blockIdx.x;
  int i = t / (nb - 1), j = t % (nb - 1);
  i = i < kb ? i : i + 1;
  j = j < kb ? j : j + 1;
  floyd_tile_update<T, TILE>(mat, ld, i, j, kb, smem);
}

}  // namespace fapb
