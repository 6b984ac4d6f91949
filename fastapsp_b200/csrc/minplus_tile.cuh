// Register-tiled min-plus tile engine shared by the min-plus merge and the
// Floyd-Warshall panel/remainder phases.
//
//   acc[i][j] = min(acc[i][j], min_k A[i][k] + B[k][j])
//
// over a BM x BN output tile, streaming K in chunks of BK through shared
// memory with a register prefetch of the next chunk (double buffering).
// Each thread owns TM x TN outputs split into 4-wide groups spaced BM/GM
// rows and BN/GN columns apart, so that every shared-memory read is one
// conflict-free 128-bit load and every relaxation is one DPX __viaddmin_s32
// (int32) or FADD+FMNMX (float).
//
// Out-of-range rows, columns and k read the sentinel, which never improves a
// result (INF + x >= INF >= acc).
#pragma once

#include "fap_common.cuh"

namespace fapb {

template <typename T, int BM_, int BN_, int BK_, int TM_, int TN_>
struct TileCfg {
  static constexpr int BM = BM_, BN = BN_, BK = BK_, TM = TM_, TN = TN_;
  static constexpr int GM = TM / 4, GN = TN / 4;   // 4-wide groups per thread
  static constexpr int TY = BM / TM, TX = BN / TN; // thread grid
  static constexpr int THREADS = TY * TX;
  static constexpr int AP = BM + 4;                // padded As row (k-major)
  static constexpr int A_ELEMS = BK * AP;
  static constexpr int B_ELEMS = BK * BN;
  static constexpr int SMEM_ELEMS = 2 * (A_ELEMS + B_ELEMS);  // two stages
  static constexpr int A_PER_THREAD = BM * BK / THREADS;
  static constexpr int B_PER_THREAD = BK * BN / THREADS;
  static_assert(TM % 4 == 0 && TN % 4 == 0, "4-wide groups");
  static_assert((BM * BK) % THREADS == 0 && (BK * BN) % THREADS == 0, "even loads");
  static_assert(B_PER_THREAD % 4 == 0, "vector B loads");
};

// Row/column owned by thread (ty, tx) for group g, lane l.
template <class C>
__device__ __forceinline__ int tile_row(int ty, int g, int l) { return g * (C::BM / C::GM) + ty * 4 + l; }
template <class C>
__device__ __forceinline__ int tile_col(int tx, int g, int l) { return g * (C::BN / C::GN) + tx * 4 + l; }

// A/B chunk loader with a register stage.  Global A is row-major (lda), B is
// row-major (ldb).  VEC_B: B rows are 16-byte aligned and n-range checks are
// made per 4-vector (the caller guarantees ldb % 4 == 0, B 16B-aligned and
// that columns beyond N up to the next multiple of 4 exist and may be read).
// NC: the sources are read-only for the whole kernel, so the non-coherent
// read-only path may be used; kernels that update A/B in place pass false.
template <typename T, class C, bool VEC_B, bool NC>
struct ChunkLoader {
  __device__ __forceinline__ static T ldv(const T *p) { return NC ? __ldg(p) : *p; }
  __device__ __forceinline__ static int4 ldv4(const int4 *p) { return NC ? __ldg(p) : *p; }

  T ra[C::A_PER_THREAD];
  T rb[C::B_PER_THREAD];

  __device__ __forceinline__ void load(const T *A, int64_t lda,
                                       const T *B, int64_t ldb, int m0, int n0,
                                       int k0, int M, int N, int K, int tid) {
    const T inf = Dist<T>::inf();
#pragma unroll
    for (int r = 0; r < C::A_PER_THREAD; r++) {
      int idx = tid + r * C::THREADS;
      int i = idx / C::BK, k = idx % C::BK;
      int gi = m0 + i, gk = k0 + k;
      ra[r] = (gi < M && gk < K) ? ldv(A + (int64_t)gi * lda + gk) : inf;
    }
    if (VEC_B) {
#pragma unroll
      for (int r = 0; r < C::B_PER_THREAD / 4; r++) {
        int idx = tid + r * C::THREADS;  // 4-vector index
        int k = idx / (C::BN / 4), j4 = (idx % (C::BN / 4)) * 4;
        int gk = k0 + k, gj = n0 + j4;
        if (gk < K && gj < N) {
          const int4 v = ldv4(reinterpret_cast<const int4 *>(B + (int64_t)gk * ldb + gj));
          rb[4 * r + 0] = *reinterpret_cast<const T *>(&v.x);
          rb[4 * r + 1] = *reinterpret_cast<const T *>(&v.y);
          rb[4 * r + 2] = *reinterpret_cast<const T *>(&v.z);
          rb[4 * r + 3] = *reinterpret_cast<const T *>(&v.w);
        } else {
          rb[4 * r + 0] = rb[4 * r + 1] = rb[4 * r + 2] = rb[4 * r + 3] = inf;
        }
      }
    } else {
#pragma unroll
      for (int r = 0; r < C::B_PER_THREAD; r++) {
        int idx = tid + r * C::THREADS;
        int k = idx / C::BN, j = idx % C::BN;
        int gk = k0 + k, gj = n0 + j;
        rb[r] = (gk < K && gj < N) ? ldv(B + (int64_t)gk * ldb + gj) : inf;
      }
    }
  }

  __device__ __forceinline__ void store(T *As, T *Bs, int tid) const {
#pragma unroll
    for (int r = 0; r < C::A_PER_THREAD; r++) {
      int idx = tid + r * C::THREADS;
      int i = idx / C::BK, k = idx % C::BK;
      As[k * C::AP + i] = ra[r];
    }
    if (VEC_B) {
#pragma unroll
      for (int r = 0; r < C::B_PER_THREAD / 4; r++) {
        int idx = tid + r * C::THREADS;
        int k = idx / (C::BN / 4), j4 = (idx % (C::BN / 4)) * 4;
        T *dst = Bs + k * C::BN + j4;
        dst[0] = rb[4 * r + 0];
        dst[1] = rb[4 * r + 1];
        dst[2] = rb[4 * r + 2];
        dst[3] = rb[4 * r + 3];
      }
    } else {
#pragma unroll
      for (int r = 0; r < C::B_PER_THREAD; r++) {
        int idx = tid + r * C::THREADS;
        int k = idx / C::BN, j = idx % C::BN;
        Bs[k * C::BN + j] = rb[r];
      }
    }
  }
};

template <typename T>
struct Vec4;
template <>
struct Vec4<int32_t> { using type = int4; };
template <>
struct Vec4<float> { using type = float4; };

// One k of a staged chunk (acc <- min(acc, As[k][.] + Bs[k][.])).
template <typename T, class C>
__device__ __forceinline__ void mma_k_step(const T *As, const T *Bs, T (&acc)[C::TM][C::TN], int ty, int tx,
                                           int k) {
  using V = typename Vec4<T>::type;
  T a[C::TM], b[C::TN];
#pragma unroll
  for (int g = 0; g < C::GM; g++) {
    V v = *reinterpret_cast<const V *>(As + k * C::AP + g * (C::BM / C::GM) + ty * 4);
    a[4 * g + 0] = v.x; a[4 * g + 1] = v.y; a[4 * g + 2] = v.z; a[4 * g + 3] = v.w;
  }
#pragma unroll
  for (int g = 0; g < C::GN; g++) {
    V v = *reinterpret_cast<const V *>(Bs + k * C::BN + g * (C::BN / C::GN) + tx * 4);
    b[4 * g + 0] = v.x; b[4 * g + 1] = v.y; b[4 * g + 2] = v.z; b[4 * g + 3] = v.w;
  }
#pragma unroll
  for (int i = 0; i < C::TM; i++)
#pragma unroll
    for (int j = 0; j < C::TN; j++) acc[i][j] = Dist<T>::relax(a[i], b[j], acc[i][j]);
}

// acc <- min(acc, As (x) Bs) over kcount k's of one staged chunk (a full
// chunk runs with k unrolled, a partial one with the rolled loop).
template <typename T, class C>
__device__ __forceinline__ void mma_chunk(const T *As, const T *Bs, T (&acc)[C::TM][C::TN],
                                          int ty, int tx, int kcount) {
  if (kcount == C::BK) {
#pragma unroll
    for (int k = 0; k < C::BK; k++) mma_k_step<T, C>(As, Bs, acc, ty, tx, k);
  } else {
#pragma unroll 1
    for (int k = 0; k < kcount; k++) mma_k_step<T, C>(As, Bs, acc, ty, tx, k);
  }
}

// Full-K pipeline: acc <- min(acc, A[m0:m0+BM, 0:K] (x) B[0:K, n0:n0+BN]).
// smem must hold C::SMEM_ELEMS elements.  Ends with a __syncthreads, so the
// caller may overwrite the A/B sources afterwards (in-place Floyd panels).
template <typename T, class C, bool VEC_B, bool NC>
__device__ __forceinline__ void minplus_tile(const T *A, int64_t lda,
                                             const T *B, int64_t ldb, int m0,
                                             int n0, int M, int N, int K,
                                             T (&acc)[C::TM][C::TN], T *smem) {
  const int tid = threadIdx.x;
  const int ty = tid / C::TX, tx = tid % C::TX;
  T *const As0 = smem;
  T *const Bs0 = smem + 2 * C::A_ELEMS;
  ChunkLoader<T, C, VEC_B, NC> ld;
  const int nchunks = (int)ceil_div(K, C::BK);
  if (nchunks == 0) return;
  ld.load(A, lda, B, ldb, m0, n0, 0, M, N, K, tid);
  ld.store(As0, Bs0, tid);
  __syncthreads();
  for (int c = 0; c < nchunks; c++) {
    const int cur = c & 1;
    if (c + 1 < nchunks) ld.load(A, lda, B, ldb, m0, n0, (c + 1) * C::BK, M, N, K, tid);
    const int kc = min(C::BK, K - c * C::BK);
    mma_chunk<T, C>(As0 + cur * C::A_ELEMS, Bs0 + cur * C::B_ELEMS, acc, ty, tx, kc);
    if (c + 1 < nchunks) ld.store(As0 + (cur ^ 1) * C::A_ELEMS, Bs0 + (cur ^ 1) * C::B_ELEMS, tid);
    __syncthreads();
  }
}

template <typename T, class C>
__device__ __forceinline__ void acc_fill(T (&acc)[C::TM][C::TN], T v) {
#pragma unroll
  for (int i = 0; i < C::TM; i++)
#pragma unroll
    for (int j = 0; j < C::TN; j++) acc[i][j] = v;
}

// Load / store the thread's outputs of a tile at (m0, n0) of a row-major
// matrix, rows < M and columns < N only.  FULL: the whole tile is in range and
// ld % 4 == 0 (vector accesses).
template <typename T, class C, bool FULL>
__device__ __forceinline__ void acc_load(T (&acc)[C::TM][C::TN], const T *P, int64_t ld, int m0,
                                         int n0, int M, int N) {
  using V = typename Vec4<T>::type;
  const int tid = threadIdx.x, ty = tid / C::TX, tx = tid % C::TX;
#pragma unroll
  for (int gi = 0; gi < C::GM; gi++)
#pragma unroll
    for (int l = 0; l < 4; l++) {
      const int r = m0 + tile_row<C>(ty, gi, l);
#pragma unroll
      for (int gj = 0; gj < C::GN; gj++) {
        const int c0 = n0 + tile_col<C>(tx, gj, 0);
        if (FULL) {
          // L2 only (ld.global.cg): the tile may have been written by another
          // SM earlier in the same launch (the Floyd work queue), and this
          // SM's L1 could still hold an older copy of it
          V v = __ldcg(reinterpret_cast<const V *>(P + (int64_t)r * ld + c0));
          acc[4 * gi + l][4 * gj + 0] = v.x;
          acc[4 * gi + l][4 * gj + 1] = v.y;
          acc[4 * gi + l][4 * gj + 2] = v.z;
          acc[4 * gi + l][4 * gj + 3] = v.w;
        } else {
#pragma unroll
          for (int q = 0; q < 4; q++)
            acc[4 * gi + l][4 * gj + q] =
                (r < M && c0 + q < N) ? __ldcg(P + (int64_t)r * ld + c0 + q) : Dist<T>::inf();
        }
      }
    }
}

template <typename T, class C, bool FULL>
__device__ __forceinline__ void acc_store(const T (&acc)[C::TM][C::TN], T *P, int64_t ld, int m0,
                                          int n0, int M, int N) {
  using V = typename Vec4<T>::type;
  const int tid = threadIdx.x, ty = tid / C::TX, tx = tid % C::TX;
#pragma unroll
  for (int gi = 0; gi < C::GM; gi++)
#pragma unroll
    for (int l = 0; l < 4; l++) {
      const int r = m0 + tile_row<C>(ty, gi, l);
#pragma unroll
      for (int gj = 0; gj < C::GN; gj++) {
        const int c0 = n0 + tile_col<C>(tx, gj, 0);
        if (FULL) {
          V v;
          v.x = acc[4 * gi + l][4 * gj + 0];
          v.y = acc[4 * gi + l][4 * gj + 1];
          v.z = acc[4 * gi + l][4 * gj + 2];
          v.w = acc[4 * gi + l][4 * gj + 3];
          *reinterpret_cast<V *>(P + (int64_t)r * ld + c0) = v;
        } else if (r < M) {
#pragma unroll
          for (int q = 0; q < 4; q++)
            if (c0 + q < N) P[(int64_t)r * ld + c0 + q] = acc[4 * gi + l][4 * gj + q];
        }
      }
    }
}

}  // namespace fapb
