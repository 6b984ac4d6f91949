/*
 * fap_oracle.c -- CPU restatement of the reference's per-subgraph solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product
 * and the "port" CPU baseline; the product never links, loads or calls it.
 *
 * Every routine restates one reference routine, in float arithmetic with the
 * reference's sentinel and strict comparisons, so that on integer weights the
 * outputs are the reference's outputs bit for bit.  The restatement is pinned
 * against the reference itself (oracle/_ref/fap_ref, built from the reference
 * sources by oracle/Makefile) and against the committed fixtures in
 * tests/golden/.
 *
 * Citations are to the reference project (Liu-xiandong/FastAPSP).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define FO_MAXVALUE 1e8f /* fap/utils/parameter.h:26 */

/* ---- binary min-heap of (dist, vertex), lexicographic like
 *      std::priority_queue<std::pair<float,int>, ..., std::greater<>> ---- */
typedef struct {
  float d;
  int v;
} fo_item;

static int fo_less(fo_item a, fo_item b) {
  return a.d < b.d || (a.d == b.d && a.v < b.v);
}

typedef struct {
  fo_item *a;
  int64_t n, cap;
} fo_heap;

static void fo_push(fo_heap *h, fo_item x) {
  if (h->n == h->cap) {
    h->cap = h->cap ? h->cap * 2 : 1024;
    h->a = (fo_item *)realloc(h->a, (size_t)h->cap * sizeof(fo_item));
  }
  int64_t i = h->n++;
  while (i > 0) {
    int64_t p = (i - 1) / 2;
    if (!fo_less(x, h->a[p])) break;
    h->a[i] = h->a[p];
    i = p;
  }
  h->a[i] = x;
}

static fo_item fo_pop(fo_heap *h) {
  fo_item top = h->a[0];
  fo_item last = h->a[--h->n];
  int64_t i = 0;
  for (;;) {
    int64_t l = 2 * i + 1, r = l + 1, m = i;
    fo_item best = last;
    if (l < h->n && fo_less(h->a[l], best)) { m = l; best = h->a[l]; }
    if (r < h->n && fo_less(h->a[r], best)) { m = r; }
    if (m == i) break;
    h->a[i] = h->a[m];
    i = m;
  }
  if (h->n > 0) h->a[i] = last;
  return top;
}

/* Single-source Dijkstra with predecessors.
 * Follows fap/kernel/batch_sssp.h:79-114 (dijkstra_path): sentinel fill,
 * lazy-deletion heap, strict '>' relaxation, path[u] = u at the source. */
void fo_dijkstra_path(int src, int n, const int *row_offset, const int *col,
                      const float *w, float *dist, int *path) {
  fo_heap h = {0, 0, 0};
  unsigned char *done = (unsigned char *)calloc((size_t)n, 1);
  for (int i = 0; i < n; i++) {
    dist[i] = FO_MAXVALUE;
    if (path) path[i] = -1;
  }
  dist[src] = 0.0f;
  if (path) path[src] = src;
  fo_item s0 = {0.0f, src};
  fo_push(&h, s0);
  while (h.n > 0) {
    fo_item x = fo_pop(&h);
    int u = x.v;
    float du = x.d;
    if (done[u]) continue;
    done[u] = 1;
    for (int e = row_offset[u]; e < row_offset[u + 1]; e++) {
      int v = col[e];
      float nd = du + w[e];
      if (dist[v] > nd) {
        fo_item y = {nd, v};
        fo_push(&h, y);
        dist[v] = nd;
        if (path) path[v] = u;
      }
    }
  }
  free(done);
  free(h.a);
}

/* Stage 1: SSSP from every boundary vertex of the part.
 * Follows fap/kernel/batch_sssp.h:232-277 (handle_boundry_path,
 * batched_sssp_path): sources are st2ed[start .. start+bdy-1]; row i of the
 * output block is the distance row of source i, columns are original ids.
 * OpenMP over sources, as the reference. */
void fo_boundary_sssp(int n, const int *row_offset, const int *col,
                      const float *w, const int *st2ed, int start, int bdy,
                      float *block, int *block_path) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < bdy; i++) {
    fo_dijkstra_path(st2ed[start + i], n, row_offset, col, w,
                     block + (int64_t)i * n,
                     block_path ? block_path + (int64_t)i * n : NULL);
  }
}

/* Stage 2.1: build the s x s Floyd matrix.
 * Follows fap/utils/util_Myalgorithm.h:30-73 (MysubMatBuild_path): intra-part
 * CSR edges in CSR order (a later duplicate overwrites an earlier one), then
 * the boundary rows copied from the SSSP rows, then a zero diagonal.  The
 * caller pre-fills mat with the sentinel (fap/fap.cpp:111-112). */
void fo_build_submat(int n, const int *row_offset, const int *col,
                     const float *w, const int *graph_id, const int *st2ed,
                     const int *ed2st, int start, int s, int bdy,
                     const float *block, float *mat) {
  for (int i = 0; i < s; i++) {
    int ver = st2ed[start + i];
    for (int e = row_offset[ver]; e < row_offset[ver + 1]; e++) {
      int nb = col[e];
      if (graph_id[ver] != graph_id[nb]) continue;
      int idx = ed2st[nb] - start;
      mat[(int64_t)i * s + idx] = w[e];
    }
  }
  for (int i = 0; i < bdy; i++)
    for (int j = 0; j < s; j++)
      mat[(int64_t)i * s + j] = block[(int64_t)i * n + st2ed[start + j]];
  for (int i = 0; i < s; i++) mat[(int64_t)i * s + i] = 0.0f;
}

/* Stage 2.2: Floyd-Warshall, in place.
 * Follows fap/kernel/floyd.h:38-49 (floyd_CPU_path): k outermost, strict '>'. */
void fo_floyd(int s, float *mat) {
  for (int k = 0; k < s; k++) {
    const float *rk = mat + (int64_t)k * s;
    for (int i = 0; i < s; i++) {
      float *ri = mat + (int64_t)i * s;
      float dik = ri[k];
      for (int j = 0; j < s; j++) {
        float c = dik + rk[j];
        if (ri[j] > c) ri[j] = c;
      }
    }
  }
}

/* Stage 3: min-plus product R[i][j] = min_k A[i][k] + S[k][j], starting from
 * the sentinel.  Follows fap/kernel/minplus.h:51-65
 * (min_plus_path_CPU_advanced) with A = F[bdy+i][0..bdy-1]
 * (fap/utils/util_Myalgorithm.h:88-95, MyMat1Build) and S = the block's
 * boundary rows (fap/fap.cpp:143-149).  Rows are independent; OpenMP over
 * rows (the reference runs them serially; the result is the same). */
void fo_minplus(int n, int s, int bdy, const float *mat, float *block) {
  const int inner = s - bdy;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < inner; i++) {
    const float *a = mat + (int64_t)(bdy + i) * s;
    float *r = block + (int64_t)(bdy + i) * n;
    for (int j = 0; j < n; j++) r[j] = FO_MAXVALUE;
    for (int k = 0; k < bdy; k++) {
      const float ak = a[k];
      const float *sk = block + (int64_t)k * n;
      for (int j = 0; j < n; j++) {
        float c = ak + sk[j];
        if (r[j] > c) r[j] = c;
      }
    }
  }
}

/* Stage 3.3: scatter the closed Floyd matrix into the block.
 * Follows fap/utils/util_Myalgorithm.h:75-86 (MysubMatDecode_path). */
void fo_decode(int n, const int *st2ed, int start, int s, const float *mat,
               float *block) {
  for (int i = 0; i < s; i++)
    for (int j = 0; j < s; j++)
      block[(int64_t)i * n + st2ed[start + j]] = mat[(int64_t)i * s + j];
}

/* One part, end to end.  Follows fap/fap.cpp:92-181 (fapGraph::run).
 * block: s x n floats; row r is vertex st2ed[start + r]. */
int fo_run_part(int n, const int *row_offset, const int *col, const float *w,
                const int *graph_id, const int *st2ed, const int *ed2st,
                int start, int s, int bdy, float *block) {
  float *mat = (float *)malloc((size_t)s * (size_t)s * sizeof(float));
  if (!mat) return -1;
  for (int64_t i = 0; i < (int64_t)s * s; i++) mat[i] = FO_MAXVALUE;
  fo_boundary_sssp(n, row_offset, col, w, st2ed, start, bdy, block, NULL);
  fo_build_submat(n, row_offset, col, w, graph_id, st2ed, ed2st, start, s,
                  bdy, block, mat);
  fo_floyd(s, mat);
  fo_minplus(n, s, bdy, mat, block);
  fo_decode(n, st2ed, start, s, mat, block);
  free(mat);
  return 0;
}

/* ---- predecessor-carrying kernels of the reference's kernel header ---- */

/* floyd_CPU_path, fap/kernel/floyd.h:38-49: k-i-j, strict >, path[i][j] =
 * path[k][j] on every improvement. */
void fo_floyd_path(int s, float *mat, int *path) {
  for (int64_t k = 0; k < s; k++)
    for (int64_t i = 0; i < s; i++)
      for (int64_t j = 0; j < s; j++) {
        const float c = mat[i * s + k] + mat[k * s + j];
        if (mat[i * s + j] > c) {
          mat[i * s + j] = c;
          path[i * s + j] = path[k * s + j];
        }
      }
}

/* min_plus_path_CPU_advanced, fap/kernel/minplus.h:51-65 (c0 == NULL: start
 * from the sentinel with path -1), and floyd_min_plus_CPU, fap/kernel/
 * floyd.h:86-102 (c0/p0 given: start from them): for k ascending, a strictly
 * smaller mat1[i][k] + mat2[k][j] replaces the value and takes
 * mat2_path[k][j].  Out of place: res/path must not alias the inputs. */
void fo_minplus_path(int M, int N, int K, const float *mat1, const float *mat2,
                     const int *mat2_path, const float *c0, const int *p0,
                     float *res, int *path) {
  for (int64_t i = 0; i < M; i++)
    for (int64_t j = 0; j < N; j++) {
      float v = c0 ? c0[i * N + j] : FO_MAXVALUE;
      int p = c0 ? p0[i * N + j] : -1;
      for (int64_t k = 0; k < K; k++) {
        const float c = mat1[i * K + k] + mat2[k * N + j];
        if (v > c) {
          v = c;
          p = mat2_path[k * N + j];
        }
      }
      res[i * N + j] = v;
      path[i * N + j] = p;
    }
}

/* floyd_path_A_CPU, fap/kernel/floyd.h:68-84, in place as the reference
 * does it (entries of row i left of j are already updated when j runs). */
void fo_floyd_path_A(float *A, int *A_path, int row, int col, const float *diag,
                     const int *diag_path) {
  for (int64_t i = 0; i < row; i++)
    for (int64_t j = 0; j < col; j++) {
      float v = A[i * col + j];
      int p = A_path[i * col + j];
      for (int64_t k = 0; k < col; k++) {
        const float c = A[i * col + k] + diag[k * col + j];
        if (v > c) {
          v = c;
          p = diag_path[k * col + j];
        }
      }
      A[i * col + j] = v;
      A_path[i * col + j] = p;
    }
}

/* floyd_path_B_CPU, fap/kernel/floyd.h:51-66, in place as the reference
 * does it (rows above i are already updated when row i runs). */
void fo_floyd_path_B(float *B, int *B_path, int row, int col, const float *diag,
                     const int *diag_path) {
  (void)diag_path;
  for (int64_t i = 0; i < row; i++)
    for (int64_t j = 0; j < col; j++) {
      float v = B[i * col + j];
      int p = B_path[i * col + j];
      for (int64_t k = 0; k < row; k++) {
        const float c = diag[i * row + k] + B[k * col + j];
        if (v > c) {
          v = c;
          p = B_path[k * col + j];
        }
      }
      B[i * col + j] = v;
      B_path[i * col + j] = p;
    }
}
