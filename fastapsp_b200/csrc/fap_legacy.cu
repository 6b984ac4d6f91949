// The reference's CUDA kernel ABI (fap/kernel/cuda/cuda_kernel.h:21-42),
// implemented on top of the C ABI in fap_b200.h.  See fap_legacy_kernel.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "fap_b200.h"
#include "fap_legacy_kernel.h"

namespace {

thread_local int t_status = FAP_OK;
thread_local fap_ctx *t_ctx = nullptr;

fap_ctx *legacy_ctx() {
  if (!t_ctx) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
    if (fap_ctx_create(dev, &t_ctx) != FAP_OK) t_ctx = nullptr;
  }
  return t_ctx;
}

bool report(int rc, const char *where) {
  t_status = rc;
  if (rc != FAP_OK) std::fprintf(stderr, "fap legacy %s: %s\n", where, fap_last_error());
  return rc == FAP_OK;
}

bool all_integral(const float *v, size_t count) {
  for (size_t i = 0; i < count; i++)
    if (v[i] != std::floor(v[i]) || v[i] < 0.0f || v[i] > 2e8f) return false;
  return true;
}

// Device buffer that frees itself.
struct Dev {
  void *p = nullptr;
  bool alloc(size_t bytes) { return cudaMalloc(&p, bytes ? bytes : 4) == cudaSuccess; }
  ~Dev() {
    if (p) cudaFree(p);
  }
};

}  // namespace

extern "C" int fap_legacy_last_status(void) { return t_status; }

void handle_boundry_Nvidia_GPU(float *subGraph, int vertexs, int edges, int bdy_num, int *adj_size,
                               int *row_offset, int *col_val, float *weight, int *st2ed,
                               int offset) {
  (void)adj_size;
  (void)edges;
  fap_ctx *c = legacy_ctx();
  if (!c) {
    report(FAP_ERR_CUDA, "handle_boundry_Nvidia_GPU");
    return;
  }
  if (bdy_num <= 0) {
    t_status = FAP_OK;
    return;
  }
  fap_dgraph *g = nullptr;
  const int64_t m = row_offset[vertexs];
  if (!report(fap_graph_create(c, vertexs, m, row_offset, col_val, weight, FAP_DTYPE_AUTO, &g),
              "handle_boundry_Nvidia_GPU"))
    return;
  report(fap_graph_sssp_rows(g, st2ed + offset, bdy_num, subGraph), "handle_boundry_Nvidia_GPU");
  fap_graph_destroy(g);
}

void floyd_GPU_Nvidia_path(int num_node, float *arc, int *path) {
  (void)path;
  fap_ctx *c = legacy_ctx();
  if (!c) {
    report(FAP_ERR_CUDA, "floyd_GPU_Nvidia_path");
    return;
  }
  if (num_node <= 0) {
    t_status = FAP_OK;
    return;
  }
  const size_t cnt = (size_t)num_node * num_node;
  const bool ints = all_integral(arc, cnt);
  Dev d;
  if (!d.alloc(cnt * 4)) {
    report(FAP_ERR_NOMEM, "floyd_GPU_Nvidia_path");
    return;
  }
  std::vector<int32_t> tmp;
  if (ints) {
    tmp.resize(cnt);
    for (size_t i = 0; i < cnt; i++) tmp[i] = (int32_t)arc[i];
    cudaMemcpy(d.p, tmp.data(), cnt * 4, cudaMemcpyHostToDevice);
  } else {
    cudaMemcpy(d.p, arc, cnt * 4, cudaMemcpyHostToDevice);
  }
  if (!report(fap_op_floyd(c, ints ? FAP_DTYPE_I32 : FAP_DTYPE_F32, num_node, d.p, num_node),
              "floyd_GPU_Nvidia_path"))
    return;
  if (ints) {
    cudaMemcpy(tmp.data(), d.p, cnt * 4, cudaMemcpyDeviceToHost);
    for (size_t i = 0; i < cnt; i++) arc[i] = (float)tmp[i];
  } else {
    cudaMemcpy(arc, d.p, cnt * 4, cudaMemcpyDeviceToHost);
  }
}

namespace {

// res[m x n] = min(1e8, mat1[m x k] (x) mat2[k x n]) on the GPU for host
// row-major matrices, in int32 when every input is an integral distance,
// else in float32.  res may be one of the inputs: both are uploaded before
// it is written.
void host_minplus(const float *mat1, const float *mat2, float *res, int m, int n, int k, const char *where) {
  fap_ctx *c = legacy_ctx();
  if (!c) {
    report(FAP_ERR_CUDA, where);
    return;
  }
  if (m <= 0 || n <= 0) {
    t_status = FAP_OK;
    return;
  }
  const size_t ca = (size_t)m * (k > 0 ? k : 0), cb = (size_t)(k > 0 ? k : 0) * n, cc = (size_t)m * n;
  const bool ints = all_integral(mat1, ca) && all_integral(mat2, cb);
  Dev A, B, C;
  if (!A.alloc(ca * 4) || !B.alloc(cb * 4) || !C.alloc(cc * 4)) {
    report(FAP_ERR_NOMEM, where);
    return;
  }
  if (ints) {
    std::vector<int32_t> t(ca > cb ? ca : cb);
    for (size_t i = 0; i < ca; i++) t[i] = (int32_t)mat1[i];
    cudaMemcpy(A.p, t.data(), ca * 4, cudaMemcpyHostToDevice);
    for (size_t i = 0; i < cb; i++) t[i] = (int32_t)mat2[i];
    cudaMemcpy(B.p, t.data(), cb * 4, cudaMemcpyHostToDevice);
  } else {
    cudaMemcpy(A.p, mat1, ca * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(B.p, mat2, cb * 4, cudaMemcpyHostToDevice);
  }
  if (!report(fap_op_minplus(c, ints ? FAP_DTYPE_I32 : FAP_DTYPE_F32, m, n, k, A.p, k > 0 ? k : 1, B.p, n,
                             C.p, n),
              where))
    return;
  if (ints) {
    std::vector<int32_t> t(cc);
    cudaMemcpy(t.data(), C.p, cc * 4, cudaMemcpyDeviceToHost);
    for (size_t i = 0; i < cc; i++) res[i] = (float)t[i];
  } else {
    cudaMemcpy(res, C.p, cc * 4, cudaMemcpyDeviceToHost);
  }
}

}  // namespace

void minplus_NVIDIA_path(float *mat1, float *mat2, int *mat2_path, float *res, int *res_path, int m,
                         int n, int k) {
  (void)mat2_path;
  (void)res_path;
  host_minplus(mat1, mat2, res, m, n, k, "minplus_NVIDIA_path");
}

void minplus_NVIDIA_GPU(float *mat1, float *mat2, float *res, int M, int N, int K) {
  host_minplus(mat1, mat2, res, M, N, K, "minplus_NVIDIA_GPU");
}

void floyd_NVIDIA_GPU(int num_node, float *arc) { floyd_GPU_Nvidia_path(num_node, arc, nullptr); }

// Column panel of a blocked Floyd (fap/kernel/floyd.h:106-115): the new
// panel from the old one and the closed diagonal block, computed out of
// place as the reference's CUDA kernel intends.
void floyd_path_A_Nvidia(float *A, int *A_path, const int row, const int col, float *diag, int *diag_path) {
  (void)A_path;
  (void)diag_path;
  host_minplus(A, diag, A, row, col, col, "floyd_path_A_Nvidia");
}

// Row panel of a blocked Floyd (fap/kernel/floyd.h:118-127).
void floyd_path_B_Nvidia(float *B, int *B_path, const int row, const int col, float *diag, int *diag_path) {
  (void)B_path;
  (void)diag_path;
  host_minplus(diag, B, B, row, col, row, "floyd_path_B_Nvidia");
}

// res = min(res, mat1 (x) mat2) (fap/kernel/floyd.h:130-139) as one product
// from the sentinel: [mat1 | E] (x) [mat2 ; res], E the min-plus identity
// (0 on the diagonal, 1e8 elsewhere), so that E (x) res = res.
void floyd_min_plus_Nvidia(float *mat1, float *mat2, int *mat2_path, float *res, int *res_path, int m, int n,
                           int k) {
  (void)mat2_path;
  (void)res_path;
  if (m <= 0 || n <= 0) {
    t_status = FAP_OK;
    return;
  }
  const int64_t kk = k > 0 ? k : 0;
  const int64_t k2 = kk + m;
  if (k2 > INT32_MAX) {
    report(FAP_ERR_RANGE, "floyd_min_plus_Nvidia");
    return;
  }
  std::vector<float> a2((size_t)m * (size_t)k2, 1e8f), b2((size_t)k2 * (size_t)n);
  for (int64_t i = 0; i < m; i++) {
    float *row = a2.data() + i * k2;
    for (int64_t j = 0; j < kk; j++) row[j] = mat1[i * kk + j];
    row[kk + i] = 0.0f;
  }
  std::copy(mat2, mat2 + kk * n, b2.begin());
  std::copy(res, res + (int64_t)m * n, b2.begin() + kk * n);
  host_minplus(a2.data(), b2.data(), res, m, n, (int)k2, "floyd_min_plus_Nvidia");
}
