// The reference's CUDA kernel ABI (fap/kernel/cuda/cuda_kernel.h:21-42),
// implemented on top of the C ABI in fap_b200.h.  See fap_legacy_kernel.h.
#include <cuda_runtime.h>

#include <cmath>
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

void minplus_NVIDIA_path(float *mat1, float *mat2, int *mat2_path, float *res, int *res_path, int m,
                         int n, int k) {
  (void)mat2_path;
  (void)res_path;
  fap_ctx *c = legacy_ctx();
  if (!c) {
    report(FAP_ERR_CUDA, "minplus_NVIDIA_path");
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
    report(FAP_ERR_NOMEM, "minplus_NVIDIA_path");
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
  if (!report(fap_op_minplus(c, ints ? FAP_DTYPE_I32 : FAP_DTYPE_F32, m, n, k, A.p, k > 0 ? k : 1, B.p,
                             n, C.p, n),
              "minplus_NVIDIA_path"))
    return;
  if (ints) {
    std::vector<int32_t> t(cc);
    cudaMemcpy(t.data(), C.p, cc * 4, cudaMemcpyDeviceToHost);
    for (size_t i = 0; i < cc; i++) res[i] = (float)t[i];
  } else {
    cudaMemcpy(res, C.p, cc * 4, cudaMemcpyDeviceToHost);
  }
}
