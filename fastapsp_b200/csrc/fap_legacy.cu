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

// ---------------------------------------------------------------------------
// Predecessor-carrying forms.  They compute in float32 on the GPU with the
// reference CPU path's own arithmetic: one IEEE single-precision add and a
// strict comparison per candidate, candidates in the reference's order, so
// distances and predecessors are bit-identical to it (also on ties).
// ---------------------------------------------------------------------------
constexpr int kPT = 32;   // output tile kPT x kPT; block kPT x 8 threads, 4 rows each

// C[i][j], P[i][j]: the first strict minimum, in the order "start" then
// k = 0, 1, ..., k-1, of the candidates A[i][k] + B[k][j], where a candidate
// that wins brings the predecessor Bp[k][j].  start = (C0[i][j], P0[i][j])
// when C0 is given (res = min(res, A (x) B), fap/kernel/floyd.h:86-102 and
// the panels :51-84), else (1e8, -1) (fap/kernel/minplus.h:51-65).
__global__ void __launch_bounds__(kPT * 8)
legacy_minplus_path_kernel(const float *__restrict__ A, const float *__restrict__ B,
                           const int *__restrict__ Bp, const float *__restrict__ C0,
                           const int *__restrict__ P0, float *__restrict__ C, int *__restrict__ P,
                           int m, int n, int k) {
  __shared__ float As[kPT][kPT + 1];
  __shared__ float Bs[kPT][kPT];
  __shared__ int Ps[kPT][kPT];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int64_t i0 = (int64_t)blockIdx.y * kPT;
  const int64_t j = (int64_t)blockIdx.x * kPT + tx;
  float v[4];
  int p[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int64_t i = i0 + ty + 8 * q;
    v[q] = 1e8f;
    p[q] = -1;
    if (C0 != nullptr && i < m && j < n) {
      v[q] = C0[i * n + j];
      p[q] = P0[i * n + j];
    }
  }
  for (int k0 = 0; k0 < k; k0 += kPT) {
    const int kc = min(kPT, k - k0);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int r = ty + 8 * q;
      const int64_t i = i0 + r;
      As[r][tx] = (i < m && tx < kc) ? A[i * k + k0 + tx] : 0.0f;
      const bool ok = r < kc && j < n;
      Bs[r][tx] = ok ? B[(int64_t)(k0 + r) * n + j] : 0.0f;
      Ps[r][tx] = ok ? Bp[(int64_t)(k0 + r) * n + j] : -1;
    }
    __syncthreads();
    for (int t = 0; t < kc; t++) {
      const float b = Bs[t][tx];
      const int bp = Ps[t][tx];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const float c = As[ty + 8 * q][t] + b;
        if (v[q] > c) {
          v[q] = c;
          p[q] = bp;
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int64_t i = i0 + ty + 8 * q;
    if (i < m && j < n) {
      C[i * n + j] = v[q];
      P[i * n + j] = p[q];
    }
  }
}

// Pivot k of Floyd-Warshall with predecessors (fap/kernel/floyd.h:38-49):
// d[i][j] = d[i][k] + d[k][j], path[i][j] = path[k][j] where that is
// strictly shorter.  With every entry non-negative, row k and column k do
// not change during pivot k (that needs d[k][k] < 0), so all (i, j) of one
// pivot may run at once and the result equals the reference's sequential
// k-i-j loop entry for entry, ties included.
__global__ void legacy_floyd_step_kernel(float *__restrict__ d, int *__restrict__ path, int n, int k) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const float dkj = d[(int64_t)k * n + j];
  const int pkj = path[(int64_t)k * n + j];
  for (int64_t i = blockIdx.y; i < n; i += gridDim.y) {
    const float c = d[i * n + k] + dkj;
    if (d[i * n + j] > c) {
      d[i * n + j] = c;
      path[i * n + j] = pkj;
    }
  }
}

bool upload(Dev &d, const void *host, size_t bytes) {
  return d.alloc(bytes) && (bytes == 0 || cudaMemcpy(d.p, host, bytes, cudaMemcpyHostToDevice) == cudaSuccess);
}

bool cuda_failed(const char *where) {
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return false;
  std::fprintf(stderr, "fap legacy %s: %s\n", where, cudaGetErrorString(e));
  t_status = FAP_ERR_CUDA;
  return true;
}

// res/res_path[m x n] by the rule of legacy_minplus_path_kernel, for host
// row-major arrays; c0/p0 (start values and predecessors) may be NULL.
// Every input is uploaded before an output is written, so res may alias
// mat1, mat2 or c0 and res_path may alias mat2_path or p0.
void host_minplus_path(const float *mat1, const float *mat2, const int *mat2_path, const float *c0,
                       const int *p0, float *res, int *res_path, int m, int n, int k, const char *where) {
  if (m <= 0 || n <= 0) {
    t_status = FAP_OK;
    return;
  }
  if (k < 0) k = 0;
  const size_t ca = (size_t)m * k, cb = (size_t)k * n, cc = (size_t)m * n;
  Dev A, B, Bp, C0, P0, C, P;
  if (!upload(A, mat1, ca * 4) || !upload(B, mat2, cb * 4) || !upload(Bp, mat2_path, cb * 4) ||
      (c0 && (!upload(C0, c0, cc * 4) || !upload(P0, p0, cc * 4))) || !C.alloc(cc * 4) ||
      !P.alloc(cc * 4)) {
    cudaGetLastError();
    report(FAP_ERR_NOMEM, where);
    return;
  }
  const dim3 grid((unsigned)((n + kPT - 1) / kPT), (unsigned)((m + kPT - 1) / kPT));
  if (grid.y > 65535u) {
    report(FAP_ERR_RANGE, where);
    return;
  }
  legacy_minplus_path_kernel<<<grid, dim3(kPT, 8)>>>(
      static_cast<const float *>(A.p), static_cast<const float *>(B.p), static_cast<const int *>(Bp.p),
      c0 ? static_cast<const float *>(C0.p) : nullptr, c0 ? static_cast<const int *>(P0.p) : nullptr,
      static_cast<float *>(C.p), static_cast<int *>(P.p), m, n, k);
  if (cuda_failed(where)) return;
  if (cudaMemcpy(res, C.p, cc * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(res_path, P.p, cc * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
    cuda_failed(where);
    return;
  }
  t_status = FAP_OK;
}

bool has_negative(const float *v, size_t count) {
  for (size_t i = 0; i < count; i++)
    if (!(v[i] >= 0.0f)) return true;
  return false;
}

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
  if (path != nullptr && num_node > 0) {
    // with predecessors: one launch per pivot, the reference's k-i-j order
    const size_t cnt = (size_t)num_node * num_node;
    if (has_negative(arc, cnt)) {
      std::fprintf(stderr, "fap legacy floyd_GPU_Nvidia_path: negative or NaN entries\n");
      t_status = FAP_ERR_INVALID;
      return;
    }
    Dev d, p;
    if (!upload(d, arc, cnt * 4) || !upload(p, path, cnt * 4)) {
      cudaGetLastError();
      report(FAP_ERR_NOMEM, "floyd_GPU_Nvidia_path");
      return;
    }
    const dim3 grid((unsigned)((num_node + 255) / 256), (unsigned)std::min(num_node, 65535));
    for (int k = 0; k < num_node; k++)
      legacy_floyd_step_kernel<<<grid, 256>>>(static_cast<float *>(d.p), static_cast<int *>(p.p), num_node, k);
    if (cuda_failed("floyd_GPU_Nvidia_path")) return;
    if (cudaMemcpy(arc, d.p, cnt * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(path, p.p, cnt * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
      cuda_failed("floyd_GPU_Nvidia_path");
      return;
    }
    t_status = FAP_OK;
    return;
  }
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
  if (mat2_path && res_path) {
    host_minplus_path(mat1, mat2, mat2_path, nullptr, nullptr, res, res_path, m, n, k, "minplus_NVIDIA_path");
    return;
  }
  host_minplus(mat1, mat2, res, m, n, k, "minplus_NVIDIA_path");
}

void minplus_NVIDIA_GPU(float *mat1, float *mat2, float *res, int M, int N, int K) {
  host_minplus(mat1, mat2, res, M, N, K, "minplus_NVIDIA_GPU");
}

void floyd_NVIDIA_GPU(int num_node, float *arc) { floyd_GPU_Nvidia_path(num_node, arc, nullptr); }

// Column panel of a blocked Floyd (fap/kernel/floyd.h:106-115): the new
// panel from the old one and the closed diagonal block, computed out of
// place as the reference's CUDA kernel intends.  With paths, each entry
// starts from its current value and predecessor, as the reference's CPU
// panel does (floyd_path_A_CPU, fap/kernel/floyd.h:68-84), and takes
// diag_path[k][j] from the first strictly shorter A[i][k] + diag[k][j].
void floyd_path_A_Nvidia(float *A, int *A_path, const int row, const int col, float *diag, int *diag_path) {
  if (A_path && diag_path) {
    host_minplus_path(A, diag, diag_path, A, A_path, A, A_path, row, col, col, "floyd_path_A_Nvidia");
    return;
  }
  host_minplus(A, diag, A, row, col, col, "floyd_path_A_Nvidia");
}

// Row panel of a blocked Floyd (fap/kernel/floyd.h:118-127); with paths,
// as floyd_path_B_CPU (:51-66) starts: current value and predecessor, then
// B_path[k][j] of the first strictly shorter diag[i][k] + B[k][j].
void floyd_path_B_Nvidia(float *B, int *B_path, const int row, const int col, float *diag, int *diag_path) {
  if (B_path) {
    host_minplus_path(diag, B, B_path, B, B_path, B, B_path, row, col, row, "floyd_path_B_Nvidia");
    return;
  }
  (void)diag_path;
  host_minplus(diag, B, B, row, col, row, "floyd_path_B_Nvidia");
}

// res = min(res, mat1 (x) mat2) (fap/kernel/floyd.h:130-139) as one product
// from the sentinel: [mat1 | E] (x) [mat2 ; res], E the min-plus identity
// (0 on the diagonal, 1e8 elsewhere), so that E (x) res = res.
void floyd_min_plus_Nvidia(float *mat1, float *mat2, int *mat2_path, float *res, int *res_path, int m, int n,
                           int k) {
  if (mat2_path && res_path) {
    // floyd_min_plus_CPU (fap/kernel/floyd.h:86-102): start from res and
    // res_path, take mat2_path[k][j] from the first strictly shorter sum
    host_minplus_path(mat1, mat2, mat2_path, res, res_path, res, res_path, m, n, k, "floyd_min_plus_Nvidia");
    return;
  }
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
