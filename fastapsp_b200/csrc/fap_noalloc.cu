// Allocation-free Floyd-Warshall entry point.
//
// Some callers cannot allocate device memory at the moment they need a
// closure: code running under a host framework that owns every byte of the
// GPU through its own pool (a database or query-engine plugin, a serving
// process that reserved its memory up front), or a latency-sensitive path
// where cudaMalloc / cudaFree would implicitly synchronise the device.
// fap_floyd_noalloc gives them the stage-2 closure with no allocation at all:
// the padded working copy that fap_op_floyd allocates lives instead in one
// file-scope device array of FAP_NOALLOC_FLOYD_MAX^2 elements (4 MiB), which
// every GPU that loads this library keeps until the process exits.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "fap_b200.h"
#include "fap_common.cuh"
#include "fap_internal.h"

using namespace fapb;

namespace {

static_assert(FAP_NOALLOC_FLOYD_MAX % kFloydTile == 0, "scratch side must be whole tiles");

// The shared working matrix.  Host code must not use this name as a device
// address: it is a host-side stand-in.  The device address comes from
// cudaGetSymbolAddress (noalloc_scratch_ptr below).
static __device__ __align__(256) int32_t g_noalloc_floyd[FAP_NOALLOC_FLOYD_MAX * FAP_NOALLOC_FLOYD_MAX];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_ptr[kMaxDevices] = {};

thread_local char t_msg[256];

int noalloc_fail(int code, const char *msg) {
  std::snprintf(t_msg, sizeof(t_msg), "fap_floyd_noalloc: %s", msg);
  return code;
}

// Device address of the scratch array on the current device; looked up
// once per device (the first call on a device does it).
int noalloc_scratch_ptr(void **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return noalloc_fail(FAP_ERR_CUDA, "no current CUDA device");
  }
  if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(FAP_ERR_CUDA, "device ordinal too large");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_ptr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_floyd);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return noalloc_fail(FAP_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
    }
    g_ptr[dev] = p;
  }
  *out = g_ptr[dev];
  return FAP_OK;
}

template <typename T>
cudaError_t noalloc_run(T *scratch, int32_t s, T *mat, int64_t ld, cudaStream_t st) {
  const int64_t ldp = round_up(s, kFloydTile);
  int64_t launches = 0;
  // The array keeps the previous call's contents: reset the padded square.
  cudaError_t e = launch_fill<T>(scratch, ldp, ldp, ldp, Dist<T>::inf(), st, &launches);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(scratch, (size_t)ldp * sizeof(T), mat, (size_t)ld * sizeof(T),
                          (size_t)s * sizeof(T), (size_t)s, cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess)
    e = launch_floyd_matrix<T>(scratch, ldp, (int)(ldp / kFloydTile), nullptr, st, &launches);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(mat, (size_t)ld * sizeof(T), scratch, (size_t)ldp * sizeof(T),
                          (size_t)s * sizeof(T), (size_t)s, cudaMemcpyDeviceToDevice, st);
  return e;
}

}  // namespace

extern "C" const char *fap_floyd_noalloc_last_error(void) { return t_msg; }

extern "C" int fap_floyd_noalloc(int dtype, int32_t s, void *mat, int64_t ld, void *stream) {
  t_msg[0] = 0;
  if (dtype != FAP_DTYPE_I32 && dtype != FAP_DTYPE_F32) return noalloc_fail(FAP_ERR_INVALID, "bad dtype");
  if (s < 0 || ld < s) return noalloc_fail(FAP_ERR_INVALID, "need 0 <= s <= ld");
  if (s > FAP_NOALLOC_FLOYD_MAX)
    return noalloc_fail(FAP_ERR_RANGE, "matrix side exceeds FAP_NOALLOC_FLOYD_MAX (1024)");
  if (s == 0) return FAP_OK;
  if (!mat) return noalloc_fail(FAP_ERR_INVALID, "mat is NULL");
  void *scratch = nullptr;
  const int rc = noalloc_scratch_ptr(&scratch);
  if (rc != FAP_OK) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const cudaError_t e =
      (dtype == FAP_DTYPE_I32)
          ? noalloc_run<int32_t>(static_cast<int32_t *>(scratch), s, static_cast<int32_t *>(mat), ld, st)
          : noalloc_run<float>(static_cast<float *>(scratch), s, static_cast<float *>(mat), ld, st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return noalloc_fail(FAP_ERR_CUDA, cudaGetErrorString(e));
  }
  return FAP_OK;
}
