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
// cudaGetSymbolAddress (noalloc_symbols below).
static __device__ __align__(256) int32_t g_noalloc_floyd[FAP_NOALLOC_FLOYD_MAX * FAP_NOALLOC_FLOYD_MAX];

// Device-side status word of the last call on this device: the Floyd
// kernels' bounded TMA waits record kDevTmaTimeout here instead of hanging.
// Cleared on the stream before every call's kernels.
static __device__ __align__(16) int g_noalloc_status;

constexpr int kMaxDevices = 64;
std::mutex g_mu;
struct Symbols {
  void *scratch = nullptr;
  int *status = nullptr;
};
Symbols g_sym[kMaxDevices];

thread_local char t_msg[256];

int noalloc_fail(int code, const char *msg) {
  std::snprintf(t_msg, sizeof(t_msg), "fap_floyd_noalloc: %s", msg);
  return code;
}

// Device addresses of the scratch array and the status word on the current
// device.  They are looked up again on every call made outside a stream
// capture (so a cudaDeviceReset, after which the module loads again at a
// possibly different address, is picked up by the next call); inside a
// capture the addresses of the last lookup on this device are used, so the
// first call on a device must come before any capture.
int noalloc_symbols(cudaStream_t st, Symbols *out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return noalloc_fail(FAP_ERR_CUDA, "no current CUDA device");
  }
  if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(FAP_ERR_CUDA, "device ordinal too large");
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
    cudaGetLastError();
    cap = cudaStreamCaptureStatusActive;   // cannot tell: do not touch the module
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (cap == cudaStreamCaptureStatusNone) {
    void *p = nullptr, *q = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_floyd);
    if (e == cudaSuccess) e = cudaGetSymbolAddress(&q, g_noalloc_status);
    if (e != cudaSuccess || p == nullptr || q == nullptr) {
      cudaGetLastError();
      return noalloc_fail(FAP_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
    }
    g_sym[dev].scratch = p;
    g_sym[dev].status = static_cast<int *>(q);
  } else if (!g_sym[dev].scratch) {
    return noalloc_fail(FAP_ERR_STATE,
                        "the first call on a device must come before any stream capture");
  }
  *out = g_sym[dev];
  return FAP_OK;
}

template <typename T>
cudaError_t noalloc_run(T *scratch, int *status, int32_t s, T *mat, int64_t ld, cudaStream_t st) {
  const int64_t ldp = round_up(s, kFloydTile);
  int64_t launches = 0;
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), st);
  // The array keeps the previous call's contents: reset the padded square.
  if (e == cudaSuccess) e = launch_fill<T>(scratch, ldp, ldp, ldp, Dist<T>::inf(), st, &launches);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(scratch, (size_t)ldp * sizeof(T), mat, (size_t)ld * sizeof(T),
                          (size_t)s * sizeof(T), (size_t)s, cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess)
    e = launch_floyd_matrix<T>(scratch, ldp, (int)(ldp / kFloydTile), status, st, &launches);
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
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  Symbols sym;
  const int rc = noalloc_symbols(st, &sym);
  if (rc != FAP_OK) return rc;
  const cudaError_t e =
      (dtype == FAP_DTYPE_I32)
          ? noalloc_run<int32_t>(static_cast<int32_t *>(sym.scratch), sym.status, s,
                                 static_cast<int32_t *>(mat), ld, st)
          : noalloc_run<float>(static_cast<float *>(sym.scratch), sym.status, s,
                               static_cast<float *>(mat), ld, st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return noalloc_fail(FAP_ERR_CUDA, cudaGetErrorString(e));
  }
  return FAP_OK;
}

extern "C" int fap_floyd_noalloc_status(void) {
  t_msg[0] = 0;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return noalloc_fail(FAP_ERR_CUDA, "no current CUDA device");
  }
  int *status = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    status = g_sym[dev].status;
  }
  if (!status) return noalloc_fail(FAP_ERR_STATE, "no call on this device yet");
  int h = 0;
  // A plain copy into host memory: no allocation.  It waits only for work
  // already queued on the legacy default stream.
  const cudaError_t e = cudaMemcpy(&h, status, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return noalloc_fail(FAP_ERR_CUDA, cudaGetErrorString(e));
  }
  if (h == kDevTmaTimeout)
    return noalloc_fail(FAP_ERR_DEVICE, "a TMA tile load did not complete in time; the matrix is not closed");
  if (h != kDevOk) return noalloc_fail(FAP_ERR_DEVICE, "device-side error");
  return FAP_OK;
}
