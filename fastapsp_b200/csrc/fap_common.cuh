// Shared definitions for the sm_100a kernels of the per-subgraph solve path.
//
// Distances are computed either in int32 (integer edge weights; DPX
// __viaddmin_s32 relaxations; bit-exact with the reference's float results
// while every finite distance stays below 2^24) or in float32 (fminf).
// Both use the reference's unreachable sentinel 1e8 (fap/utils/parameter.h:26)
// and its strict-improvement rule, so the sentinel is a fixed point:
// INF + w >= INF for every w >= 0, and INF + INF = 2e8 fits in int32.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fap_b200.h"

namespace fapb {

constexpr int kInfI32 = 100000000;  // 1e8, the reference's MAXVALUE
constexpr float kInfF32 = 1e8f;

template <typename T>
struct Dist;

template <>
struct Dist<int32_t> {
  static constexpr int kDtype = FAP_DTYPE_I32;
  __host__ __device__ static constexpr int32_t inf() { return kInfI32; }
  // min(a + b, c) in one DPX instruction.
  __device__ static __forceinline__ int32_t relax(int32_t a, int32_t b, int32_t c) {
    return __viaddmin_s32(a, b, c);
  }
  __device__ static __forceinline__ int32_t add(int32_t a, int32_t b) { return a + b; }
  __device__ static __forceinline__ int32_t min(int32_t a, int32_t b) { return ::min(a, b); }
  // Relaxation helper for atomics: non-negative int32 ordering.
  __device__ static __forceinline__ int32_t atomic_min(int32_t *p, int32_t v) {
    return atomicMin(p, v);
  }
};

template <>
struct Dist<float> {
  static constexpr int kDtype = FAP_DTYPE_F32;
  __host__ __device__ static constexpr float inf() { return kInfF32; }
  __device__ static __forceinline__ float relax(float a, float b, float c) {
    return fminf(a + b, c);
  }
  __device__ static __forceinline__ float add(float a, float b) { return a + b; }
  __device__ static __forceinline__ float min(float a, float b) { return fminf(a, b); }
  // For non-negative floats the IEEE bit patterns order like int32, so an
  // integer atomicMin on the bits is a float atomicMin.
  __device__ static __forceinline__ float atomic_min(float *p, float v) {
    return __int_as_float(atomicMin(reinterpret_cast<int *>(p), __float_as_int(v)));
  }
};

__host__ __device__ inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }
__host__ __device__ inline int64_t ceil_div(int64_t x, int64_t m) { return (x + m - 1) / m; }

// Device-side status word: kernels never trap; they record the first error
// here and return.  The host reads it after the stage.
enum DevStatus : int {
  kDevOk = 0,
  kDevSsspRoundLimit = 1,   // SSSP did not converge within its round bound
  kDevBadIndex = 2,         // an input index was out of range (skipped)
  kDevTmaTimeout = 3,       // a TMA stage never completed (bounded wait gave up)
  kDevQueueTimeout = 4,     // a work-queue item's dependencies never completed (bounded wait gave up)
};

__device__ inline void set_status(int *status, int code) {
  if (status) atomicCAS(status, 0, code);
}

}  // namespace fapb
