// Shared device helpers for the mvmc-b200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>

namespace mvmcb {

// Status codes returned through the C ABI (see include/mvmc_b200.h).
enum Status : int {
  kOk = 0,
  kErrArgument = -1,
  kErrCuda = -2,
  kErrModel = -3,
  kErrNumeric = -4,
  kErrTimeout = -5,
  kErrState = -6,
};

// Sticky device status bits written by kernels (never a trap).
enum DeviceStatus : unsigned {
  kDevSingular = 1u,       // a Pfaffian/inverse met a zero pivot
  kDevNonFinite = 2u,      // a non-finite Pfaffian / weight / energy
  kDevInitLoops = 4u,      // makeInitialSample exhausted its retries
  kDevBounds = 8u,         // an index check failed (checked builds)
  kDevCandidateLoop = 16u, // a proposal loop exceeded its bound
};

#define MVMCB_CUDA(call)                                                         \
  do {                                                                           \
    cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess) {                                                     \
      std::fprintf(stderr, "mvmc_b200: %s failed: %s (%s:%d)\n", #call,          \
                   cudaGetErrorString(e_), __FILE__, __LINE__);                  \
      return ::mvmcb::kErrCuda;                                                  \
    }                                                                            \
  } while (0)

template <typename T>
__device__ __forceinline__ T dev_abs(T x) {
  return x < T(0) ? -x : x;
}

// Warp argmax of |v| with the lowest index winning ties (first maximum).
__device__ __forceinline__ void warp_argmax_first(double& v, int& idx) {
  for (int off = 16; off > 0; off >>= 1) {
    const double ov = __shfl_down_sync(0xffffffffu, v, off);
    const int oi = __shfl_down_sync(0xffffffffu, idx, off);
    if (ov > v || (ov == v && oi < idx)) {
      v = ov;
      idx = oi;
    }
  }
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

}  // namespace mvmcb
