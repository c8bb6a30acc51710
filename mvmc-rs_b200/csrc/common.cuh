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
  kDevTimeout = 32u,       // a bounded device wait (mbarrier) expired
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

// A device attribute of the CURRENT device, cached per device ordinal (launch shapes
// queried on one GPU must not be reused on another with fewer SMs or less shared memory).
inline int current_device_attr(cudaDeviceAttr attr) {
  constexpr int kMaxDevices = 64;
  static int cache[kMaxDevices][3];  // value + 1; 0 = not queried yet
  int dev = 0;
  cudaGetDevice(&dev);
  const int slot = attr == cudaDevAttrMultiProcessorCount ? 0
                   : attr == cudaDevAttrMaxSharedMemoryPerBlockOptin ? 1
                   : attr == cudaDevAttrL2CacheSize ? 2 : -1;
  int value = 0;
  if (dev < 0 || dev >= kMaxDevices || slot < 0) {
    cudaDeviceGetAttribute(&value, attr, dev);
    return value;
  }
  if (cache[dev][slot] == 0) {
    cudaDeviceGetAttribute(&value, attr, dev);
    cache[dev][slot] = value + 1;
  }
  return cache[dev][slot] - 1;
}

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
