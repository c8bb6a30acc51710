// SR-CG on caller-owned device buffers with no device allocation.
//
// Some callers cannot let a library call cudaMalloc: a host program whose device memory
// is owned by its own pooling allocator (a framework's caching allocator, a fixed memory
// budget shared with other models) would see a raw cudaMalloc fragment its pool or push
// it over budget, and cudaMalloc / cudaFree can synchronise the device and stall the
// caller's other streams. For them this entry point runs the same cooperative SR-CG
// kernel as mvmc_b200_cg_solve, but takes every input and output as a device pointer
// and keeps its working vectors in a fixed array compiled into this library.
//
// The array holds kNoAllocScratchDoubles doubles (8 MiB) on every GPU that loads the
// library, for the lifetime of the process. A solve needs
//   3·na (residual, direction, product) + ns (row products)
//   + nchunk·na (column partial sums) + 2·blocks (two slots of block partials)
// doubles of it; larger problems are rejected with MVMC_B200_EARG and a message.
// Every call uses the same array: calls that overlap on the GPU (two streams, or two
// host threads on one device) race on it and must be serialised by the caller. Each
// call writes every scratch element before reading it, so nothing needs clearing.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/mvmc_b200.h"
#include "../host/abi_common.h"
#include "common.cuh"
#include "engine.cuh"

namespace mvmcb {

int launch_sr_cg(CgArgs a, cudaStream_t stream);
int cg_grid_blocks(long long ns, int na);
int cg_nchunk(long long ns, int na, int kind, int blocks);

namespace {

constexpr long long kNoAllocScratchDoubles = 1LL << 20;  // 8 MiB per GPU

// Device storage of the working vectors. In host code this name is only a host-side
// stand-in for the symbol: its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) double g_cg_scratch[kNoAllocScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once per device
// (with that device current) on its first call.
int scratch_on_current_device(double** out) {
  int dev = 0;
  MVMCB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_last_error("cg_solve_noalloc: device ordinal out of range");
    return kErrArgument;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_cg_scratch);
    if (e != cudaSuccess) {
      set_last_error(std::string("cg_solve_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
      return kErrCuda;
    }
    g_scratch_ptr[dev] = static_cast<double*>(ptr);
  }
  *out = g_scratch_ptr[dev];
  return kOk;
}

}  // namespace
}  // namespace mvmcb

extern "C" int mvmc_b200_cg_solve_noalloc(const double* samples, long long ns, int na, const double* mean,
                                          const double* diag, const double* g, double inv_w, double shift,
                                          double tol, int max_iter, int diag_scale, double* x, double* result,
                                          void* stream) {
  using namespace mvmcb;
  if (!samples || !mean || !diag || !g || !x || !result || na <= 0 || ns <= 0 || max_iter < 0) {
    set_last_error("cg_solve_noalloc: null pointer or non-positive size");
    return kErrArgument;
  }
  if (3LL * na + ns > kNoAllocScratchDoubles) {
    set_last_error("cg_solve_noalloc: problem exceeds the 8 MiB scratch array (3*na + ns + partials > 1048576 doubles)");
    return kErrArgument;
  }
  const int blocks = cg_grid_blocks(ns, na);
  const int nchunk = cg_nchunk(ns, na, 0, blocks);
  const long long need = 3LL * na + ns + static_cast<long long>(nchunk) * na + 2LL * blocks;
  if (need > kNoAllocScratchDoubles) {
    set_last_error("cg_solve_noalloc: problem needs " + std::to_string(need) +
                   " scratch doubles; the array holds 1048576 (8 MiB)");
    return kErrArgument;
  }
  double* scratch = nullptr;
  const int rc = scratch_on_current_device(&scratch);
  if (rc != kOk) return rc;
  CgArgs a;
  a.O = samples;
  a.mean = mean;
  a.diag = diag;
  a.g = g;
  a.x = x;
  a.r = scratch;
  a.d = scratch + na;
  a.q = scratch + 2LL * na;
  a.y = scratch + 3LL * na;
  a.part = a.y + ns;
  a.red = a.part + static_cast<long long>(nchunk) * na;
  a.scal = result;
  a.ns = ns;
  a.na = na;
  a.nchunk = nchunk;
  a.max_iter = max_iter;
  a.diag_scale = diag_scale;
  a.inv_w = inv_w;
  a.shift = shift;
  a.tol = tol;
  return launch_sr_cg(a, static_cast<cudaStream_t>(stream));
}
