// K1: batched skew Pfaffian + inverse (PfaffianStages::pfaffian_inverse_batch).
//
// One CTA per plane. Planes up to the shared-memory limit are swept in shared memory
// (row stride n+1 to spread banks); larger FP64 planes are swept in place in the output
// buffer (L2-resident working set). Input and output are column-major as in
// crates/mvmc-core/src/stage_backend.rs:121-165; the returned inverse is the true X⁻¹.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "../../include/mvmc_b200.h"
#include "common.cuh"
#include "pfinv.cuh"

namespace mvmcb {

constexpr int kPfinvThreads = 256;
int device_sm_count();

// Column-major X read row-major is Xᵀ = −X, so loading −buffer gives X row-major and the
// row-major X⁻¹ negated is the column-major X⁻¹.
template <typename T, bool kSmem>
__global__ void __launch_bounds__(kPfinvThreads)
    k_pfinv_batch(const double* __restrict__ x, const int* __restrict__ sizes,
                  const long long* __restrict__ offsets, int n_uniform, int planes, int n_max,
                  double* __restrict__ pf, double* __restrict__ inv, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem[];
  const size_t scratch = (gj_shared_bytes<T>(n_max) + 15) & ~size_t(15);
  GJShared<T> s = gj_carve<T>(smem, n_max);
  for (int plane = blockIdx.x; plane < planes; plane += gridDim.x) {
    const int n = sizes ? sizes[plane] : n_uniform;
    const long long off = offsets ? offsets[plane] : static_cast<long long>(plane) * n * n;
    const double* xp = x + off;
    double* ip = inv + off;
    T* A;
    int lda;
    if (kSmem) {
      A = reinterpret_cast<T*>(smem + scratch);
      lda = n + 1;
    } else {
      A = reinterpret_cast<T*>(ip);  // only instantiated for T = double
      lda = n;
    }
    for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
      const int i = k / n, j = k - i * n;
      A[i * lda + j] = static_cast<T>(-xp[k]);
    }
    __syncthreads();
    double pfv;
    int st;
    gj_pfinv<T>(A, lda, n, s, pfv, st);
    for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
      const int i = k / n, j = k - i * n;
      ip[k] = -static_cast<double>(A[i * lda + j]);
    }
    if (threadIdx.x == 0) {
      pf[plane] = pfv;
      status[plane] = st;
    }
    __syncthreads();
  }
}

// One barrier per pivot step: the matrix and its ping-pong partner in shared memory.
template <typename T, int JPL>
__global__ void __launch_bounds__(kPfinvThreads)
    k_pfinv_pp(const double* __restrict__ x, const int* __restrict__ sizes,
               const long long* __restrict__ offsets, int n_uniform, int planes, int n_max,
               double* __restrict__ pf, double* __restrict__ inv, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem[];
  T* A = reinterpret_cast<T*>(smem);
  T* B = A + static_cast<size_t>(n_max) * n_max;
  for (int plane = blockIdx.x; plane < planes; plane += gridDim.x) {
    const int n = sizes ? sizes[plane] : n_uniform;
    const long long off = offsets ? offsets[plane] : static_cast<long long>(plane) * n * n;
    const double* xp = x + off;
    double* ip = inv + off;
    for (int k = threadIdx.x; k < n * n; k += blockDim.x) A[k] = static_cast<T>(-xp[k]);
    __syncthreads();
    double pfv;
    int st;
    gj_pfinv_pp<T, JPL>(A, B, n, pfv, st);
    for (int k = threadIdx.x; k < n * n; k += blockDim.x) ip[k] = -static_cast<double>(A[k]);
    if (threadIdx.x == 0) {
      pf[plane] = pfv;
      status[plane] = st;
    }
    __syncthreads();
  }
}

template <typename T, int JPL>
int launch_pfinv_pp(const double* x, const int* sizes, const long long* offsets, int n_uniform,
                    int planes, int n_max, double* pf, double* inv, int* status, cudaStream_t stream) {
  const size_t smem = 2 * sizeof(T) * static_cast<size_t>(n_max) * n_max;
  auto kernel = k_pfinv_pp<T, JPL>;
  MVMCB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  int per_sm = 0;
  MVMCB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kPfinvThreads, smem));
  const int grid = std::max(1, std::min(planes, std::max(1, per_sm) * device_sm_count()));
  kernel<<<grid, kPfinvThreads, smem, stream>>>(x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

template <typename T>
int dispatch_pfinv_pp(const double* x, const int* sizes, const long long* offsets, int n_uniform,
                      int planes, int n_max, double* pf, double* inv, int* status, cudaStream_t stream) {
  if (n_max <= 32) return launch_pfinv_pp<T, 1>(x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status, stream);
  if (n_max <= 64) return launch_pfinv_pp<T, 2>(x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status, stream);
  if (n_max <= 128) return launch_pfinv_pp<T, 4>(x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status, stream);
  if (n_max <= 224) return launch_pfinv_pp<T, 7>(x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status, stream);
  return launch_pfinv_pp<T, 8>(x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status, stream);
}

template <typename T>
size_t pfinv_smem_bytes(int n_max, bool smem_matrix) {
  size_t b = (gj_shared_bytes<T>(n_max) + 15) & ~size_t(15);
  if (smem_matrix) b += sizeof(T) * static_cast<size_t>(n_max) * (n_max + 1);
  return b;
}

int device_smem_limit() {
  static int limit = -1;
  if (limit < 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&limit, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  }
  return limit;
}

int device_sm_count() {
  static int count = -1;
  if (count < 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
  }
  return count;
}

template <typename T, bool kSmem>
int launch_pfinv(const double* x, const int* sizes, const long long* offsets, int n_uniform,
                 int planes, int n_max, double* pf, double* inv, int* status, cudaStream_t stream) {
  const size_t smem = pfinv_smem_bytes<T>(n_max, kSmem);
  MVMCB_CUDA(cudaFuncSetAttribute(k_pfinv_batch<T, kSmem>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem)));
  int per_sm = 0;
  MVMCB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pfinv_batch<T, kSmem>,
                                                           kPfinvThreads, smem));
  const int grid = std::max(1, std::min(planes, std::max(1, per_sm) * device_sm_count()));
  k_pfinv_batch<T, kSmem><<<grid, kPfinvThreads, smem, stream>>>(x, sizes, offsets, n_uniform,
                                                                  planes, n_max, pf, inv, status);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

int pfinv_device(const double* x, const int* sizes, const long long* offsets, int n_uniform,
                 int planes, int n_max, double* pf, double* inv, int* status, int precision,
                 cudaStream_t stream) {
  if (planes <= 0) return kOk;
  if (n_max <= 0 || (n_max & 1) || !x || !pf || !inv || !status) return kErrArgument;
  const int limit = device_smem_limit();
  const size_t pp_bytes = 2 * static_cast<size_t>(n_max) * n_max * (precision == 32 ? 4 : 8);
  if (n_max <= 256 && pp_bytes <= static_cast<size_t>(limit)) {
    if (precision == 32)
      return dispatch_pfinv_pp<float>(x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status, stream);
    if (precision == 64)
      return dispatch_pfinv_pp<double>(x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status, stream);
  }
  if (precision == 32) {
    if (pfinv_smem_bytes<float>(n_max, true) > static_cast<size_t>(limit)) return kErrArgument;
    return launch_pfinv<float, true>(x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status,
                                     stream);
  }
  if (precision != 64) return kErrArgument;
  if (pfinv_smem_bytes<double>(n_max, true) <= static_cast<size_t>(limit))
    return launch_pfinv<double, true>(x, sizes, offsets, n_uniform, planes, n_max, pf, inv,
                                      status, stream);
  return launch_pfinv<double, false>(x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status,
                                     stream);
}

}  // namespace mvmcb

using namespace mvmcb;

extern "C" int mvmc_b200_pfinv_batch_device(const double* x, const int* sizes,
                                            const long long* offsets, int n_uniform, int planes,
                                            int n_max, double* pf, double* inv, int* status,
                                            int precision, void* stream) {
  return pfinv_device(x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status, precision,
                      static_cast<cudaStream_t>(stream));
}

namespace {
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};
}  // namespace

extern "C" int mvmc_b200_pfinv_batch(const double* x, int n, int planes, double* pf, double* inv,
                                     int* status) {
  if (n <= 0 || (n & 1) || planes < 0) return kErrArgument;
  if (planes == 0) return kOk;
  const size_t nn = static_cast<size_t>(n) * n * planes;
  DevBuf dx, dinv, dpf, dst;
  MVMCB_CUDA(cudaMalloc(&dx.p, nn * sizeof(double)));
  MVMCB_CUDA(cudaMalloc(&dinv.p, nn * sizeof(double)));
  MVMCB_CUDA(cudaMalloc(&dpf.p, planes * sizeof(double)));
  MVMCB_CUDA(cudaMalloc(&dst.p, planes * sizeof(int)));
  MVMCB_CUDA(cudaMemcpy(dx.p, x, nn * sizeof(double), cudaMemcpyHostToDevice));
  int rc = pfinv_device(static_cast<double*>(dx.p), nullptr, nullptr, n, planes, n,
                        static_cast<double*>(dpf.p), static_cast<double*>(dinv.p),
                        static_cast<int*>(dst.p), 64, nullptr);
  if (rc != kOk) return rc;
  MVMCB_CUDA(cudaMemcpy(inv, dinv.p, nn * sizeof(double), cudaMemcpyDeviceToHost));
  MVMCB_CUDA(cudaMemcpy(pf, dpf.p, planes * sizeof(double), cudaMemcpyDeviceToHost));
  MVMCB_CUDA(cudaMemcpy(status, dst.p, planes * sizeof(int), cudaMemcpyDeviceToHost));
  return kOk;
}

extern "C" int mvmc_b200_pfinv_batch_mixed(const double* x, const int* sizes, int planes,
                                           int precision, double* pf, double* inv, int* status) {
  if (planes < 0 || !sizes) return kErrArgument;
  if (planes == 0) return kOk;
  std::vector<long long> offsets(planes);
  long long total = 0;
  int n_max = 0;
  for (int p = 0; p < planes; ++p) {
    if (sizes[p] <= 0 || (sizes[p] & 1)) return kErrArgument;
    offsets[p] = total;
    total += static_cast<long long>(sizes[p]) * sizes[p];
    n_max = std::max(n_max, sizes[p]);
  }
  DevBuf dx, dinv, dpf, dst, dsz, doff;
  MVMCB_CUDA(cudaMalloc(&dx.p, total * sizeof(double)));
  MVMCB_CUDA(cudaMalloc(&dinv.p, total * sizeof(double)));
  MVMCB_CUDA(cudaMalloc(&dpf.p, planes * sizeof(double)));
  MVMCB_CUDA(cudaMalloc(&dst.p, planes * sizeof(int)));
  MVMCB_CUDA(cudaMalloc(&dsz.p, planes * sizeof(int)));
  MVMCB_CUDA(cudaMalloc(&doff.p, planes * sizeof(long long)));
  MVMCB_CUDA(cudaMemcpy(dx.p, x, total * sizeof(double), cudaMemcpyHostToDevice));
  MVMCB_CUDA(cudaMemcpy(dsz.p, sizes, planes * sizeof(int), cudaMemcpyHostToDevice));
  MVMCB_CUDA(cudaMemcpy(doff.p, offsets.data(), planes * sizeof(long long), cudaMemcpyHostToDevice));
  int rc = pfinv_device(static_cast<double*>(dx.p), static_cast<int*>(dsz.p),
                        static_cast<long long*>(doff.p), 0, planes, n_max,
                        static_cast<double*>(dpf.p), static_cast<double*>(dinv.p),
                        static_cast<int*>(dst.p), precision, nullptr);
  if (rc != kOk) return rc;
  MVMCB_CUDA(cudaMemcpy(inv, dinv.p, total * sizeof(double), cudaMemcpyDeviceToHost));
  MVMCB_CUDA(cudaMemcpy(pf, dpf.p, planes * sizeof(double), cudaMemcpyDeviceToHost));
  MVMCB_CUDA(cudaMemcpy(status, dst.p, planes * sizeof(int), cudaMemcpyDeviceToHost));
  return kOk;
}
