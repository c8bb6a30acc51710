// K5: SR-CG on the device.
//
// SampledSrOperator::solve_with_product (crates/mvmc-core/src/sr_cg.rs:700-880 of
// AtelierArith/mvmc-rs) with the C recurrence: threshold tol²·n², δ = β·δ (plain) or
// δ = δ_new (DiagScale), r = g − S·x at every 20th iteration, breakdown |d·q| < 1e-20,
// status = iterations or −(iter+1). S·v = Oᵀ(O·v)/W − (⟨O⟩·v)⟨O⟩ + δ_shift·diag·v
// (apply_with_product, sr_cg.rs:952-1009; COrderSr::cg_local_product,
// sr_backend.rs:518-606), the two passes over the compact active sample matrix O[s][i].
// One cooperative launch runs every iteration: no host round trip until the solve ends.
// Every reduction has a fixed order, so the recurrence is bitwise repeatable.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "common.cuh"
#include "engine.cuh"

namespace cgr = cooperative_groups;

namespace mvmcb {

constexpr int kCgThreads = 256;


__device__ double block_sum(double v, double* sh) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0) {
    for (int k = 0; k < static_cast<int>(blockDim.x >> 5); ++k) t += sh[k];
    sh[32] = t;
  }
  __syncthreads();
  t = sh[32];
  __syncthreads();
  return t;
}

// Grid-wide deterministic dot: every block gets the same value.
__device__ double grid_dot(cgr::grid_group& grid, const double* a, const double* b, int n,
                           double* red, double* sh) {
  double v = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v += a[i] * b[i];
  v = block_sum(v, sh);
  if (threadIdx.x == 0) red[blockIdx.x] = v;
  grid.sync();
  double t = 0.0;
  for (int k = 0; k < static_cast<int>(gridDim.x); ++k) t += red[k];
  grid.sync();
  return t;
}

// out = S·v
__device__ void sr_apply(cgr::grid_group& grid, const CgArgs& a, const double* v, double* out, double* sh) {
  const int lane = threadIdx.x & 31;
  const long long gw = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
  for (long long s = gw; s < a.ns; s += nwarps) {
    const double* row = a.O + s * a.na;
    double t = 0.0;
    for (int i = lane; i < a.na; i += 32) t += row[i] * v[i];
    t = warp_sum(t);
    if (lane == 0) a.y[s] = t;
  }
  const double coef = grid_dot(grid, a.mean, v, a.na, a.red, sh);  // includes a grid.sync
  const int ntile = (a.na + blockDim.x - 1) / blockDim.x;
  const long long chunk = (a.ns + a.nchunk - 1) / a.nchunk;
  for (int item = blockIdx.x; item < ntile * a.nchunk; item += gridDim.x) {
    const int tile = item % ntile, c = item / ntile;
    const int i = tile * blockDim.x + threadIdx.x;
    if (i >= a.na) continue;
    const long long s0 = c * chunk, s1 = min(a.ns, s0 + chunk);
    double t = 0.0;
    for (long long s = s0; s < s1; ++s) t += a.O[s * a.na + i] * a.y[s];
    a.part[static_cast<long long>(c) * a.na + i] = t;
  }
  grid.sync();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.na; i += gridDim.x * blockDim.x) {
    double z = 0.0;
    for (int c = 0; c < a.nchunk; ++c) z += a.part[static_cast<long long>(c) * a.na + i];
    out[i] = a.inv_w * z - coef * a.mean[i] + a.shift * a.diag[i] * v[i];
  }
  grid.sync();
}

__device__ __forceinline__ double precond(const CgArgs& a, int i, double r) {
  double dq = (1.0 + a.shift) * a.diag[i];
  if (!isfinite(dq) || fabs(dq) < 1e-12) dq = dq < 0.0 ? -1e-12 : 1e-12;
  return r / dq;
}

__global__ void __launch_bounds__(kCgThreads) k_sr_cg(CgArgs a) {
  cgr::grid_group grid = cgr::this_grid();
  __shared__ double sh[40];
  const int n = a.na;
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstride = gridDim.x * blockDim.x;
  const double threshold = a.tol * a.tol * static_cast<double>(n) * static_cast<double>(n);
  double delta;
  for (int i = gtid; i < n; i += gstride) {
    a.x[i] = 0.0;
    a.r[i] = a.g[i];
  }
  grid.sync();
  if (a.diag_scale) {
    sr_apply(grid, a, a.x, a.r, sh);
    for (int i = gtid; i < n; i += gstride) {
      a.r[i] = a.g[i] - a.r[i];
      a.d[i] = precond(a, i, a.r[i]);
    }
    grid.sync();
    delta = grid_dot(grid, a.r, a.d, n, a.red, sh);
  } else {
    for (int i = gtid; i < n; i += gstride) a.d[i] = a.g[i];
    grid.sync();
    delta = grid_dot(grid, a.r, a.r, n, a.red, sh);
  }
  long long status = 0;
  int iter = 0;
  bool done = false;
  if (!isfinite(delta)) {
    status = -1;
    done = true;
  }
  while (!done && iter < a.max_iter) {
    const long long failed = -(static_cast<long long>(iter) + 1);
    if (!isfinite(delta)) { status = failed; done = true; break; }
    if (fabs(delta) < threshold) break;
    sr_apply(grid, a, a.d, a.q, sh);
    const double dq = grid_dot(grid, a.d, a.q, n, a.red, sh);
    if (!isfinite(dq) || fabs(dq) < 1e-20) { status = failed; done = true; break; }
    const double alpha = delta / dq;
    if (!isfinite(alpha)) { status = failed; done = true; break; }
    for (int i = gtid; i < n; i += gstride) a.x[i] += alpha * a.d[i];
    grid.sync();
    if ((iter + 1) % 20 == 0) {
      sr_apply(grid, a, a.x, a.r, sh);
      for (int i = gtid; i < n; i += gstride) a.r[i] = a.g[i] - a.r[i];
    } else {
      for (int i = gtid; i < n; i += gstride) a.r[i] -= alpha * a.q[i];
    }
    grid.sync();
    double delta_new;
    if (a.diag_scale) {
      for (int i = gtid; i < n; i += gstride) a.q[i] = precond(a, i, a.r[i]);
      grid.sync();
      delta_new = grid_dot(grid, a.r, a.q, n, a.red, sh);
    } else {
      delta_new = grid_dot(grid, a.r, a.r, n, a.red, sh);
    }
    if (!isfinite(delta_new) || fabs(delta) < 1e-20) { status = failed; done = true; break; }
    const double beta = delta_new / delta;
    if (!isfinite(beta)) { status = failed; done = true; break; }
    if (a.diag_scale) {
      delta = delta_new;
      for (int i = gtid; i < n; i += gstride) a.d[i] = a.q[i] + beta * a.d[i];
    } else {
      delta *= beta;
      for (int i = gtid; i < n; i += gstride) a.d[i] = a.r[i] + beta * a.d[i];
    }
    grid.sync();
    ++iter;
  }
  if (!done) {
    if (iter == a.max_iter && fabs(delta) >= threshold) status = -(static_cast<long long>(a.max_iter) + 1);
    else status = iter;
  }
  if (gtid == 0) {
    a.scal[0] = delta;
    a.scal[1] = static_cast<double>(status);
    a.scal[2] = static_cast<double>(iter);
  }
}

// Gather the active columns of the stored O rows: Oa[s][si] = store[s][map[si] + 1].
__global__ void k_gather_active(const double* __restrict__ store, int sr_size, long long ns,
                                const int* __restrict__ map, int na, double* __restrict__ oa) {
  const long long total = ns * na;
  for (long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; k < total;
       k += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long s = k / na;
    const int si = static_cast<int>(k - s * na);
    oa[k] = store[s * sr_size + map[si] + 1];
  }
}

int launch_gather_active(const double* store, int sr_size, long long ns, const int* map, int na,
                         double* oa, cudaStream_t stream) {
  const long long total = ns * na;
  const int grid = static_cast<int>(std::min<long long>((total + 255) / 256, 148LL * 32));
  k_gather_active<<<std::max(1, grid), 256, 0, stream>>>(store, sr_size, ns, map, na, oa);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

// Blocks of the cooperative solve: enough to stream the sample matrix (about 64K
// elements per block), never more than are co-resident.
int cg_grid_blocks(long long ns, int na) {
  static int cap = -1;
  if (cap < 0) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sr_cg, kCgThreads, 0);
    cap = sms * std::max(1, std::min(per, 4));
  }
  const long long want = (ns * static_cast<long long>(na) + 65535) / 65536;
  return static_cast<int>(std::max<long long>(1, std::min<long long>(cap, want)));
}

int launch_sr_cg(CgArgs a, cudaStream_t stream) {
  void* args[] = {&a};
  MVMCB_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_sr_cg), cg_grid_blocks(a.ns, a.na), kCgThreads,
                                         args, 0, stream));
  return kOk;
}

}  // namespace mvmcb

// Fixed-operand solve through the C ABI (SrStages::cg_step, sr_backend.rs:193-297).
namespace {
struct Buf {
  void* p = nullptr;
  ~Buf() {
    if (p) cudaFree(p);
  }
};
}  // namespace

extern "C" int mvmc_b200_cg_solve(const double* samples, long long ns, int na, const double* mean,
                                  const double* diag, const double* g, double inv_w, double shift,
                                  double tol, int max_iter, int diag_scale, double* x,
                                  long long* status) {
  using namespace mvmcb;
  if (!samples || !mean || !diag || !g || !x || !status || na <= 0 || ns <= 0) return kErrArgument;
  const int blocks = cg_grid_blocks(ns, na);
  const int ntile = (na + 255) / 256;
  const int nchunk = static_cast<int>(std::max<long long>(1, std::min<long long>(ns, std::max(1, blocks / ntile))));
  Buf o, vec, y, part, red, scal;
  MVMCB_CUDA(cudaMalloc(&o.p, sizeof(double) * ns * na));
  MVMCB_CUDA(cudaMalloc(&vec.p, sizeof(double) * 7 * na));
  MVMCB_CUDA(cudaMalloc(&y.p, sizeof(double) * ns));
  MVMCB_CUDA(cudaMalloc(&part.p, sizeof(double) * nchunk * na));
  MVMCB_CUDA(cudaMalloc(&red.p, sizeof(double) * 4096));
  MVMCB_CUDA(cudaMalloc(&scal.p, sizeof(double) * 8));
  double* v = static_cast<double*>(vec.p);
  MVMCB_CUDA(cudaMemcpy(o.p, samples, sizeof(double) * ns * na, cudaMemcpyHostToDevice));
  MVMCB_CUDA(cudaMemcpy(v, mean, sizeof(double) * na, cudaMemcpyHostToDevice));
  MVMCB_CUDA(cudaMemcpy(v + na, diag, sizeof(double) * na, cudaMemcpyHostToDevice));
  MVMCB_CUDA(cudaMemcpy(v + 2 * na, g, sizeof(double) * na, cudaMemcpyHostToDevice));
  CgArgs a;
  a.O = static_cast<double*>(o.p);
  a.mean = v;
  a.diag = v + na;
  a.g = v + 2 * na;
  a.x = v + 3 * na;
  a.r = v + 4 * na;
  a.d = v + 5 * na;
  a.q = v + 6 * na;
  a.y = static_cast<double*>(y.p);
  a.part = static_cast<double*>(part.p);
  a.red = static_cast<double*>(red.p);
  a.scal = static_cast<double*>(scal.p);
  a.ns = ns;
  a.na = na;
  a.nchunk = nchunk;
  a.max_iter = max_iter;
  a.diag_scale = diag_scale;
  a.inv_w = inv_w;
  a.shift = shift;
  a.tol = tol;
  const int rc = launch_sr_cg(a, nullptr);
  if (rc != kOk) return rc;
  double sc[8];
  MVMCB_CUDA(cudaMemcpy(x, a.x, sizeof(double) * na, cudaMemcpyDeviceToHost));
  MVMCB_CUDA(cudaMemcpy(sc, a.scal, sizeof(double) * 8, cudaMemcpyDeviceToHost));
  *status = static_cast<long long>(sc[1]);
  return kOk;
}
