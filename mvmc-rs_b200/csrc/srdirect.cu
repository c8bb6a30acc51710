// Direct SR on the device (NSRCG = 0): the Gram of the SR sample matrix, the S/g
// assembly on the active set, and the Cholesky solve.
//
// Reference: stochastic_opt_real_with_sr_info_timed (crates/mvmc-core/src/sr.rs:77-160 of
// AtelierArith/mvmc-rs) over the SrStages seam — gram_real (sr_backend.rs:464; the C order
// is one dgemm of the stored rows, c_order_gram_real :312), assemble_s_g (:484-511) and
// cholesky_solve (sr.rs:535: LAPACK dpotrf('U') + dpotrs).
//
// K6 k_gram: OO = Σ_s O_s O_sᵀ / Wc over the stored rows, 64×64 output tiles of the lower
// triangle per block (4×4 per thread), the sample axis staged through shared memory in
// chunks of 16 rows; every entry is summed in sample order, then mirrored.
// K7 k_cholesky: one cooperative launch, right-looking with 32-wide panels: block 0
// factors the diagonal block in shared memory, all blocks solve the panel rows below it,
// all blocks update the trailing lower triangle in 64×64 tiles (grid barrier between the
// three). S = L Lᵀ with L = Uᵀ of dpotrf('U'). K8 k_cholesky_solve: one block, the
// forward and backward substitutions blocked by 32.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/mvmc_b200.h"
#include "../host/abi_common.h"
#include "common.cuh"

namespace cgr = cooperative_groups;

namespace mvmcb {

constexpr int kGramTile = 64;
constexpr int kGramK = 16;
constexpr int kCholB = 32;   // panel width
constexpr int kCholT = 64;   // trailing-update tile (kCholThreads = 16 × 16 threads, 4 × 4 each)
constexpr int kCholThreads = 256;

// OO[i][j] (i ≥ j tiles) of the rows store[s][0..n) for s < ns, scaled by inv_w.
__global__ void __launch_bounds__(256) k_gram(const double* __restrict__ store, int n, long long ns, double inv_w,
                                              double* __restrict__ oo) {
  __shared__ double As[kGramK][kGramTile + 1];
  __shared__ double Bs[kGramK][kGramTile + 1];
  const int ntile = (n + kGramTile - 1) / kGramTile;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  for (int t = blockIdx.x; t < ntile * (ntile + 1) / 2; t += gridDim.x) {
    // triangular tile index → (ti, tj), ti ≥ tj
    int ti = static_cast<int>((sqrt(8.0 * t + 1.0) - 1.0) / 2.0);
    while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
    while (ti * (ti + 1) / 2 > t) --ti;
    const int tj = t - ti * (ti + 1) / 2;
    const int i0 = ti * kGramTile, j0 = tj * kGramTile;
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
    for (long long s0 = 0; s0 < ns; s0 += kGramK) {
      for (int e = tid; e < kGramK * kGramTile; e += blockDim.x) {
        const int r = e / kGramTile, c = e - r * kGramTile;
        const long long s = s0 + r;
        As[r][c] = (s < ns && i0 + c < n) ? store[s * n + i0 + c] : 0.0;
        Bs[r][c] = (s < ns && j0 + c < n) ? store[s * n + j0 + c] : 0.0;
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < kGramK; ++k) {
        double av[4], bv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) av[a] = As[k][ty + 16 * a];
#pragma unroll
        for (int b = 0; b < 4; ++b) bv[b] = Bs[k][tx + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) acc[a][b] += av[a] * bv[b];
      }
      __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int i = i0 + ty + 16 * a, j = j0 + tx + 16 * b;
        if (i < n && j < n && i >= j) {
          const double v = acc[a][b] * inv_w;
          oo[static_cast<size_t>(i) * n + j] = v;
          oo[static_cast<size_t>(j) * n + i] = v;
        }
      }
  }
}

// S[si][sj] = OO[pi][pj] − OO[0][pi]·OO[0][pj] (pi = map[si] + 1), diagonal × (1 + sta_del).
__global__ void k_assemble_s(const double* __restrict__ oo, int n, const int* __restrict__ map, int na,
                             double ratio_diag, double* __restrict__ s) {
  const long long total = static_cast<long long>(na) * na;
  for (long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; k < total;
       k += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int si = static_cast<int>(k / na), sj = static_cast<int>(k - static_cast<long long>(si) * na);
    const int pi = map[si] + 1, pj = map[sj] + 1;
    double v = oo[static_cast<size_t>(pi) * n + pj] - oo[pi] * oo[pj];
    if (si == sj) v *= ratio_diag;
    s[k] = v;
  }
}

// S of the active block from the tensor-core Gram of the centred, column-scaled samples
// (G = ÕᵀÕ, FP32, row stride ldg): S_ij = Wc⁻¹·cs_i·G_ij·cs_j, plus sta_del·var_i on the
// diagonal (the same operator the Gram form of SR-CG applies), in FP64.
__global__ void k_assemble_s_gram(const float* __restrict__ g, int ldg, const double* __restrict__ cs,
                                  const double* __restrict__ var, int na, double inv_wc, double sta_del,
                                  double* __restrict__ s) {
  const long long total = static_cast<long long>(na) * na;
  for (long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; k < total;
       k += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(k / na), j = static_cast<int>(k - static_cast<long long>(i) * na);
    double v = inv_wc * (cs[i] * static_cast<double>(g[static_cast<size_t>(i) * ldg + j]) * cs[j]);
    if (i == j) v += sta_del * var[i];
    s[k] = v;
  }
}

// In-place lower Cholesky of the row-major n×n matrix a (the lower triangle is read and
// written). info: 0, or the 1-based row of the first non-positive / non-finite pivot.
__global__ void __launch_bounds__(kCholThreads) k_cholesky(double* __restrict__ a, int n, int* info) {
  cgr::grid_group grid = cgr::this_grid();
  __shared__ double D[kCholB][kCholB + 1];
  __shared__ double Ti[kCholT][kCholB + 1];
  __shared__ double Tj[kCholT][kCholB + 1];
  __shared__ int s_fail;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int k0 = 0; k0 < n; k0 += kCholB) {
    const int kb = min(kCholB, n - k0);
    // (1) diagonal block
    if (blockIdx.x == 0) {
      for (int e = tid; e < kb * kb; e += nt) {
        const int r = e / kb, c = e - r * kb;
        D[r][c] = c <= r ? a[static_cast<size_t>(k0 + r) * n + k0 + c] : 0.0;
      }
      if (tid == 0) s_fail = 0;
      __syncthreads();
      for (int j = 0; j < kb; ++j) {
        if (tid == 0) {
          double d = D[j][j];
          for (int k = 0; k < j; ++k) d -= D[j][k] * D[j][k];
          if (!(d > 0.0) || !isfinite(d)) {
            if (!s_fail) s_fail = k0 + j + 1;
            d = 1.0;
          }
          D[j][j] = sqrt(d);
        }
        __syncthreads();
        for (int i = j + 1 + tid; i < kb; i += nt) {
          double t = D[i][j];
          for (int k = 0; k < j; ++k) t -= D[i][k] * D[j][k];
          D[i][j] = t / D[j][j];
        }
        __syncthreads();
      }
      for (int e = tid; e < kb * kb; e += nt) {
        const int r = e / kb, c = e - r * kb;
        if (c <= r) a[static_cast<size_t>(k0 + r) * n + k0 + c] = D[r][c];
      }
      if (tid == 0 && s_fail && *info == 0) *info = s_fail;
    }
    grid.sync();
    if (*info != 0) return;  // every block reads the same flag after the barrier
    const int rest = n - k0 - kb;
    if (rest <= 0) break;
    // (2) panel rows below: L[i][k0..k0+kb) = A[i][k0..) · D⁻ᵀ
    for (int e = tid; e < kb * kb; e += nt) {
      const int r = e / kb, c = e - r * kb;
      D[r][c] = c <= r ? a[static_cast<size_t>(k0 + r) * n + k0 + c] : 0.0;
    }
    __syncthreads();
    for (int r = blockIdx.x * nt + tid; r < rest; r += gridDim.x * nt) {
      double* row = a + static_cast<size_t>(k0 + kb + r) * n + k0;
      double x[kCholB];
#pragma unroll
      for (int j = 0; j < kCholB; ++j) {
        if (j < kb) {
          double t = row[j];
          for (int k = 0; k < j; ++k) t -= x[k] * D[j][k];
          x[j] = t / D[j][j];
        }
      }
#pragma unroll
      for (int j = 0; j < kCholB; ++j)
        if (j < kb) row[j] = x[j];
    }
    grid.sync();
    // (3) trailing update of the lower triangle in 64×64 tiles (4×4 outputs per thread,
    // the tile's two 64×32 panel slices staged in shared memory)
    const int m = (rest + kCholT - 1) / kCholT;
    const int ntiles = m * (m + 1) / 2;
    const int tr = tid / 16, tc = tid % 16;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      int ti = static_cast<int>((sqrt(8.0 * t + 1.0) - 1.0) / 2.0);
      while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
      while (ti * (ti + 1) / 2 > t) --ti;
      const int tj = t - ti * (ti + 1) / 2;
      const int i0 = k0 + kb + ti * kCholT, j0 = k0 + kb + tj * kCholT;
      for (int e = tid; e < kCholT * kCholB; e += nt) {
        const int r = e / kCholB, c = e - r * kCholB;
        Ti[r][c] = (i0 + r < n && c < kb) ? a[static_cast<size_t>(i0 + r) * n + k0 + c] : 0.0;
        Tj[r][c] = (j0 + r < n && c < kb) ? a[static_cast<size_t>(j0 + r) * n + k0 + c] : 0.0;
      }
      __syncthreads();
      double acc[4][4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = 0.0;
#pragma unroll 8
      for (int k = 0; k < kCholB; ++k) {
        double li[4], lj[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          li[u] = Ti[tr + 16 * u][k];
          lj[u] = Tj[tc + 16 * u][k];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) acc[u][v] += li[u] * lj[v];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const int i = i0 + tr + 16 * u, j = j0 + tc + 16 * v;
          if (i < n && j < n && j <= i) a[static_cast<size_t>(i) * n + j] -= acc[u][v];
        }
      __syncthreads();
    }
    grid.sync();
  }
}

// x = (L Lᵀ)⁻¹ b in place, L the lower factor of k_cholesky; one block.
__global__ void __launch_bounds__(kCholThreads) k_cholesky_solve(const double* __restrict__ l, int n,
                                                                 double* __restrict__ b) {
  __shared__ double part[kCholThreads / kCholB][kCholB];
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
  // forward: L y = b
  for (int k0 = 0; k0 < n; k0 += kCholB) {
    const int kb = min(kCholB, n - k0);
    if (tid < 32) {
      double y = lane < kb ? b[k0 + lane] : 0.0;
      for (int j = 0; j < kb; ++j) {
        if (lane == j) y = y / l[static_cast<size_t>(k0 + j) * n + k0 + j];
        const double yj = __shfl_sync(0xffffffffu, y, j);
        if (lane > j && lane < kb) y -= l[static_cast<size_t>(k0 + lane) * n + k0 + j] * yj;
      }
      if (lane < kb) b[k0 + lane] = y;
    }
    __syncthreads();
    for (int i = k0 + kb + tid; i < n; i += nt) {
      double t = 0.0;
      const double* row = l + static_cast<size_t>(i) * n + k0;
      for (int k = 0; k < kb; ++k) t += row[k] * b[k0 + k];
      b[i] -= t;
    }
    __syncthreads();
  }
  // backward: Lᵀ x = y, blocks from the bottom
  const int nb = (n + kCholB - 1) / kCholB;
  for (int bi = nb - 1; bi >= 0; --bi) {
    const int k0 = bi * kCholB, kb = min(kCholB, n - k0), below = k0 + kb;
    // y_J −= Σ_{i ≥ below} L[i][J] x_i: column j = tid % 32, row groups by tid / 32
    {
      const int j = tid % kCholB, grp = tid / kCholB, ngrp = nt / kCholB;
      double t = 0.0;
      if (j < kb)
        for (int i = below + grp; i < n; i += ngrp) t += l[static_cast<size_t>(i) * n + k0 + j] * b[i];
      part[grp][j] = t;
    }
    __syncthreads();
    if (tid < 32) {
      double x = 0.0;
      if (lane < kb) {
        double t = 0.0;
        for (int g = 0; g < nt / kCholB; ++g) t += part[g][lane];
        x = b[k0 + lane] - t;
      }
      for (int j = kb - 1; j >= 0; --j) {
        if (lane == j) x = x / l[static_cast<size_t>(k0 + j) * n + k0 + j];
        const double xj = __shfl_sync(0xffffffffu, x, j);
        if (lane < j) x -= l[static_cast<size_t>(k0 + j) * n + k0 + lane] * xj;
      }
      if (lane < kb) b[k0 + lane] = x;
    }
    __syncthreads();
  }
}

int launch_gram(const double* store, int n, long long ns, double inv_w, double* oo, cudaStream_t stream) {
  const int ntile = (n + kGramTile - 1) / kGramTile;
  const int tiles = ntile * (ntile + 1) / 2;
  k_gram<<<std::max(1, std::min(tiles, 148 * 8)), 256, 0, stream>>>(store, n, ns, inv_w, oo);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

int launch_assemble_s(const double* oo, int n, const int* map, int na, double ratio_diag, double* s,
                      cudaStream_t stream) {
  const long long total = static_cast<long long>(na) * na;
  const int grid = static_cast<int>(std::max<long long>(1, std::min<long long>((total + 255) / 256, 148LL * 16)));
  k_assemble_s<<<grid, 256, 0, stream>>>(oo, n, map, na, ratio_diag, s);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

int launch_assemble_s_gram(const float* g, int ldg, const double* cs, const double* var, int na, double inv_wc,
                           double sta_del, double* s, cudaStream_t stream) {
  const long long total = static_cast<long long>(na) * na;
  const int grid = static_cast<int>(std::max<long long>(1, std::min<long long>((total + 255) / 256, 148LL * 16)));
  k_assemble_s_gram<<<grid, 256, 0, stream>>>(g, ldg, cs, var, na, inv_wc, sta_del, s);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

// Factor a (n×n, device) and solve for b (device) in place; *info_dev set on failure.
int launch_cholesky_solve(double* a, int n, double* b, int* info_dev, cudaStream_t stream) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  MVMCB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cholesky, kCholThreads, 0));
  const int m = (n + kCholB - 1) / kCholB;
  const int blocks = std::max(1, std::min(sms * std::max(1, std::min(per, 2)), m * (m + 1) / 2));
  MVMCB_CUDA(cudaMemsetAsync(info_dev, 0, sizeof(int), stream));
  void* args[] = {&a, &n, &info_dev};
  MVMCB_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_cholesky), blocks, kCholThreads, args, 0, stream));
  k_cholesky_solve<<<1, kCholThreads, 0, stream>>>(a, n, b);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

}  // namespace mvmcb

namespace {
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};
}  // namespace

// SrStages::gram_real (sr_backend.rs:464): out = Σ_s store[s]·store[s]ᵀ (host buffers;
// store rows of n values, samples rows).
extern "C" int mvmc_b200_gram(const double* store, int n, long long samples, double* out) {
  using namespace mvmcb;
  if (!store || !out || n <= 0 || samples < 0) return kErrArgument;
  DevBuf s, o;
  MVMCB_CUDA(cudaMalloc(&s.p, sizeof(double) * std::max<long long>(1, samples * n)));
  MVMCB_CUDA(cudaMalloc(&o.p, sizeof(double) * static_cast<size_t>(n) * n));
  if (samples > 0) MVMCB_CUDA(cudaMemcpy(s.p, store, sizeof(double) * samples * n, cudaMemcpyHostToDevice));
  const int rc = launch_gram(static_cast<double*>(s.p), n, samples, 1.0, static_cast<double*>(o.p), nullptr);
  if (rc != kOk) return rc;
  MVMCB_CUDA(cudaMemcpy(out, o.p, sizeof(double) * static_cast<size_t>(n) * n, cudaMemcpyDeviceToHost));
  return kOk;
}

// SrStages::cholesky_solve (sr_backend.rs:243-247): solve S x = rhs for the symmetric
// positive-definite row-major S (host buffers); rhs becomes x. Returns 1 when the
// factorisation meets a non-positive pivot or the solution is not finite (the reference's
// Err(())), 0 on success, < 0 on argument / CUDA errors.
extern "C" int mvmc_b200_cholesky_solve(const double* s, double* rhs, int n) {
  using namespace mvmcb;
  if (!s || !rhs || n <= 0) return kErrArgument;
  DevBuf a, b, info;
  MVMCB_CUDA(cudaMalloc(&a.p, sizeof(double) * static_cast<size_t>(n) * n));
  MVMCB_CUDA(cudaMalloc(&b.p, sizeof(double) * n));
  MVMCB_CUDA(cudaMalloc(&info.p, sizeof(int)));
  MVMCB_CUDA(cudaMemcpy(a.p, s, sizeof(double) * static_cast<size_t>(n) * n, cudaMemcpyHostToDevice));
  MVMCB_CUDA(cudaMemcpy(b.p, rhs, sizeof(double) * n, cudaMemcpyHostToDevice));
  const int rc = launch_cholesky_solve(static_cast<double*>(a.p), n, static_cast<double*>(b.p),
                                       static_cast<int*>(info.p), nullptr);
  if (rc != kOk) return rc;
  int h_info = 0;
  MVMCB_CUDA(cudaMemcpy(&h_info, info.p, sizeof(int), cudaMemcpyDeviceToHost));
  MVMCB_CUDA(cudaMemcpy(rhs, b.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (h_info != 0) return 1;
  for (int i = 0; i < n; ++i)
    if (!std::isfinite(rhs[i])) return 1;
  return kOk;
}
