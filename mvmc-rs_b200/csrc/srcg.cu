// K5: SR-CG on the device.
//
// SampledSrOperator::solve_with_product (crates/mvmc-core/src/sr_cg.rs:700-880 of
// AtelierArith/mvmc-rs) with the C recurrence: threshold tol²·n², δ = β·δ (plain) or
// δ = δ_new (DiagScale), r = g − S·x at every 20th iteration, breakdown |d·q| < 1e-20,
// status = iterations or −(iter+1). S·v = Oᵀ(O·v)/W − (⟨O⟩·v)⟨O⟩ + δ_shift·diag·v
// (apply_with_product, sr_cg.rs:952-1009; COrderSr::cg_local_product,
// sr_backend.rs:518-606) over the compact active sample matrix O[s][i].
// One cooperative launch runs every iteration: no host round trip until the solve ends.
// Every reduction has a fixed order, so the recurrence is bitwise repeatable.
//
// The product reads O once per application: each block owns a contiguous range of
// sample rows and takes them R at a time into registers (thread t holds columns
// t, t + T, ...); a block-wide sum gives the R row products y_s = O_s·v, and the same
// registers accumulate Σ_s y_s·O_s into per-thread column sums. The per-block column
// partials are then summed across blocks in block order.
//
// Reduced-precision operator (mixed path): the active matrix is stored centred and
// column-scaled in FP32 or BF16 (half or a quarter of the FP64 bytes, so that at the SR
// configurations it stays in L2 across iterations) and the products accumulate in FP32;
// vectors, dots and the α/β recurrence stay FP64. As a matrix-vector pair at ≤ 1 flop per
// byte this form is bound by memory bandwidth on the CUDA cores. The Gram form (o_kind 3)
// moves the contraction to the tensor cores instead: G = OlᵀOl is formed once per SR step
// (gram_tc.cu, tcgen05.mma on BF16 or TF32 inputs) and every iteration then applies the
// L2-resident na × na G, one warp per row.
#include <cooperative_groups.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <type_traits>

#include "../host/abi_common.h"
#include "common.cuh"
#include "engine.cuh"

namespace cgr = cooperative_groups;

namespace mvmcb {

constexpr int kCgThreads = 512;   // one block of 16 warps per SM
constexpr int kCgMaxCols = 16;    // columns per thread: na ≤ kCgThreads · kCgMaxCols

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

// Sum of the per-block partials red[0..gridDim) in a fixed order (lane l adds blocks l,
// l+32, …, then a fixed shuffle tree), computed by warp 0 and broadcast through sh[33]:
// every block gets the same bits. red must be complete (after a grid barrier).
__device__ double blocks_total(const double* red, double* sh) {
  if (threadIdx.x < 32) {
    double t = 0.0;
    for (int k = threadIdx.x; k < static_cast<int>(gridDim.x); k += 32) t += red[k];
    t = warp_sum(t);
    if (threadIdx.x == 0) sh[33] = t;
  }
  __syncthreads();
  const double t = sh[33];
  __syncthreads();
  return t;
}

// Grid-wide sum of one value per thread into slot `red` (gridDim doubles): block sum, one
// grid barrier, fixed-order total. The slot may be written again only after a later grid
// barrier that every block passes after reading it.
__device__ double grid_sum(cgr::grid_group& grid, double v, double* red, double* sh) {
  v = block_sum(v, sh);
  if (threadIdx.x == 0) red[blockIdx.x] = v;
  grid.sync();
  return blocks_total(red, sh);
}

// Grid-wide deterministic dot: every block gets the same value.
__device__ double grid_dot(cgr::grid_group& grid, const double* a, const double* b, int n,
                           double* red, double* sh) {
  double v = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v += a[i] * b[i];
  const double t = grid_sum(grid, v, red, sh);
  grid.sync();
  return t;
}

// Element access of the stored sample matrix: FP64 (C order), FP32 or BF16.
template <typename OT>
struct Elem;
template <>
struct Elem<double> {
  using CT = double;
  __device__ static double load(const double* p) { return __ldg(p); }
};
template <>
struct Elem<float> {
  using CT = float;
  __device__ static float load(const float* p) { return __ldg(p); }
};
template <>
struct Elem<__nv_bfloat16> {
  using CT = float;
  __device__ static float load(const __nv_bfloat16* p) { return __bfloat162float(*p); }
};

// R block sums at once: sh needs 32·R + R doubles.
template <int R>
__device__ void block_sum_vec(double (&v)[R], double* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = warp_sum(v[r]);
  if (lane == 0) {
#pragma unroll
    for (int r = 0; r < R; ++r) sh[warp * R + r] = v[r];
  }
  __syncthreads();
  if (threadIdx.x < R) {
    double t = 0.0;
    for (int w = 0; w < nwarp; ++w) t += sh[w * R + threadIdx.x];
    sh[32 * R + threadIdx.x] = t;
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = sh[32 * R + r];
  __syncthreads();
}

// Rows per register batch for KC columns per thread.
template <int KC>
struct RowBatch {
  static constexpr int R = KC <= 2 ? 8 : (KC <= 4 ? 4 : (KC <= 8 ? 2 : 1));
};

// out = S·v. FP64: Oᵀ(O·v)/Wc − (⟨O⟩·v)⟨O⟩ + shift·diag ⊙ v. Reduced precision (centred,
// scaled rows): cs ⊙ Olᵀ(Ol·(cs ⊙ v))/Wc + shift·diag ⊙ v.
// v may be in global or shared memory; out (global) gets S·v; returns v·(S·v), the same in
// every block. Two grid barriers: after the column partials and after the dot partials.
template <typename OT, int KC>
__device__ double sr_apply_rows(cgr::grid_group& grid, const CgArgs& a, const double* v, double* out, double* red,
                                double* sh, unsigned char* smem) {
  using CT = typename Elem<OT>::CT;
  constexpr int R = RowBatch<KC>::R;
  constexpr bool kLow = !std::is_same<OT, double>::value;
  CT* vs = reinterpret_cast<CT*>(smem + sizeof(double) * static_cast<size_t>(a.na));
  const int tid = threadIdx.x, nt = blockDim.x, na = a.na;
  for (int i = tid; i < na; i += nt) vs[i] = kLow ? static_cast<CT>(a.cs[i] * v[i]) : static_cast<CT>(v[i]);
  __syncthreads();
  // ⟨O⟩·v, the same value in every block (fixed order)
  double coef = 0.0;
  if (!kLow) {
    double t = 0.0;
    for (int i = tid; i < na; i += nt) t += a.mean[i] * v[i];
    coef = block_sum(t, sh);
  }
  const OT* O = kLow ? static_cast<const OT*>(a.Ol) : reinterpret_cast<const OT*>(a.O);
  const long long lda = kLow ? a.lda : na;
  const long long per = (a.ns + gridDim.x - 1) / gridDim.x;
  const long long s0 = static_cast<long long>(blockIdx.x) * per, s1 = min(a.ns, s0 + per);
  double z[KC];
#pragma unroll
  for (int k = 0; k < KC; ++k) z[k] = 0.0;
  if constexpr (R == 1) {
    // wide rows: chunks of one row per warp; each warp forms y_s = O_s·v of its row with a
    // shuffle sum (no block barrier per row), then every thread adds y_s·O_s of the chunk's
    // rows to its columns (the second read of a row comes from L2). One block barrier per
    // chunk; the chunk's y values are double-buffered.
    __shared__ double ych[2][kCgThreads / 32];
    const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    int buf = 0;
    for (long long sb = s0; sb < s1; sb += nw, buf ^= 1) {
      const long long s = sb + warp;
      if (s < s1) {
        const OT* row = O + s * lda;
        // sixteen loads in flight per lane: the row streams from memory at full rate
        constexpr int U = 16;
        double t[4] = {0.0, 0.0, 0.0, 0.0};
        int i = lane;
        for (; i + 32 * (U - 1) < na; i += 32 * U) {
          CT x[U];
#pragma unroll
          for (int u = 0; u < U; ++u) x[u] = Elem<OT>::load(row + i + 32 * u);
#pragma unroll
          for (int u = 0; u < U; ++u) t[u & 3] += static_cast<double>(x[u] * vs[i + 32 * u]);
        }
        for (; i < na; i += 32) t[0] += static_cast<double>(Elem<OT>::load(row + i) * vs[i]);
        const double y = warp_sum((t[0] + t[1]) + (t[2] + t[3]));
        if (lane == 0) ych[buf][warp] = y;
      }
      __syncthreads();
      const int rows = static_cast<int>(min(static_cast<long long>(nw), s1 - sb));
#pragma unroll 2
      for (int r = 0; r < rows; ++r) {
        const double yv = ych[buf][r];
        const OT* row = O + (sb + r) * lda;
#pragma unroll
        for (int k = 0; k < KC; ++k) {
          const int i = tid + k * nt;
          if (i < na) z[k] += static_cast<double>(Elem<OT>::load(row + i)) * yv;
        }
      }
    }
  } else
  for (long long sb = s0; sb < s1; sb += R) {
    CT x[R][KC];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const long long s = sb + r;
#pragma unroll
      for (int k = 0; k < KC; ++k) {
        const int i = tid + k * nt;
        x[r][k] = (s < s1 && i < na) ? Elem<OT>::load(O + s * lda + i) : CT(0);
      }
    }
    double y[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      CT t = CT(0);
#pragma unroll
      for (int k = 0; k < KC; ++k) {
        const int i = tid + k * nt;
        if (i < na) t += x[r][k] * vs[i];
      }
      y[r] = static_cast<double>(t);
    }
    block_sum_vec<R>(y, sh);
#pragma unroll
    for (int r = 0; r < R; ++r) {
#pragma unroll
      for (int k = 0; k < KC; ++k) z[k] += static_cast<double>(x[r][k]) * y[r];
    }
  }
  double* part = a.part + static_cast<long long>(blockIdx.x) * na;
#pragma unroll
  for (int k = 0; k < KC; ++k) {
    const int i = tid + k * nt;
    if (i < na) part[i] = z[k];
  }
  grid.sync();
  // Column totals over the blocks: tiles of 64 columns, each column's block partials split
  // over nt/64 threads (loads in flight together), the sub-sums added in order.
  __shared__ double ssub[kCgThreads];
  const int nsub = nt / 64, nb = static_cast<int>(gridDim.x), bper = (nb + nsub - 1) / nsub;
  const int cl = tid & 63, sub = tid >> 6, b0 = sub * bper, b1 = min(nb, b0 + bper);
  double dot = 0.0;
  for (int tile = blockIdx.x; tile * 64 < na; tile += gridDim.x) {
    const int col = tile * 64 + cl;
    double t = 0.0;
    if (col < na) {
#pragma unroll 4
      for (int b = b0; b < b1; ++b) t += a.part[static_cast<long long>(b) * na + col];
    }
    ssub[sub * 64 + cl] = t;
    __syncthreads();
    if (tid < 64 && col < na) {
      double tot = 0.0;
      for (int u = 0; u < nsub; ++u) tot += ssub[u * 64 + tid];
      const double o = kLow ? a.inv_w * (a.cs[col] * tot) + a.shift * a.diag[col] * v[col]
                            : a.inv_w * tot - coef * a.mean[col] + a.shift * a.diag[col] * v[col];
      out[col] = o;
      dot += v[col] * o;
    }
    __syncthreads();
  }
  return grid_sum(grid, dot, red, sh);
}

template <typename OT, int KC>
struct ApplyRows {
  double* sh;
  unsigned char* smem;
  __device__ double operator()(cgr::grid_group& g, const CgArgs& a, const double* v, double* out, double* red) const {
    return sr_apply_rows<OT, KC>(g, a, v, out, red, sh, smem);
  }
};

__device__ __forceinline__ double precond(const CgArgs& a, int i, double r) {
  double dq = (1.0 + a.shift) * a.diag[i];
  if (!isfinite(dq) || fabs(dq) < 1e-12) dq = dq < 0.0 ? -1e-12 : 1e-12;
  return r / dq;
}

// The C recurrence around an S·v product (apply), three grid barriers per iteration: the
// product's column partials, its dot d·(S·d) with the product itself, and the residual
// update with the new δ. Every block keeps the whole direction d in shared memory (dsh) and
// forms the next one itself from the published residual, so d is never exchanged; x, r and
// the preconditioned residual (kept in q) are updated by their owning threads.
template <typename Apply>
__device__ void cg_run(cgr::grid_group& grid, const CgArgs& a, double* sh, double* dsh, const Apply& apply) {
  const int n = a.na, tid = threadIdx.x, nt = blockDim.x;
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstride = gridDim.x * blockDim.x;
  const double threshold = a.tol * a.tol * static_cast<double>(n) * static_cast<double>(n);
  double* red0 = a.red;               // slot of the product's dot
  double* red1 = a.red + gridDim.x;   // slot of δ
  double delta;
  for (int i = gtid; i < n; i += gstride) {
    a.x[i] = 0.0;
    a.r[i] = a.g[i];
  }
  grid.sync();
  if (a.diag_scale) {
    apply(grid, a, a.x, a.q, red0);
    for (int i = gtid; i < n; i += gstride) {
      a.r[i] = a.g[i] - a.q[i];
      a.q[i] = precond(a, i, a.r[i]);
    }
    grid.sync();
    delta = grid_dot(grid, a.r, a.q, n, a.red, sh);
  } else {
    delta = grid_dot(grid, a.r, a.r, n, a.red, sh);
  }
  const double* zsrc = a.diag_scale ? a.q : a.r;
  for (int i = tid; i < n; i += nt) dsh[i] = zsrc[i];
  __syncthreads();
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
    const double dq = apply(grid, a, dsh, a.q, red0);
    if (!isfinite(dq) || fabs(dq) < 1e-20) { status = failed; done = true; break; }
    const double alpha = delta / dq;
    if (!isfinite(alpha)) { status = failed; done = true; break; }
    const bool refresh = (iter + 1) % 20 == 0;
    double part = 0.0;
    for (int i = gtid; i < n; i += gstride) {
      a.x[i] += alpha * dsh[i];
      if (!refresh) {
        const double ri = a.r[i] - alpha * a.q[i];
        a.r[i] = ri;
        const double zi = a.diag_scale ? precond(a, i, ri) : ri;
        if (a.diag_scale) a.q[i] = zi;
        part += ri * zi;
      }
    }
    if (refresh) {
      grid.sync();  // x complete
      apply(grid, a, a.x, a.q, red0);
      for (int i = gtid; i < n; i += gstride) {
        const double ri = a.g[i] - a.q[i];
        a.r[i] = ri;
        const double zi = a.diag_scale ? precond(a, i, ri) : ri;
        if (a.diag_scale) a.q[i] = zi;
        part += ri * zi;
      }
    }
    const double delta_new = grid_sum(grid, part, red1, sh);
    if (!isfinite(delta_new) || fabs(delta) < 1e-20) { status = failed; done = true; break; }
    const double beta = delta_new / delta;
    if (!isfinite(beta)) { status = failed; done = true; break; }
    if (a.diag_scale) delta = delta_new;
    else delta *= beta;
    for (int i = tid; i < n; i += nt) dsh[i] = zsrc[i] + beta * dsh[i];
    __syncthreads();
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


// Gram form (o_kind 3): out = Wc⁻¹·cs ⊙ (G·(cs ⊙ v)) + shift·diag ⊙ v with G = ÕᵀÕ formed once
// on the tensor cores (FP32, na × na, row stride lda). One warp per row of G (FP64
// accumulation, lanes then shuffles in a fixed order), rows strided over the grid.
__device__ double sr_apply_gram(cgr::grid_group& grid, const CgArgs& a, const double* v, double* out, double* red,
                                double* sh, unsigned char* smem) {
  double* u = reinterpret_cast<double*>(smem + sizeof(double) * static_cast<size_t>(a.na));
  const int tid = threadIdx.x, nt = blockDim.x, na = a.na, lane = tid & 31;
  for (int i = tid; i < na; i += nt) u[i] = a.cs[i] * v[i];
  __syncthreads();
  const float* G = static_cast<const float*>(a.Ol);
  const int gw = (blockIdx.x * nt + tid) >> 5, nw = (gridDim.x * nt) >> 5;
  double dot = 0.0;
  for (int i = gw; i < na; i += nw) {
    const float* row = G + static_cast<long long>(i) * a.lda;
    // sixteen loads in flight per lane (G is read from L2)
    constexpr int U = 16;
    double tt[4] = {0.0, 0.0, 0.0, 0.0};
    int j = lane;
    for (; j + 32 * (U - 1) < na; j += 32 * U) {
      float g[U];
#pragma unroll
      for (int k = 0; k < U; ++k) g[k] = __ldg(row + j + 32 * k);
#pragma unroll
      for (int k = 0; k < U; ++k) tt[k & 3] += static_cast<double>(g[k]) * u[j + 32 * k];
    }
    for (; j < na; j += 32) tt[0] += static_cast<double>(__ldg(row + j)) * u[j];
    const double t = warp_sum((tt[0] + tt[1]) + (tt[2] + tt[3]));
    if (lane == 0) {
      const double o = a.inv_w * (a.cs[i] * t) + a.shift * a.diag[i] * v[i];
      out[i] = o;
      dot += v[i] * o;
    }
  }
  return grid_sum(grid, dot, red, sh);
}

struct ApplyGram {
  double* sh;
  unsigned char* smem;
  __device__ double operator()(cgr::grid_group& g, const CgArgs& a, const double* v, double* out, double* red) const {
    return sr_apply_gram(g, a, v, out, red, sh, smem);
  }
};

__global__ void __launch_bounds__(kCgThreads, 1) k_sr_cg_gram(CgArgs a) {
  cgr::grid_group grid = cgr::this_grid();
  __shared__ double sh[32 * 8 + 8 + 8];
  extern __shared__ __align__(16) unsigned char smem[];
  cg_run(grid, a, sh, reinterpret_cast<double*>(smem), ApplyGram{sh, smem});
}

template <typename OT, int KC>
__global__ void __launch_bounds__(kCgThreads, 1) k_sr_cg(CgArgs a) {
  cgr::grid_group grid = cgr::this_grid();
  __shared__ double sh[32 * 8 + 8 + 8];
  extern __shared__ __align__(16) unsigned char smem[];
  if (a.nchunk < static_cast<int>(gridDim.x)) {  // partial buffer too small: refuse
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      a.scal[0] = 0.0;
      a.scal[1] = -1.0;
      a.scal[2] = 0.0;
    }
    return;
  }
  cg_run(grid, a, sh, reinterpret_cast<double*>(smem), ApplyRows<OT, KC>{sh, smem});
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

// Local sampled product of a rank's samples (SrStages::cg_local_product,
// sr_backend.rs:249-255): z = Σ_s O_s (O_s · v), no mean, diagonal or cross-rank terms.
// y[s] = O_s·v by one warp per row; per-chunk column sums; the chunks added in order.
__global__ void k_local_rowdot(const double* __restrict__ oa, long long ns, int na, const double* __restrict__ v,
                               double* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const long long gw = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const long long nw = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
  for (long long s = gw; s < ns; s += nw) {
    double t = 0.0;
    for (int i = lane; i < na; i += 32) t += oa[s * na + i] * v[i];
    t = warp_sum(t);
    if (lane == 0) y[s] = t;
  }
}

__global__ void k_local_colpart(const double* __restrict__ oa, long long ns, int na, const double* __restrict__ y,
                                int nchunk, double* __restrict__ part) {
  const int ntile = (na + blockDim.x - 1) / blockDim.x;
  const long long chunk = (ns + nchunk - 1) / nchunk;
  for (int item = blockIdx.x; item < ntile * nchunk; item += gridDim.x) {
    const int tile = item % ntile, c = item / ntile;
    const int i = tile * blockDim.x + threadIdx.x;
    if (i >= na) continue;
    const long long s0 = c * chunk, s1 = min(ns, s0 + chunk);
    double t = 0.0;
    for (long long s = s0; s < s1; ++s) t += oa[s * na + i] * y[s];
    part[static_cast<long long>(c) * na + i] = t;
  }
}

__global__ void k_local_colsum(const double* __restrict__ part, int nchunk, int na, double* __restrict__ z) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < na; i += gridDim.x * blockDim.x) {
    double t = 0.0;
    for (int c = 0; c < nchunk; ++c) t += part[static_cast<long long>(c) * na + i];
    z[i] = t;
  }
}

int local_product_chunks(long long ns, int na) {
  const int ntile = (na + 255) / 256;
  return static_cast<int>(std::max<long long>(1, std::min<long long>(ns, std::max(1, 592 / ntile))));
}

// y: ns doubles, part: local_product_chunks(ns, na)·na doubles (device).
int launch_local_product(const double* oa, long long ns, int na, const double* v, double* z, double* y,
                         double* part, cudaStream_t stream) {
  const int nchunk = local_product_chunks(ns, na);
  const int rows_grid = static_cast<int>(std::max<long long>(1, std::min<long long>((ns + 7) / 8, 148LL * 16)));
  k_local_rowdot<<<rows_grid, 256, 0, stream>>>(oa, ns, na, v, y);
  const int ntile = (na + 255) / 256;
  k_local_colpart<<<std::max(1, std::min(ntile * nchunk, 148 * 8)), 256, 0, stream>>>(oa, ns, na, y, nchunk, part);
  k_local_colsum<<<std::max(1, (na + 255) / 256), 256, 0, stream>>>(part, nchunk, na, z);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

// One block per SM of the current device (co-resident for the cooperative launch).
int cg_grid_blocks(long long ns, int na) {
  (void)ns;
  (void)na;
  return std::max(1, current_device_attr(cudaDevAttrMultiProcessorCount));
}

int cg_grid_blocks_kind(long long ns, int na, int kind) {
  (void)kind;
  return cg_grid_blocks(ns, na);
}

// Column partial rows (part[nchunk][na]): one per block.
int cg_nchunk(long long ns, int na, int kind, int blocks) {
  (void)ns;
  (void)na;
  (void)kind;
  return blocks;
}

int low_lda(int na, int kind) {
  (void)kind;
  return na;
}

template <typename OT>
__device__ __forceinline__ OT to_low(double v);
template <>
__device__ __forceinline__ float to_low<float>(double v) {
  return static_cast<float>(v);
}
template <>
__device__ __forceinline__ __nv_bfloat16 to_low<__nv_bfloat16>(double v) {
  return __float2bfloat16_rn(static_cast<float>(v));
}

// Ol[s][i] = (store[s][map[i] + 1] − mean[i]) / cs[i]; zero for skipped samples (their
// stored row is zero, leading 1 included).
template <typename OT>
__global__ void k_gather_active_low(const double* __restrict__ store, int sr_size, long long ns,
                                    const int* __restrict__ map, int na, int lda, const double* __restrict__ mean,
                                    const double* __restrict__ cs, OT* __restrict__ out) {
  const long long total = ns * lda;
  for (long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; k < total;
       k += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long s = k / lda;
    const int si = static_cast<int>(k - s * lda);
    double v = 0.0;
    if (si < na && store[s * sr_size] != 0.0) v = (store[s * sr_size + map[si] + 1] - mean[si]) / cs[si];
    out[k] = to_low<OT>(v);
  }
}

int launch_gather_active_low(const double* store, int sr_size, long long ns, const int* map, int na,
                             const double* mean, const double* cs, int kind, void* out, cudaStream_t stream) {
  const int lda = low_lda(na, kind);
  const long long total = ns * lda;
  const int grid = static_cast<int>(std::max<long long>(1, std::min<long long>((total + 255) / 256, 148LL * 32)));
  if (kind == 1)
    k_gather_active_low<float><<<grid, 256, 0, stream>>>(store, sr_size, ns, map, na, lda, mean, cs,
                                                          static_cast<float*>(out));
  else
    k_gather_active_low<__nv_bfloat16><<<grid, 256, 0, stream>>>(store, sr_size, ns, map, na, lda, mean, cs,
                                                                  static_cast<__nv_bfloat16*>(out));
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

template <typename OT, int KC>
int launch_cg_kc(CgArgs& a, cudaStream_t stream) {
  void* args[] = {&a};
  // the direction d (FP64) and the staged product input (element type)
  const size_t smem = (sizeof(double) + sizeof(typename Elem<OT>::CT)) * static_cast<size_t>(a.na);
  auto kernel = k_sr_cg<OT, KC>;
  MVMCB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  MVMCB_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(kernel), cg_grid_blocks(a.ns, a.na), kCgThreads,
                                         args, smem, stream));
  return kOk;
}

template <typename OT>
int launch_cg_type(CgArgs& a, cudaStream_t stream) {
  const int kc = (a.na + kCgThreads - 1) / kCgThreads;
  if (kc <= 1) return launch_cg_kc<OT, 1>(a, stream);
  if (kc <= 2) return launch_cg_kc<OT, 2>(a, stream);
  if (kc <= 4) return launch_cg_kc<OT, 4>(a, stream);
  if (kc <= 8) return launch_cg_kc<OT, 8>(a, stream);
  if (kc <= kCgMaxCols) return launch_cg_kc<OT, kCgMaxCols>(a, stream);
  set_last_error("sr-cg: more than " + std::to_string(kCgThreads * kCgMaxCols) + " active parameters");
  return kErrArgument;
}

int launch_sr_cg(CgArgs a, cudaStream_t stream) {
  if (a.o_kind == 3) {  // Gram form: G (FP32) in a.Ol, no sample pass per iteration
    void* args[] = {&a};
    const size_t smem = 2 * sizeof(double) * static_cast<size_t>(a.na);
    MVMCB_CUDA(cudaFuncSetAttribute(k_sr_cg_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    MVMCB_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_sr_cg_gram), cg_grid_blocks(a.ns, a.na),
                                           kCgThreads, args, smem, stream));
    return kOk;
  }
  if (a.nchunk < cg_grid_blocks(a.ns, a.na)) {
    set_last_error("sr-cg: partial buffer holds fewer rows than the grid has blocks");
    return kErrArgument;
  }
  if (a.o_kind == 1) return launch_cg_type<float>(a, stream);
  if (a.o_kind == 2) return launch_cg_type<__nv_bfloat16>(a, stream);
  return launch_cg_type<double>(a, stream);
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
  const int nchunk = cg_nchunk(ns, na, 0, blocks);
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
