// K1: batched skew Pfaffian + inverse (PfaffianStages::pfaffian_inverse_batch).
//
// One CTA per plane. Planes with n ≤ 128 are swept in registers (k_pfinv_reg); larger
// planes up to the shared-memory limit are swept in shared memory (ping-pong, or row stride
// n+1 to spread banks); larger FP64 planes are swept in place in the output buffer
// (L2-resident working set). Input and output are column-major as in
// crates/mvmc-core/src/stage_backend.rs:121-165; the returned inverse is the true X⁻¹.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <map>
#include <cstring>
#include <cstdlib>
#include <cstdio>
#include <vector>

#include "../../include/mvmc_b200.h"
#include "common.cuh"
#include "pfinv.cuh"

namespace mvmcb {

constexpr int kPfinvThreads = 256;
int device_sm_count();
int pfinv_complex_device(const double* x, int n, int planes, double* pf, double* inv, int* status,
                         cudaStream_t stream);

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

// Register-resident sweep for n ≤ G·R: thread (tr, tc) of a G×G block owns the R×R
// elements (tr + G·a, tc + G·b) in registers, so every element update is two FMAs on
// registers. A pivot step needs only rows p and q: the G threads holding the next pivot
// row p publish it in shared memory together with its pivot search (first maximum of
// |A[p][j]| over unswept j, a shuffle reduction inside their warp), the pivot A[p][q], its
// reciprocal and the parity increment; the threads holding row q publish it after the
// first barrier. Two barriers per pivot; buffers are double-buffered by step parity; the
// swept set is a 128-bit mask kept identically by every thread.
template <typename T, int G, int R>
__global__ void __launch_bounds__(G * G, (G == 8 ? (sizeof(T) == 8 ? 4 : 6) : (G == 16 ? (R >= 8 ? 1 : (sizeof(T) == 8 ? 3 : 4)) : 1)))
    k_pfinv_reg(const double* __restrict__ x, const int* __restrict__ sizes,
                const long long* __restrict__ offsets, int n_uniform, int planes, int n_max,
                double* __restrict__ pf, double* __restrict__ inv, int* __restrict__ status) {
  static_assert(G * R <= 128, "the swept mask holds 128 indices");
  static_assert(G == 8 || G == 16 || G == 32, "a thread row is a quarter, half or whole warp");
  extern __shared__ __align__(16) unsigned char smem[];
  T* stage = reinterpret_cast<T*>(smem);                         // [n][n + 1]
  T* rows = stage + static_cast<size_t>(n_max) * (n_max + 1);  // rowp[2][n_max], rowq[2][n_max]
  __shared__ int s_q[2], s_par[2];
  __shared__ T s_av[2], s_ia[2];
  const int tid = threadIdx.x, nt = blockDim.x, tr = tid / G, tc = tid % G;
  const unsigned segmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (tid & (32 - G)));
  for (int plane = blockIdx.x; plane < planes; plane += gridDim.x) {
    const int n = sizes ? sizes[plane] : n_uniform;
    const long long off = offsets ? offsets[plane] : static_cast<long long>(plane) * n * n;
    const double* xp = x + off;
    double* ip = inv + off;
    const int lda = n + 1;
    {
      int i = tid / n, j = tid - (tid / n) * n;
      const int di = nt / n, dj = nt - (nt / n) * n;
      for (int k = tid; k < n * n; k += nt) {
        stage[i * lda + j] = static_cast<T>(-xp[k]);
        i += di;
        j += dj;
        if (j >= n) {
          j -= n;
          ++i;
        }
      }
    }
    __syncthreads();
    T e[R][R];
#pragma unroll
    for (int a = 0; a < R; ++a)
#pragma unroll
      for (int b = 0; b < R; ++b) {
        const int i = tr + G * a, j = tc + G * b;
        e[a][b] = (i < n && j < n) ? stage[i * lda + j] : T(0);
      }
    unsigned long long sw0 = 0ull, sw1 = 0ull;  // swept indices 0..63, 64..127
    auto is_swept = [&](int j) { return ((j < 64 ? sw0 >> j : sw1 >> (j - 64)) & 1ull) != 0ull; };
    // the threads holding row r publish it into buffer buf with its pivot search
    auto publish = [&](int r, int buf) {
      const int ar = r / G;
      T* dst = rows + buf * n_max;
      double best = -1.0;
      int bi = n;
      T bval = T(0);
#pragma unroll
      for (int a = 0; a < R; ++a) {
        if (a != ar) continue;
#pragma unroll
        for (int b = 0; b < R; ++b) {
          const int j = tc + G * b;
          if (j >= n) continue;
          dst[j] = e[a][b];
          if (j != r && !is_swept(j)) {
            const double v = fabs(static_cast<double>(e[a][b]));
            if (v > best) {
              best = v;
              bi = j;
              bval = e[a][b];
            }
          }
        }
      }
#pragma unroll
      for (int o = G / 2; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(segmask, best, o);
        const int oi = __shfl_xor_sync(segmask, bi, o);
        const T oval = __shfl_xor_sync(segmask, bval, o);
        if (ov > best || (ov == best && oi < bi)) {
          best = ov;
          bi = oi;
          bval = oval;
        }
      }
      if (tc == 0) {
        const bool ok = best > 0.0;
        s_q[buf] = ok ? bi : n;
        s_av[buf] = bval;
        s_ia[buf] = ok ? T(1) / bval : T(0);
        int cnt = 0;  // unswept indices strictly between r and q
#pragma unroll
        for (int w = 0; w < 2; ++w) {
          const int lo = max(r + 1, 64 * w), hi = min(bi, 64 * w + 64);
          if (ok && lo < hi) {
            const int len = hi - lo;
            const unsigned long long range = (len == 64 ? ~0ull : ((1ull << len) - 1ull)) << (lo - 64 * w);
            cnt += __popcll(~(w == 0 ? sw0 : sw1) & range);
          }
        }
        s_par[buf] = cnt;
      }
    };
    if (tr == 0) publish(0, 0);
    int p = 0, parity = 0, st = 0;
    double pfv = 1.0;
    for (int k = 0; k < n / 2; ++k) {
      const int par = k & 1;
      const T* rp = rows + par * n_max;
      T* rq = rows + (2 + par) * n_max;
      __syncthreads();  // row p and its pivot published
      const int q = s_q[par];
      if (q >= n) {
        st = p + 1;
        break;
      }
      const T av = s_av[par], ia = s_ia[par];
      parity += s_par[par];
      pfv *= static_cast<double>(av);
      if (tr == q % G) {
        const int aq = q / G;
#pragma unroll
        for (int a = 0; a < R; ++a) {
          if (a != aq) continue;
#pragma unroll
          for (int b = 0; b < R; ++b) {
            const int j = tc + G * b;
            if (j < n) rq[j] = e[a][b];
          }
        }
      }
      __syncthreads();  // row q published
      // rank-2 update of every element (rows and columns p, q are overwritten below)
      T rpj[R], rqj[R];
#pragma unroll
      for (int b = 0; b < R; ++b) {
        const int j = tc + G * b;
        rpj[b] = j < n ? rp[j] : T(0);
        rqj[b] = j < n ? rq[j] : T(0);
      }
#pragma unroll
      for (int a = 0; a < R; ++a) {
        const int i = tr + G * a;
        const T rpi = i < n ? rp[i] * ia : T(0), rqi = i < n ? rq[i] * ia : T(0);
#pragma unroll
        for (int b = 0; b < R; ++b) e[a][b] += rqi * rpj[b] - rpi * rqj[b];
      }
      // columns p, q: A[i][p] = −rq[i]/a, A[i][q] = rp[i]/a; then rows p, q (they take
      // precedence): A[p][j] = rq[j]/a, A[q][j] = −rp[j]/a, A[p][q] = −1/a, A[q][p] = 1/a,
      // A[p][p] = A[q][q] = 0. Only the threads holding those rows or columns take part.
      if (tc == p % G || tc == q % G) {
#pragma unroll
        for (int b = 0; b < R; ++b) {
          const int j = tc + G * b;
          if (j != p && j != q) continue;
#pragma unroll
          for (int a = 0; a < R; ++a) {
            const int i = tr + G * a;
            if (i < n) e[a][b] = j == p ? -rq[i] * ia : rp[i] * ia;
          }
        }
      }
      if (tr == p % G || tr == q % G) {
#pragma unroll
        for (int a = 0; a < R; ++a) {
          const int i = tr + G * a;
          if (i != p && i != q) continue;
#pragma unroll
          for (int b = 0; b < R; ++b) {
            const int j = tc + G * b;
            if (i == p) e[a][b] = (j == q) ? -ia : (j == p ? T(0) : rqj[b] * ia);
            else e[a][b] = (j == p) ? ia : (j == q ? T(0) : -rpj[b] * ia);
          }
        }
      }
      if (p < 64) sw0 |= 1ull << p;
      else sw1 |= 1ull << (p - 64);
      if (q < 64) sw0 |= 1ull << q;
      else sw1 |= 1ull << (q - 64);
      int np = n;
      if (~sw0) np = min(n, __ffsll(static_cast<long long>(~sw0)) - 1);
      else if (~sw1) np = min(n, 64 + __ffsll(static_cast<long long>(~sw1)) - 1);
      if (np < n && tr == np % G) publish(np, 1 - par);
      p = np < n ? np : 0;
    }
#pragma unroll
    for (int a = 0; a < R; ++a)
#pragma unroll
      for (int b = 0; b < R; ++b) {
        const int i = tr + G * a, j = tc + G * b;
        if (i < n && j < n) ip[static_cast<size_t>(i) * n + j] = -static_cast<double>(e[a][b]);
      }
    if (tid == 0) {
      double v = (parity & 1) ? -pfv : pfv;
      if (st == 0 && !isfinite(v)) st = -1;
      if (st != 0) v = 0.0;
      pf[plane] = v;
      status[plane] = st;
    }
    __syncthreads();
  }
}

// Uniform batches of side N ∈ {32, 64}: the register sweep with one barrier per pivot step.
// Thread (tr, tc) of a G×G block owns the R×R elements (tr + G·a, tc + G·b), R = N/G. At
// the barrier of step k shared memory holds the current rows p_k and q_k and the current
// row of the next pivot index p_{k+1}; every thread then (1) applies the rank-2 update of
// step k to its elements, (2) recomputes row p_{k+1} after the update in registers (every
// warp the whole row, N/32 columns per lane, from the three published rows) and finds its
// pivot q_{k+1} by the first-maximum rule with a warp reduction — all warps get the same
// bits, so no barrier is needed to agree on it — and (3) the owners of rows q_{k+1} and
// p_{k+2} publish them (warp 0 publishes row p_{k+1}) into the other buffer set. Rows and
// columns p, q are overwritten after each update (as in k_pfinv_reg), so the owners' copies
// of row p_{k+1} are never read: only the recomputed row is used.
template <typename T, int N, int G, int MB>
__global__ void __launch_bounds__(G * G, MB)
    k_pfinv_uni(const double* __restrict__ x, int planes, double* __restrict__ pf, double* __restrict__ inv,
                int* __restrict__ status) {
  static_assert(N == 32 || N == 64, "one 64-bit swept mask, whole warps per row pass");
  constexpr int R = N / G, NT = G * G, C = N / 32, LDA = N + 1;
  extern __shared__ __align__(16) unsigned char smem[];
  T* stage = reinterpret_cast<T*>(smem);  // [N][N + 1]
  T* bufs = stage + N * LDA;              // [2 parities][3 rows: p, q, next p][N]
  const int tid = threadIdx.x, tr = tid / G, tc = tid % G, lane = tid & 31;
  const unsigned long long all = N == 64 ? ~0ull : ((1ull << N) - 1ull);
  for (int plane = blockIdx.x; plane < planes; plane += gridDim.x) {
    const double* xp = x + static_cast<size_t>(plane) * N * N;
    double* ip = inv + static_cast<size_t>(plane) * N * N;
    for (int k = tid; k < N * N; k += NT) stage[(k / N) * LDA + k % N] = static_cast<T>(-xp[k]);
    __syncthreads();
    T e[R][R];
#pragma unroll
    for (int a = 0; a < R; ++a)
#pragma unroll
      for (int b = 0; b < R; ++b) e[a][b] = stage[(tr + G * a) * LDA + tc + G * b];
    // first maximum of |row[j]| over unswept j ≠ r (values v[c] at j = lane + 32c), the
    // pivot value and the number of unswept indices strictly between r and the pivot
    auto pivot = [&](const T* v, int r, unsigned long long sw, int& q, T& av, int& cnt) {
      double best = -1.0;
      int bi = N;
      T bval = T(0);
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int j = lane + 32 * c;
        if (j != r && !((sw >> j) & 1ull)) {
          const double a = fabs(static_cast<double>(v[c]));
          if (a > best) {
            best = a;
            bi = j;
            bval = v[c];
          }
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        const T ov = __shfl_xor_sync(0xffffffffu, bval, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
          bval = ov;
        }
      }
      q = best > 0.0 ? bi : N;
      av = bval;
      cnt = 0;
      if (q < N && q > r + 1) {
        const int len = q - r - 1;
        const unsigned long long range = (len == 64 ? ~0ull : ((1ull << len) - 1ull)) << (r + 1);
        cnt = __popcll(~sw & range);
      }
    };
    auto lowest_unswept = [&](unsigned long long sw) {
      const unsigned long long free = ~sw & all;
      return free ? __ffsll(static_cast<long long>(free)) - 1 : N;
    };
    // step 0: rows straight from the staged matrix
    unsigned long long sw = 0ull;
    int p = 0, q, cnt, st = 0, parity = 0;
    T av;
    {
      T v[C];
#pragma unroll
      for (int c = 0; c < C; ++c) v[c] = stage[lane + 32 * c];
      pivot(v, 0, sw, q, av, cnt);
    }
    double pfv = 1.0;
    const T* rP = stage;
    const T* rQ = stage + (q < N ? q : 0) * LDA;
    int pn = lowest_unswept(sw | 1ull | (q < N ? (1ull << q) : 0ull));
    const T* rN = stage + (pn < N ? pn : 0) * LDA;
    for (int k = 0; k < N / 2; ++k) {
      if (q >= N) {
        st = p + 1;
        break;
      }
      const T ia = T(1) / av;
      parity += cnt;
      pfv *= static_cast<double>(av);
      // (1) rank-2 update of step k, then columns and rows p, q
      T rpj[R], rqj[R];
#pragma unroll
      for (int b = 0; b < R; ++b) {
        rpj[b] = rP[tc + G * b];
        rqj[b] = rQ[tc + G * b];
      }
#pragma unroll
      for (int a = 0; a < R; ++a) {
        const int i = tr + G * a;
        const T rpi = rP[i] * ia, rqi = rQ[i] * ia;
#pragma unroll
        for (int b = 0; b < R; ++b) e[a][b] += rqi * rpj[b] - rpi * rqj[b];
      }
      if (tc == p % G || tc == q % G) {
#pragma unroll
        for (int b = 0; b < R; ++b) {
          const int j = tc + G * b;
          if (j != p && j != q) continue;
#pragma unroll
          for (int a = 0; a < R; ++a) {
            const int i = tr + G * a;
            e[a][b] = j == p ? -rQ[i] * ia : rP[i] * ia;
          }
        }
      }
      if (tr == p % G || tr == q % G) {
#pragma unroll
        for (int a = 0; a < R; ++a) {
          const int i = tr + G * a;
          if (i != p && i != q) continue;
#pragma unroll
          for (int b = 0; b < R; ++b) {
            const int j = tc + G * b;
            if (i == p) e[a][b] = (j == q) ? -ia : (j == p ? T(0) : rqj[b] * ia);
            else e[a][b] = (j == p) ? ia : (j == q ? T(0) : -rpj[b] * ia);
          }
        }
      }
      sw |= (1ull << p) | (1ull << q);
      if (k == N / 2 - 1) break;
      // (2) row p' = pn after this update, in every warp, and its pivot
      T v[C];
      {
        const T rpp = rP[pn] * ia, rqp = rQ[pn] * ia;
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const int j = lane + 32 * c;
          T val = rN[j] + (rqp * rP[j] - rpp * rQ[j]);
          if (j == p) val = -rQ[pn] * ia;
          if (j == q) val = rP[pn] * ia;
          v[c] = val;
        }
      }
      int qn, cn;
      T an;
      pivot(v, pn, sw, qn, an, cn);
      const int pnn = qn < N ? lowest_unswept(sw | (1ull << pn) | (1ull << qn)) : N;
      // (3) publish rows p', q' and the next p'' into the other buffer set
      T* oP = bufs + ((k + 1) & 1) * 3 * N;
      T* oQ = oP + N;
      T* oN = oQ + N;
      if (tid < 32) {
#pragma unroll
        for (int c = 0; c < C; ++c) oP[lane + 32 * c] = v[c];
      }
      if (qn < N && tr == qn % G) {
        const int aq = qn / G;
#pragma unroll
        for (int a = 0; a < R; ++a) {
          if (a != aq) continue;
#pragma unroll
          for (int b = 0; b < R; ++b) oQ[tc + G * b] = e[a][b];
        }
      }
      if (pnn < N && tr == pnn % G) {
        const int an2 = pnn / G;
#pragma unroll
        for (int a = 0; a < R; ++a) {
          if (a != an2) continue;
#pragma unroll
          for (int b = 0; b < R; ++b) oN[tc + G * b] = e[a][b];
        }
      }
      __syncthreads();
      rP = oP;
      rQ = oQ;
      rN = oN;
      p = pn;
      q = qn;
      av = an;
      cnt = cn;
      pn = pnn;
    }
#pragma unroll
    for (int a = 0; a < R; ++a)
#pragma unroll
      for (int b = 0; b < R; ++b) ip[static_cast<size_t>(tr + G * a) * N + tc + G * b] = -static_cast<double>(e[a][b]);
    if (tid == 0) {
      double val = (parity & 1) ? -pfv : pfv;
      if (st == 0 && !isfinite(val)) st = -1;
      if (st != 0) val = 0.0;
      pf[plane] = val;
      status[plane] = st;
    }
    __syncthreads();
  }
}

// Uniform batches of side N ∈ {32, 64}, one warp per plane with no block barrier: the
// plane lives in shared memory (row-major, the warp's own slice), lane l owns columns
// l + 32c. A pivot step: every lane reads its columns of row p and the warp finds the
// first maximum by shuffles; the lanes snapshot rows p and q (their own columns) into the
// warp's two snapshot rows, and after a warp barrier update every row of their columns,
// reading the row coefficients (row q and row p at the row's index) from the snapshots.
// Same element formula and pivot rule as k_pfinv_reg / k_pfinv_uni.
// Warps (planes) per block: FP64 planes of 64 take 34 KB each, so two per block and three
// blocks fill an SM's shared memory.
template <typename T, int N>
struct PfWarps {
  static constexpr int kPerBlock = (N == 64 && sizeof(T) == 8) ? 2 : 4;
};
template <typename T, int N>
__global__ void __launch_bounds__(32 * PfWarps<T, N>::kPerBlock)
    k_pfinv_warp(const double* __restrict__ x, int planes, double* __restrict__ pf, double* __restrict__ inv,
                 int* __restrict__ status) {
  static_assert(N == 32 || N == 64, "one 64-bit swept mask, whole lanes per column set");
  constexpr int C = N / 32, kPfWarpsPerBlock = PfWarps<T, N>::kPerBlock;
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T* A = reinterpret_cast<T*>(smem) + static_cast<size_t>(warp) * (N * N + 2 * N);
  T* SP = A + N * N;  // snapshot of row p
  T* SQ = SP + N;     // snapshot of row q
  const unsigned long long all = N == 64 ? ~0ull : ((1ull << N) - 1ull);
  for (int plane = blockIdx.x * kPfWarpsPerBlock + warp; plane < planes; plane += gridDim.x * kPfWarpsPerBlock) {
    const double* xp = x + static_cast<size_t>(plane) * N * N;
    for (int k = lane; k < N * N; k += 32) A[k] = static_cast<T>(-xp[k]);
    __syncwarp();
    unsigned long long sw = 0ull;
    int st = 0, parity = 0;
    double pfv = 1.0;
    for (int step = 0; step < N / 2; ++step) {
      const unsigned long long free = ~sw & all;
      const int p = __ffsll(static_cast<long long>(free)) - 1;
      // pivot q: first maximum of |A(p, j)| over unswept j != p
      double best = -1.0;
      int bi = N;
      T rp[C], rq[C];
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int j = lane + 32 * c;
        rp[c] = A[p * N + j];
        if (j != p && !((sw >> j) & 1ull)) {
          const double v = fabs(static_cast<double>(rp[c]));
          if (v > best) {
            best = v;
            bi = j;
          }
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (!(best > 0.0)) {
        st = p + 1;
        break;
      }
      const int q = bi;
      const T a = A[p * N + q];
      const T ia = T(1) / a;
      pfv *= static_cast<double>(a);
      {
        const int len = q - p - 1;
        if (len > 0) {
          const unsigned long long range = (len == 64 ? ~0ull : ((1ull << len) - 1ull)) << (p + 1);
          parity += __popcll(~sw & range);
        }
      }
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int j = lane + 32 * c;
        rq[c] = A[q * N + j];
        SP[j] = rp[c];
        SQ[j] = rq[c];
      }
      __syncwarp();
#pragma unroll 4
      for (int i = 0; i < N; ++i) {
        const T rpi = SP[i], rqi = SQ[i];
        const T ai = rqi * ia, bi2 = rpi * ia;
        T* Ai = A + i * N;
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const int j = lane + 32 * c;
          T v;
          if (i == p) v = (j == q) ? -ia : (j == p ? T(0) : rq[c] * ia);
          else if (i == q) v = (j == p) ? ia : (j == q ? T(0) : -rp[c] * ia);
          else if (j == p) v = -rqi * ia;
          else if (j == q) v = rpi * ia;
          else v = Ai[j] + (ai * rp[c] - bi2 * rq[c]);
          Ai[j] = v;
        }
      }
      sw |= (1ull << p) | (1ull << q);
      __syncwarp();
    }
    double* ip = inv + static_cast<size_t>(plane) * N * N;
    for (int k = lane; k < N * N; k += 32) ip[k] = -static_cast<double>(A[k]);
    if (lane == 0) {
      double v = (parity & 1) ? -pfv : pfv;
      if (st == 0 && !isfinite(v)) st = -1;
      if (st != 0) v = 0.0;
      pf[plane] = v;
      status[plane] = st;
    }
    __syncwarp();
  }
}

template <typename T, int N>
int launch_pfinv_warp(const double* x, int planes, double* pf, double* inv, int* status, cudaStream_t stream) {
  constexpr int kPfWarpsPerBlock = PfWarps<T, N>::kPerBlock;
  const size_t smem = sizeof(T) * kPfWarpsPerBlock * (static_cast<size_t>(N) * N + 2 * static_cast<size_t>(N));
  auto kernel = k_pfinv_warp<T, N>;
  MVMCB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  int per_sm = 0;
  MVMCB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 32 * kPfWarpsPerBlock, smem));
  const int blocks_needed = (planes + kPfWarpsPerBlock - 1) / kPfWarpsPerBlock;
  const int grid = std::max(1, std::min(blocks_needed, std::max(1, per_sm) * device_sm_count()));
  kernel<<<grid, 32 * kPfWarpsPerBlock, smem, stream>>>(x, planes, pf, inv, status);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

template <typename T, int N, int G, int MB>
int launch_pfinv_uni(const double* x, int planes, double* pf, double* inv, int* status, cudaStream_t stream) {
  const size_t smem = sizeof(T) * (static_cast<size_t>(N) * (N + 1) + 6 * static_cast<size_t>(N));
  auto kernel = k_pfinv_uni<T, N, G, MB>;
  MVMCB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  int per_sm = 0;
  MVMCB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, G * G, smem));
  const int grid = std::max(1, std::min(planes, std::max(1, per_sm) * device_sm_count()));
  kernel<<<grid, G * G, smem, stream>>>(x, planes, pf, inv, status);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

template <typename T, int G, int R>
int launch_pfinv_reg(const double* x, const int* sizes, const long long* offsets, int n_uniform, int planes,
                     int n_max, double* pf, double* inv, int* status, cudaStream_t stream) {
  const size_t smem = sizeof(T) * (static_cast<size_t>(n_max) * (n_max + 1) + 4 * static_cast<size_t>(n_max));
  auto kernel = k_pfinv_reg<T, G, R>;
  MVMCB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  int per_sm = 0;
  MVMCB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, G * G, smem));
  const int grid = std::max(1, std::min(planes, std::max(1, per_sm) * device_sm_count()));
  kernel<<<grid, G * G, smem, stream>>>(x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

// ---- tile-shape autotuner of the register sweep ----------------------------------------
// Every candidate computes each element with the same two-FMA update, the same first-maximum
// pivot search and the same Pf product order, so the choice changes the speed and never the
// bits. Candidates per size class: G×G threads with R×R elements each, n ≤ G·R.
struct RegTile {
  int g, r;
};

template <typename T>
int launch_reg_tile(RegTile t, const double* x, const int* sizes, const long long* offsets, int n_uniform,
                    int planes, int n_max, double* pf, double* inv, int* status, cudaStream_t stream) {
#define MVMCB_TILE(G, R)                                                                                   \
  if (t.g == G && t.r == R && n_max <= G * R)                                                              \
    return launch_pfinv_reg<T, G, R>(x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status, stream);
  MVMCB_TILE(16, 2)
  MVMCB_TILE(8, 4)
  MVMCB_TILE(16, 4)
  MVMCB_TILE(8, 8)
  MVMCB_TILE(32, 4)
  MVMCB_TILE(16, 8)
#undef MVMCB_TILE
  return kErrArgument;
}

std::vector<RegTile> reg_tile_candidates(int n_max) {
  if (n_max <= 32) return {{16, 2}, {8, 4}};
  if (n_max <= 64) return {{16, 4}, {8, 8}};
  return {{32, 4}, {16, 8}};
}

// MVMC_B200_PFINV_TILE=GxR forces a tile; MVMC_B200_AUTOTUNE=0 keeps the first candidate.
// Otherwise the first call for a (precision, size class, planes bucket) times every
// candidate on the caller's own batch (two launches each after one warm-up, CUDA events on
// the caller's stream) and keeps the fastest for the process.
template <typename T>
int dispatch_pfinv_reg(const double* x, const int* sizes, const long long* offsets, int n_uniform, int planes,
                       int n_max, double* pf, double* inv, int* status, cudaStream_t stream) {
  const std::vector<RegTile> cand = reg_tile_candidates(n_max);
  if (const char* f = std::getenv("MVMC_B200_PFINV_TILE")) {
    RegTile t{0, 0};
    if (std::sscanf(f, "%dx%d", &t.g, &t.r) == 2)
      return launch_reg_tile<T>(t, x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status, stream);
  }
  const char* a = std::getenv("MVMC_B200_AUTOTUNE");
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(stream, &cap);
  if ((a && std::strcmp(a, "0") == 0) || cap != cudaStreamCaptureStatusNone)
    return launch_reg_tile<T>(cand[0], x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status, stream);
  static std::mutex mu;
  static std::map<long long, int> chosen;
  const int cls = n_max <= 32 ? 32 : (n_max <= 64 ? 64 : 128);
  int bucket = 0;
  while ((1 << bucket) < planes && bucket < 30) ++bucket;
  const long long key = (static_cast<long long>(sizeof(T)) * 1000 + cls) * 64 + bucket;
  int pick = -1;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = chosen.find(key);
    if (it != chosen.end()) pick = it->second;
  }
  if (pick < 0) {
    cudaEvent_t e0, e1;
    MVMCB_CUDA(cudaEventCreate(&e0));
    MVMCB_CUDA(cudaEventCreate(&e1));
    float best = 0.0f;
    for (size_t c = 0; c < cand.size(); ++c) {
      int rc = launch_reg_tile<T>(cand[c], x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status, stream);
      if (rc != kOk) continue;
      MVMCB_CUDA(cudaEventRecord(e0, stream));
      for (int rep = 0; rep < 2 && rc == kOk; ++rep)
        rc = launch_reg_tile<T>(cand[c], x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status, stream);
      MVMCB_CUDA(cudaEventRecord(e1, stream));
      MVMCB_CUDA(cudaEventSynchronize(e1));
      float ms = 0.0f;
      MVMCB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (rc == kOk && (pick < 0 || ms < best)) {
        best = ms;
        pick = static_cast<int>(c);
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (pick < 0) pick = 0;
    std::lock_guard<std::mutex> lock(mu);
    chosen[key] = pick;
  }
  return launch_reg_tile<T>(cand[pick], x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status, stream);
}

template <typename T>
size_t pfinv_smem_bytes(int n_max, bool smem_matrix) {
  size_t b = (gj_shared_bytes<T>(n_max) + 15) & ~size_t(15);
  if (smem_matrix) b += sizeof(T) * static_cast<size_t>(n_max) * (n_max + 1);
  return b;
}

int device_smem_limit() { return current_device_attr(cudaDevAttrMaxSharedMemoryPerBlockOptin); }

int device_sm_count() { return current_device_attr(cudaDevAttrMultiProcessorCount); }

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
  if (!sizes && n_uniform == n_max && (n_max == 32 || n_max == 64) && (precision == 32 || precision == 64) &&
      !std::getenv("MVMC_B200_PFINV_TILE")) {
    // uniform batches of 32 or 64 (MVMC_B200_PFINV_TILE keeps the two-barrier tiles), all
    // with the same bits as those tiles. Side 32: one warp per plane, no block barrier
    // (B = 8192: 0.24 ms FP64 / 0.17 ms FP32 against 0.46 / 0.37 ms for the two-barrier tile).
    // Side 64: one barrier per pivot step (1.31 ms FP64 / 1.03 ms FP32 against 1.49 / 1.16 ms;
    // a warp per plane holds a 34 KB FP64 plane, so only six fit an SM: 3.2 ms).
    if (n_max == 32)
      return precision == 32 ? launch_pfinv_warp<float, 32>(x, planes, pf, inv, status, stream)
                             : launch_pfinv_warp<double, 32>(x, planes, pf, inv, status, stream);
    if (precision == 32) return launch_pfinv_uni<float, 64, 16, 4>(x, planes, pf, inv, status, stream);
    return launch_pfinv_uni<double, 64, 16, 3>(x, planes, pf, inv, status, stream);
  }
  if (n_max <= 128 && (precision == 32 || precision == 64)) {
    if (precision == 32)
      return dispatch_pfinv_reg<float>(x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status, stream);
    return dispatch_pfinv_reg<double>(x, sizes, offsets, n_uniform, planes, n_max, pf, inv, status, stream);
  }
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
// Host-buffer entry points: the batch runs in chunks of about 32 MB on two streams, so the
// copy of chunk c+1 to the device, the sweep of chunk c and the copy of chunk c−1 back
// overlap (fully with pinned host buffers; pageable buffers are staged by the driver). The
// device buffers and streams are kept for the process and reused by later calls.
struct HostPipe {
  int device = -1;
  cudaStream_t stream[2] = {nullptr, nullptr};
  double* x[2] = {nullptr, nullptr};
  double* inv[2] = {nullptr, nullptr};
  double* pf[2] = {nullptr, nullptr};
  int* st[2] = {nullptr, nullptr};
  int* sz[2] = {nullptr, nullptr};
  long long* off[2] = {nullptr, nullptr};
  size_t cap_elems = 0;
  int cap_planes = 0;
};
std::mutex g_pipe_mu;
HostPipe g_pipe;

int pipe_reserve(size_t elems, int planes) {
  int dev = 0;
  MVMCB_CUDA(cudaGetDevice(&dev));
  HostPipe& h = g_pipe;
  if (h.device != dev) {
    h = HostPipe{};  // a new device: the old buffers stay with their context
    h.device = dev;
    for (int b = 0; b < 2; ++b) MVMCB_CUDA(cudaStreamCreateWithFlags(&h.stream[b], cudaStreamNonBlocking));
  }
  if (elems > h.cap_elems || planes > h.cap_planes) {
    for (int b = 0; b < 2; ++b) {
      cudaFree(h.x[b]); cudaFree(h.inv[b]); cudaFree(h.pf[b]); cudaFree(h.st[b]); cudaFree(h.sz[b]); cudaFree(h.off[b]);
      h.x[b] = h.inv[b] = h.pf[b] = nullptr;
      h.st[b] = h.sz[b] = nullptr;
      h.off[b] = nullptr;
    }
    h.cap_elems = h.cap_planes = 0;
    for (int b = 0; b < 2; ++b) {
      MVMCB_CUDA(cudaMalloc(&h.x[b], elems * sizeof(double)));
      MVMCB_CUDA(cudaMalloc(&h.inv[b], elems * sizeof(double)));
      MVMCB_CUDA(cudaMalloc(&h.pf[b], planes * sizeof(double)));
      MVMCB_CUDA(cudaMalloc(&h.st[b], planes * sizeof(int)));
      MVMCB_CUDA(cudaMalloc(&h.sz[b], planes * sizeof(int)));
      MVMCB_CUDA(cudaMalloc(&h.off[b], planes * sizeof(long long)));
    }
    h.cap_elems = elems;
    h.cap_planes = planes;
  }
  return kOk;
}

// Drains both pipe streams when a call leaves early, so that no copy into the caller's
// host buffers is still in flight when the caller regains them.
struct PipeDrain {
  HostPipe& h;
  ~PipeDrain() {
    for (int b = 0; b < 2; ++b)
      if (h.stream[b]) cudaStreamSynchronize(h.stream[b]);
  }
};

// sizes == nullptr: uniform n_uniform planes. comps = 1 for real planes, 2 for complex
// planes ((re, im) pairs; uniform sizes only).
int pfinv_host(const double* x, const int* sizes, int n_uniform, int planes, int precision, int comps, double* pf,
               double* inv, int* status) {
  std::vector<long long> offsets(planes + 1, 0);
  int n_max = n_uniform;
  for (int p = 0; p < planes; ++p) {
    const int n = sizes ? sizes[p] : n_uniform;
    if (n <= 0 || (n & 1)) return kErrArgument;
    offsets[p + 1] = offsets[p] + static_cast<long long>(n) * n;
    n_max = std::max(n_max, n);
  }
  // chunks of about 32 MB of planes (at least one plane)
  const long long target = (32ll << 20) / static_cast<long long>(sizeof(double) * comps);
  std::vector<int> starts{0};
  while (starts.back() < planes) {
    int e = starts.back() + 1;
    while (e < planes && offsets[e + 1] - offsets[starts.back()] <= target) ++e;
    starts.push_back(e);
  }
  size_t max_elems = 0;
  int max_planes = 0;
  for (size_t c = 0; c + 1 < starts.size(); ++c) {
    max_elems = std::max<size_t>(max_elems, offsets[starts[c + 1]] - offsets[starts[c]]);
    max_planes = std::max(max_planes, starts[c + 1] - starts[c]);
  }
  std::lock_guard<std::mutex> lock(g_pipe_mu);
  int rc = pipe_reserve(max_elems * comps, max_planes * comps);
  if (rc != kOk) return rc;
  HostPipe& h = g_pipe;
  PipeDrain drain{h};
  std::vector<long long> rel(max_planes);
  for (size_t c = 0; c + 1 < starts.size(); ++c) {
    const int b = static_cast<int>(c & 1), p0 = starts[c], np = starts[c + 1] - p0;
    const long long e0 = offsets[p0] * comps, ne = (offsets[starts[c + 1]] - offsets[p0]) * comps;
    cudaStream_t st = h.stream[b];
    MVMCB_CUDA(cudaMemcpyAsync(h.x[b], x + e0, ne * sizeof(double), cudaMemcpyHostToDevice, st));
    if (sizes) {
      for (int p = 0; p < np; ++p) rel[p] = offsets[p0 + p] - offsets[p0];
      MVMCB_CUDA(cudaMemcpyAsync(h.sz[b], sizes + p0, np * sizeof(int), cudaMemcpyHostToDevice, st));
      MVMCB_CUDA(cudaMemcpyAsync(h.off[b], rel.data(), np * sizeof(long long), cudaMemcpyHostToDevice, st));
    }
    if (comps == 2)
      rc = pfinv_complex_device(h.x[b], n_uniform, np, h.pf[b], h.inv[b], h.st[b], st);
    else
      rc = pfinv_device(h.x[b], sizes ? h.sz[b] : nullptr, sizes ? h.off[b] : nullptr, n_uniform, np, n_max,
                        h.pf[b], h.inv[b], h.st[b], precision, st);
    if (rc != kOk) return rc;
    MVMCB_CUDA(cudaMemcpyAsync(inv + e0, h.inv[b], ne * sizeof(double), cudaMemcpyDeviceToHost, st));
    MVMCB_CUDA(cudaMemcpyAsync(pf + static_cast<size_t>(p0) * comps, h.pf[b], np * comps * sizeof(double),
                               cudaMemcpyDeviceToHost, st));
    MVMCB_CUDA(cudaMemcpyAsync(status + p0, h.st[b], np * sizeof(int), cudaMemcpyDeviceToHost, st));
  }
  for (int b = 0; b < 2; ++b) MVMCB_CUDA(cudaStreamSynchronize(h.stream[b]));
  return kOk;
}
}  // namespace

extern "C" int mvmc_b200_pfinv_batch(const double* x, int n, int planes, double* pf, double* inv,
                                     int* status) {
  if (n <= 0 || (n & 1) || planes < 0) return kErrArgument;
  if (planes == 0) return kOk;
  if (!x || !pf || !inv || !status) return kErrArgument;
  return pfinv_host(x, nullptr, n, planes, 64, 1, pf, inv, status);
}

extern "C" int mvmc_b200_pfinv_batch_mixed(const double* x, const int* sizes, int planes,
                                           int precision, double* pf, double* inv, int* status) {
  if (planes < 0 || !sizes) return kErrArgument;
  if (planes == 0) return kOk;
  if (!x || !pf || !inv || !status) return kErrArgument;
  return pfinv_host(x, sizes, 0, planes, precision, 1, pf, inv, status);
}

extern "C" int mvmc_b200_pfinv_batch_complex(const double* x, int n, int planes, double* pf, double* inv,
                                             int* status) {
  if (n <= 0 || (n & 1) || planes < 0) return kErrArgument;
  if (planes == 0) return kOk;
  if (!x || !pf || !inv || !status) return kErrArgument;
  return pfinv_host(x, nullptr, n, planes, 64, 2, pf, inv, status);
}
