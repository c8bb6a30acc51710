// Skew-symmetric Gauss–Jordan sweep with 2×2 pivots: Pfaffian and inverse in one pass.
//
// For a skew matrix X (n even) the in-place Gauss–Jordan sweep over the index pair
// (p, q) with pivot block [[0, a], [-a, 0]], a = X[p][q], keeps the matrix skew:
//   A[i][j] += (rowq[i]·rowp[j] − rowp[i]·rowq[j]) / a        (i, j ∉ {p, q})
//   A[p][j]  = rowq[j] / a,  A[q][j] = −rowp[j] / a,  A[p][q] = −1/a
// where rowp, rowq are rows p and q before the sweep. After n/2 sweeps covering every
// index once, A = X⁻¹ and Pf(X) = sgn(σ) Π a_k with σ = (p1 q1 p2 q2 …).
// Pivoting: p = smallest unswept index, q = argmax_{unswept j≠p} |A[p][j]| (first
// maximum) — the Parlett–Reid partial pivoting rule applied row-wise.
//
// This replaces pfapack's dsktf2 → utu2pfa → utu2inv pipeline
// (crates/pfapack/src/ltl.rs:34-188, utu2.rs:52-110,338-515 of AtelierArith/mvmc-rs)
// with one sweep of n/2 rank-2 updates: 2n³ flops on the full matrix (n³ on half),
// no triangular solves, no permutation passes, every update a uniform data-parallel
// rank-2 step.
#pragma once

#include "common.cuh"

namespace mvmcb {

template <typename T>
struct GJShared {
  T* rowp;      // [n] snapshot of row p
  T* rowq;      // [n] snapshot of row q
  int* swept;   // [n]
  int* ctl;     // [4]: p, q, status, parity
  double* pfv;  // [1] running product of pivots
};

template <typename T>
__host__ __device__ constexpr size_t gj_shared_bytes(int n) {
  return 2 * sizeof(T) * static_cast<size_t>(n) + sizeof(int) * static_cast<size_t>(n) +
         4 * sizeof(int) + sizeof(double) + 64;
}

template <typename T>
__device__ __forceinline__ GJShared<T> gj_carve(unsigned char* base, int n) {
  GJShared<T> s;
  size_t off = 0;
  s.pfv = reinterpret_cast<double*>(base + off);
  off += 16;
  s.rowp = reinterpret_cast<T*>(base + off);
  off += sizeof(T) * n;
  s.rowq = reinterpret_cast<T*>(base + off);
  off += sizeof(T) * n;
  off = (off + 15) & ~size_t(15);
  s.swept = reinterpret_cast<int*>(base + off);
  off += sizeof(int) * n;
  s.ctl = reinterpret_cast<int*>(base + off);
  return s;
}

// CTA-wide. A is row-major with leading dimension lda (shared or global memory).
// On exit A holds X⁻¹; pf_out/status_out are valid in every thread.
// status: 0 ok, k > 0 singular (1-based row of the zero pivot row), -1 non-finite Pf.
template <typename T>
__device__ void gj_pfinv(T* A, int lda, int n, const GJShared<T>& s, double& pf_out,
                         int& status_out) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  for (int j = tid; j < n; j += nt) s.swept[j] = 0;
  if (tid == 0) {
    s.ctl[0] = 0;
    s.ctl[2] = 0;
    s.ctl[3] = 0;
    *s.pfv = 1.0;
  }
  __syncthreads();
  for (int k = 0; k < n / 2; ++k) {
    const int p = s.ctl[0];
    for (int j = tid; j < n; j += nt) s.rowp[j] = A[p * lda + j];
    __syncthreads();
    if (warp == 0) {
      double best = -1.0;
      int bi = n;
      for (int j = lane; j < n; j += 32) {
        if (!s.swept[j] && j != p) {
          const double v = fabs(static_cast<double>(s.rowp[j]));
          if (v > best) {
            best = v;
            bi = j;
          }
        }
      }
      warp_argmax_first(best, bi);
      const int q = __shfl_sync(0xffffffffu, bi, 0);
      best = __shfl_sync(0xffffffffu, best, 0);
      int cnt = 0;
      for (int j = lane; j < n; j += 32) cnt += (!s.swept[j] && j > p && j < q) ? 1 : 0;
      for (int off = 16; off > 0; off >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
      __syncwarp();
      if (lane == 0) {
        if (!(best > 0.0)) {
          s.ctl[2] = p + 1;
        } else {
          *s.pfv *= static_cast<double>(s.rowp[q]);
          s.ctl[3] += cnt;
          s.ctl[1] = q;
          s.swept[p] = 1;
          s.swept[q] = 1;
        }
      }
      __syncwarp();
      int nxt = n;
      for (int j = lane; j < n; j += 32)
        if (!s.swept[j] && j < nxt) nxt = j;
      for (int off = 16; off > 0; off >>= 1) nxt = min(nxt, __shfl_xor_sync(0xffffffffu, nxt, off));
      if (lane == 0) s.ctl[0] = nxt < n ? nxt : 0;
    }
    __syncthreads();
    if (s.ctl[2] != 0) break;
    const int q = s.ctl[1];
    for (int j = tid; j < n; j += nt) s.rowq[j] = A[q * lda + j];
    __syncthreads();
    const T ia = T(1) / s.rowp[q];
    for (int i = warp; i < n; i += nwarp) {
      const T rpi = s.rowp[i], rqi = s.rowq[i];
      T* Ai = A + i * lda;
      if (i == p) {
        for (int j = lane; j < n; j += 32) Ai[j] = (j == q) ? -ia : (j == p ? T(0) : s.rowq[j] * ia);
      } else if (i == q) {
        for (int j = lane; j < n; j += 32) Ai[j] = (j == p) ? ia : (j == q ? T(0) : -s.rowp[j] * ia);
      } else {
        for (int j = lane; j < n; j += 32) {
          T v;
          if (j == p) v = -rqi * ia;
          else if (j == q) v = rpi * ia;
          else v = Ai[j] + (rqi * s.rowp[j] - rpi * s.rowq[j]) * ia;
          Ai[j] = v;
        }
      }
    }
    __syncthreads();
  }
  const int status = s.ctl[2];
  double pf = (s.ctl[3] & 1) ? -*s.pfv : *s.pfv;
  int st = status;
  if (st == 0 && !isfinite(pf)) st = -1;
  if (st != 0) pf = 0.0;
  pf_out = pf;
  status_out = st;
  __syncthreads();
}

}  // namespace mvmcb

namespace mvmcb {

// In-place form for planes in global memory whose ping-pong partner would not stay in L2
// beside the other resident samples: rows p and q are snapshot in shared memory (snap,
// 2n elements) and the sweep updates A in place; three barriers per pivot step. Same
// element arithmetic, pivot rule and status codes as gj_pfinv_pp. n <= 32·JPL, lda = n.
template <typename T, int JPL, int RB = 1>
__device__ void gj_pfinv_ip(T* A, T* snap, int n, double& pf_out, int& status_out) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  unsigned swept = 0;  // bit c: column lane + 32c swept
  int p = 0, parity = 0, status = 0;
  double pf = 1.0;
  T* rowp = snap;
  T* rowq = snap + n;
  for (int k = 0; k < n / 2; ++k) {
    for (int j = tid; j < n; j += nt) rowp[j] = A[static_cast<size_t>(p) * n + j];
    __syncthreads();
    T rp[JPL];
    double best = -1.0;
    int bi = n;
#pragma unroll
    for (int c = 0; c < JPL; ++c) {
      const int j = lane + 32 * c;
      rp[c] = j < n ? rowp[j] : T(0);
      if (j < n && j != p && !((swept >> c) & 1u)) {
        const double v = fabs(static_cast<double>(rp[c]));
        if (v > best) {
          best = v;
          bi = j;
        }
      }
    }
    warp_argmax_first(best, bi);
    const int q = __shfl_sync(0xffffffffu, bi, 0);
    best = __shfl_sync(0xffffffffu, best, 0);
    if (!(best > 0.0)) {
      status = p + 1;
      break;  // every warp reads the same snapshot: all leave together
    }
    int cnt = 0;
#pragma unroll
    for (int c = 0; c < JPL; ++c) {
      const int j = lane + 32 * c;
      cnt += (j < n && !((swept >> c) & 1u) && j > p && j < q) ? 1 : 0;
    }
    for (int off = 16; off > 0; off >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
    parity += cnt;
    const T a = rowp[q];
    pf *= static_cast<double>(a);
    const T ia = T(1) / a;
    for (int j = tid; j < n; j += nt) rowq[j] = A[static_cast<size_t>(q) * n + j];
    __syncthreads();
    T rq[JPL];
#pragma unroll
    for (int c = 0; c < JPL; ++c) {
      const int j = lane + 32 * c;
      rq[c] = j < n ? rowq[j] : T(0);
    }
    for (int i0 = warp; i0 < n; i0 += nwarp * RB) {
      T ci[RB][JPL];
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const int i = i0 + r * nwarp;
        const T* Ci = A + static_cast<size_t>(i) * n;
#pragma unroll
        for (int c = 0; c < JPL; ++c) {
          const int j = lane + 32 * c;
          ci[r][c] = (i < n && j < n) ? Ci[j] : T(0);
        }
      }
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const int i = i0 + r * nwarp;
        if (i >= n) continue;
        T* Ci = A + static_cast<size_t>(i) * n;
        if (i == p || i == q) {
#pragma unroll
          for (int c = 0; c < JPL; ++c) {
            const int j = lane + 32 * c;
            if (j >= n) continue;
            T v;
            if (i == p) v = (j == q) ? -ia : (j == p ? T(0) : rq[c] * ia);
            else v = (j == p) ? ia : (j == q ? T(0) : -rp[c] * ia);
            Ci[j] = v;
          }
          continue;
        }
        const T rpi = rowp[i], rqi = rowq[i];
        const T cp = -rqi * ia, cq = rpi * ia;
#pragma unroll
        for (int c = 0; c < JPL; ++c) {
          const int j = lane + 32 * c;
          if (j >= n) continue;
          const T v = ci[r][c] + (rqi * rp[c] - rpi * rq[c]) * ia;
          Ci[j] = j == p ? cp : (j == q ? cq : v);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < JPL; ++c) {
      const int j = lane + 32 * c;
      if (j == p || j == q) swept |= 1u << c;
    }
    int nxt = n;
#pragma unroll
    for (int c = 0; c < JPL; ++c) {
      const int j = lane + 32 * c;
      if (j < n && !((swept >> c) & 1u) && j < nxt) nxt = j;
    }
    for (int off = 16; off > 0; off >>= 1) nxt = min(nxt, __shfl_xor_sync(0xffffffffu, nxt, off));
    p = nxt < n ? nxt : 0;
    __syncthreads();  // the swept rows are complete before the next snapshot
  }
  double v = (parity & 1) ? -pf : pf;
  if (status == 0 && !isfinite(v)) status = -1;
  if (status != 0) v = 0.0;
  pf_out = v;
  status_out = status;
  __syncthreads();
}

// Ping-pong form of the sweep: one barrier per pivot step. Every warp picks the pivot
// redundantly from the unmodified source buffer (identical data, identical choice), reads
// rows p and q from it, and writes the swept matrix into the other buffer. Lane l owns
// columns j = l + 32c (c < JPL), with the swept flags of its columns in registers.
// A holds X on entry; the result X⁻¹ is returned in A (B is scratch of the same size).
// n <= 32·JPL, lda = n. Same pivot rule and status codes as gj_pfinv.
template <typename T, int JPL, int RB = 1>
__device__ void gj_pfinv_pp(T* A, T* B, int n, double& pf_out, int& status_out) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  unsigned swept = 0;  // bit c: column lane + 32c swept
  int p = 0, parity = 0, status = 0;
  double pf = 1.0;
  T* C = A;
  T* D = B;
  for (int k = 0; k < n / 2; ++k) {
    const T* rowp = C + static_cast<size_t>(p) * n;
    T rp[JPL];
    double best = -1.0;
    int bi = n;
#pragma unroll
    for (int c = 0; c < JPL; ++c) {
      const int j = lane + 32 * c;
      rp[c] = j < n ? rowp[j] : T(0);
      if (j < n && j != p && !((swept >> c) & 1u)) {
        const double v = fabs(static_cast<double>(rp[c]));
        if (v > best) {
          best = v;
          bi = j;
        }
      }
    }
    warp_argmax_first(best, bi);
    const int q = __shfl_sync(0xffffffffu, bi, 0);
    best = __shfl_sync(0xffffffffu, best, 0);
    if (!(best > 0.0)) {
      status = p + 1;
      break;
    }
    // parity: unswept columns strictly between p and q
    int cnt = 0;
#pragma unroll
    for (int c = 0; c < JPL; ++c) {
      const int j = lane + 32 * c;
      cnt += (j < n && !((swept >> c) & 1u) && j > p && j < q) ? 1 : 0;
    }
    for (int off = 16; off > 0; off >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
    parity += cnt;
    const T* rowq = C + static_cast<size_t>(q) * n;
    const T a = rowp[q];
    pf *= static_cast<double>(a);
    const T ia = T(1) / a;
    T rq[JPL];
#pragma unroll
    for (int c = 0; c < JPL; ++c) {
      const int j = lane + 32 * c;
      rq[c] = j < n ? rowq[j] : T(0);
    }
    // RB rows per batch: their loads are issued before any store (RB > 1 for buffers in
    // global memory, where each row costs an L2 round trip)
    for (int i0 = warp; i0 < n; i0 += nwarp * RB) {
      T ci[RB][JPL];
      T rpi[RB], rqi[RB];
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const int i = i0 + r * nwarp;
        const T* Ci = C + static_cast<size_t>(i) * n;
        rpi[r] = i < n ? rowp[i] : T(0);
        rqi[r] = i < n ? rowq[i] : T(0);
#pragma unroll
        for (int c = 0; c < JPL; ++c) {
          const int j = lane + 32 * c;
          ci[r][c] = (i < n && j < n) ? Ci[j] : T(0);
        }
      }
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const int i = i0 + r * nwarp;
        if (i >= n) continue;
        T* Di = D + static_cast<size_t>(i) * n;
        if (i == p || i == q) {  // the pivot rows (uniform across the warp)
#pragma unroll
          for (int c = 0; c < JPL; ++c) {
            const int j = lane + 32 * c;
            if (j >= n) continue;
            T v;
            if (i == p) v = (j == q) ? -ia : (j == p ? T(0) : rq[c] * ia);
            else v = (j == p) ? ia : (j == q ? T(0) : -rp[c] * ia);
            Di[j] = v;
          }
          continue;
        }
        const T cp = -rqi[r] * ia, cq = rpi[r] * ia;  // columns p and q of this row
#pragma unroll
        for (int c = 0; c < JPL; ++c) {
          const int j = lane + 32 * c;
          if (j >= n) continue;
          const T v = ci[r][c] + (rqi[r] * rp[c] - rpi[r] * rq[c]) * ia;
          Di[j] = j == p ? cp : (j == q ? cq : v);
        }
      }
    }
    // mark p, q and find the next pivot row (smallest unswept index)
#pragma unroll
    for (int c = 0; c < JPL; ++c) {
      const int j = lane + 32 * c;
      if (j == p || j == q) swept |= 1u << c;
    }
    int nxt = n;
#pragma unroll
    for (int c = 0; c < JPL; ++c) {
      const int j = lane + 32 * c;
      if (j < n && !((swept >> c) & 1u) && j < nxt) nxt = j;
    }
    for (int off = 16; off > 0; off >>= 1) nxt = min(nxt, __shfl_xor_sync(0xffffffffu, nxt, off));
    p = nxt < n ? nxt : 0;
    __syncthreads();
    T* t = C;
    C = D;
    D = t;
  }
  if (C != A && status == 0) {
    for (int k = tid; k < n * n; k += nt) A[k] = C[k];
    __syncthreads();
  }
  double v = (parity & 1) ? -pf : pf;
  if (status == 0 && !isfinite(v)) status = -1;
  if (status != 0) v = 0.0;
  pf_out = v;
  status_out = status;
}

}  // namespace mvmcb

namespace mvmcb {

// Packed form of the sweep for planes whose full n×n FP64 matrix exceeds shared memory but
// whose strict upper triangle fits (n = 224: 195 KB): A(i, j), i < j, lives at
// P[rs[i] + j] with rs[i] = i·n − i(i+1)/2 − i − 1; A(j, i) = −A(i, j) and A(i, i) = 0, and
// the sweep keeps the matrix skew, so updating the triangle suffices (half the flops and
// bytes of the full sweep). Same pivot rule and status codes as gj_pfinv_pp; the element
// update A(i, j) += (A(q, i)/a)·A(p, j) − (A(p, i)/a)·A(q, j) scales the row coefficients
// first (two dependent FMAs per element). Per pivot step: every warp finds (p, q) redundantly from the snapshot of row
// p, the CTA snapshots row q (one barrier), then updates the triangle in place, writing
// the snapshot of the next pivot row as it goes (one barrier). rowp is [2][n] (double
// buffered), rowq [n]; on exit P holds the triangle of X⁻¹.
__device__ __forceinline__ double packed_at(const double* P, const int* rs, int i, int j) {
  return i < j ? P[rs[i] + j] : (i > j ? -P[rs[j] + i] : 0.0);
}

template <int JPL, int RB = 2>
__device__ void gj_pfinv_packed(double* P, const int* rs, int n, double* rowp2, double* rowq, double& pf_out,
                                int& status_out) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  unsigned swept = 0;  // bit c: column lane + 32c swept (identical in every warp)
  int p = 0, parity = 0, status = 0;
  double pf = 1.0;
  double* rowp = rowp2;
  for (int j = tid; j < n; j += nt) rowp[j] = packed_at(P, rs, 0, j);
  __syncthreads();
  for (int k = 0; k < n / 2; ++k) {
    // pivot q of row p: first maximum of |A(p, j)| over unswept j ≠ p (every warp)
    double best = -1.0;
    int bi = n;
#pragma unroll
    for (int c = 0; c < JPL; ++c) {
      const int j = lane + 32 * c;
      if (j < n && j != p && !((swept >> c) & 1u)) {
        const double v = fabs(rowp[j]);
        if (v > best) {
          best = v;
          bi = j;
        }
      }
    }
    warp_argmax_first(best, bi);
    const int q = __shfl_sync(0xffffffffu, bi, 0);
    best = __shfl_sync(0xffffffffu, best, 0);
    if (!(best > 0.0)) {
      status = p + 1;
      break;  // every warp read the same snapshot: all leave together
    }
    int cnt = 0;
#pragma unroll
    for (int c = 0; c < JPL; ++c) {
      const int j = lane + 32 * c;
      cnt += (j < n && !((swept >> c) & 1u) && j > p && j < q) ? 1 : 0;
    }
    for (int off = 16; off > 0; off >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
    parity += cnt;
    const double a = rowp[q];
    pf *= a;
    const double ia = 1.0 / a;
#pragma unroll
    for (int c = 0; c < JPL; ++c) {
      const int j = lane + 32 * c;
      if (j == p || j == q) swept |= 1u << c;
    }
    int pn = n;  // next pivot row: smallest unswept index
#pragma unroll
    for (int c = 0; c < JPL; ++c) {
      const int j = lane + 32 * c;
      if (j < n && !((swept >> c) & 1u) && j < pn) pn = j;
    }
    for (int off = 16; off > 0; off >>= 1) pn = min(pn, __shfl_xor_sync(0xffffffffu, pn, off));
    for (int j = tid; j < n; j += nt) rowq[j] = packed_at(P, rs, q, j);
    __syncthreads();
    double* rown = rowp == rowp2 ? rowp2 + n : rowp2;  // snapshot of the next pivot row
    if (tid == 0 && pn < n) rown[pn] = 0.0;
    // lane l owns columns j = l + 32c: the pivot rows' values of its columns stay in
    // registers for the whole step, and two rows' loads are issued before any store. Rows
    // p and q are rewritten by warps 0 and 1 after the others; in the other rows the
    // columns p, q and pn are single slots (c, lane) known before the loop, and chunks of
    // 32 columns that lie wholly left of the diagonal are skipped.
    double rp[JPL], rq[JPL];
#pragma unroll
    for (int c = 0; c < JPL; ++c) {
      const int j = lane + 32 * c;
      rp[c] = j < n ? rowp[j] : 0.0;
      rq[c] = j < n ? rowq[j] : 0.0;
    }
    const int cp_ = lane == (p & 31) ? p >> 5 : -1, cq_ = lane == (q & 31) ? q >> 5 : -1;
    const int cn_ = pn < n && lane == (pn & 31) ? pn >> 5 : -1;
    for (int i0 = warp; i0 < n - 1; i0 += nwarp * RB) {
      double x[RB][JPL];
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const int i = i0 + r * nwarp;
        const bool row_on = i < n - 1 && i != p && i != q;
#pragma unroll
        for (int c = 0; c < JPL; ++c) {
          const int j = lane + 32 * c;
          x[r][c] = (row_on && 32 * c + 31 > i && j > i && j < n) ? P[rs[i] + j] : 0.0;
        }
      }
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const int i = i0 + r * nwarp;
        if (i >= n - 1 || i == p || i == q) continue;
        // the row's coefficients scaled by 1/a first: two dependent FMAs per element
        const double ai = rowq[i] * ia, bi = rowp[i] * ia;
        double* Pi = P + rs[i];
        const bool is_pn = i == pn;
#pragma unroll
        for (int c = 0; c < JPL; ++c) {
          if (32 * c + 31 <= i) continue;  // wholly left of the diagonal (uniform)
          const int j = lane + 32 * c;
          if (j <= i || j >= n) continue;
          double v = x[r][c] + ai * rp[c] - bi * rq[c];
          if (c == cp_) v = -ai;  // column p
          if (c == cq_) v = bi;   // column q
          Pi[j] = v;
          if (is_pn) rown[j] = v;
          if (c == cn_) rown[i] = -v;  // column of the next pivot row
        }
      }
    }
    if (warp == 0 || warp == (1 % nwarp)) {  // rows p (warp 0) and q (warp 1)
      for (int which = (warp == 0 ? 0 : 1); which < 2; which += (nwarp > 1 ? 2 : 1)) {
        const int i = which == 0 ? p : q;
        double* Pi = P + rs[i];
#pragma unroll
        for (int c = 0; c < JPL; ++c) {
          const int j = lane + 32 * c;
          if (j <= i || j >= n) continue;
          const double v = which == 0 ? (j == q ? -ia : rq[c] * ia) : -rp[c] * ia;
          Pi[j] = v;
          if (c == cn_) rown[i] = -v;
        }
      }
    }
    p = pn < n ? pn : 0;
    rowp = rown;
    __syncthreads();
  }
  double v = (parity & 1) ? -pf : pf;
  if (status == 0 && !isfinite(v)) status = -1;
  if (status != 0) v = 0.0;
  pf_out = v;
  status_out = status;
  __syncthreads();
}

}  // namespace mvmcb
