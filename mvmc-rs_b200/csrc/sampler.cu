// K2: resident Metropolis sampler (one CTA per walker).
//
// Reproduces vmc_make_sample_real_engine (crates/mvmc-core/src/sampling/driver.rs:175-438)
// and HostEngine::run_block (sampling/engine.rs:188-476) of AtelierArith/mvmc-rs for the
// real sz-conserved path, with C's exact draw contract:
//   get_update_type (candidate.rs:320), make_candidate_hopping / _exchange
//   (candidate.rs:137,230), update_ele_config (projection.rs:418,441), log_proj_ratio
//   (projection.rs:403; for a hop in the direct-table form of the local energy's
//   projection ratio, exactly 0 for an exchange, with the counters rebuilt from the
//   configuration where a sample is saved), metropolis_decision (metropolis.rs:42-83), the
//   Pfaffian ratios and rank-2 / rank-4 updates (updates.rs:73,395,588,779,1154,1429),
//   and the refresh when the accept window exceeds Nsite (engine.rs:454-474).
// Thread 0 runs the serial Markov-chain logic from the walker's SFMT state in shared
// memory; the CTA runs the Pfaffian-ratio dots and the inverse updates over all QP
// planes at once. Planes live in shared memory when they fit, else in the walker's
// global slice (L2-resident working set).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "common.cuh"
#include "engine.cuh"
#include "pfinv.cuh"
#include "sfmt.cuh"

namespace mvmcb {


struct SampLayout {
  size_t sf, ctl, dctl, idx, cfg, num, cnt, pf, pfn, proj, qpw, jidx, vec, gj, ws, planes, total;
};

// The Jastrow index table is staged in shared memory for lattices up to this many sites.
constexpr int kJidxSmemSites = 96;

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

template <typename T>
__host__ __device__ inline SampLayout samp_layout(const DevModel& m, bool smem_planes, bool smem_ws) {
  SampLayout L;
  size_t o = 0;
  L.sf = o; o = align16(o + sizeof(uint32_t) * kSfmtN32);
  L.ctl = o; o = align16(o + sizeof(int) * 32);
  L.dctl = o; o = align16(o + sizeof(double) * 8);
  L.idx = o; o = align16(o + sizeof(int) * m.n);
  L.cfg = o; o = align16(o + sizeof(int) * m.ns2);
  L.num = o; o = align16(o + sizeof(int) * m.ns2);
  L.cnt = o; o = align16(o + sizeof(int) * (m.nproj + 1));
  L.pf = o; o = align16(o + sizeof(double) * m.nqp);
  L.pfn = o; o = align16(o + sizeof(double) * m.nqp);
  L.proj = o; o = align16(o + sizeof(double) * (m.nproj + 1));
  L.qpw = o; o = align16(o + sizeof(double) * m.nqp);
  L.jidx = o;
  if (m.ns <= kJidxSmemSites) o = align16(o + sizeof(int) * static_cast<size_t>(m.ns) * m.ns);
  L.vec = o; o = align16(o + sizeof(T) * 4 * static_cast<size_t>(m.nqp) * m.n + sizeof(double) * 8 * m.nqp);
  L.gj = o; o = align16(o + gj_shared_bytes<double>(m.n));
  L.ws = o;
  // FP64 sweep buffers: one scratch buffer beside FP64 planes in shared memory, else two
  // (the plane is gathered into the first).
  const size_t nn8 = sizeof(double) * static_cast<size_t>(m.n) * m.n;
  if (smem_ws) o = align16(o + (sizeof(T) == sizeof(double) && smem_planes ? nn8 : 2 * nn8));
  L.planes = o;
  if (smem_planes) o = align16(o + sizeof(T) * static_cast<size_t>(m.nqp) * m.n * m.n);
  L.total = o;
  return L;
}

// Control slots in shared memory.
enum Ctl {
  cSkip = 0, cType, cMi, cRi, cRj, cS, cMj, cT, cMsa, cMsb, cAccept, cRefresh, cInfo, cNacc,
  cBurn, cAttempt, cStop
};
enum DCtl { dLogIp = 0, dLogIpNew = 1, dDproj = 2, dRefreshMask = 3 };

template <typename T>
struct WalkerSmem {
  uint32_t* sf;
  int* ctl;
  double* dctl;
  int *idx, *cfg, *num, *cnt;
  double *pf, *pfn, *proj, *qpw;
  const int* jidx; // Jastrow index table (shared memory when small, else global)
  T* vec;          // [nqp][4][n]
  double* pscal;   // [nqp][8] per-plane scalars
  GJShared<double> gj;
  double* ws;      // FP64 sweep buffer (FP32 planes: the matrix; FP64 planes: the scratch)
  double* ws2;     // second FP64 sweep buffer
  T* planes;       // [nqp][n][n]
};

__device__ __forceinline__ int rs_of(const DevModel& m, const int* idx, int k) {
  return idx[k] + (k >= m.ne ? m.ns : 0);
}

template <typename T>
__device__ __forceinline__ T slater_at(const DevModel& m, int q, int r1, int r2);
template <>
__device__ __forceinline__ double slater_at<double>(const DevModel& m, int q, int r1, int r2) {
  return __ldg(m.slater + (static_cast<size_t>(q) * m.ns2 + r1) * m.ns2 + r2);
}
template <>
__device__ __forceinline__ float slater_at<float>(const DevModel& m, int q, int r1, int r2) {
  return __ldg(m.slater32 + (static_cast<size_t>(q) * m.ns2 + r1) * m.ns2 + r2);
}

// ---- projection counters --------------------------------------------------------------
__device__ void make_proj_cnt_serial(const DevModel& m, const int* num, int* cnt) {
  for (int k = 0; k < m.nproj; ++k) cnt[k] = 0;
  for (int ri = 0; ri < m.ns; ++ri) {
    const int g = m.gutz_idx[ri];
    if (m.n_gutz > 0 && g >= 0 && g < m.nproj) cnt[g] += num[ri] * num[ri + m.ns];
  }
  if (m.n_jast > 0)
    for (int ri = 0; ri < m.ns; ++ri) {
      const int xi = num[ri] + num[ri + m.ns] - 1;
      if (xi == 0) continue;
      for (int rj = ri + 1; rj < m.ns; ++rj) {
        const int j = __ldg(m.jast_idx + ri * m.ns + rj);
        if (j < 0) continue;
        const int xj = num[rj] + num[rj + m.ns] - 1;
        if (m.n_gutz + j < m.nproj) cnt[m.n_gutz + j] += xi * xj;
      }
    }
}

// Δ ln P of a hop from `source` to `dest` by one warp, `num` holding the configuration
// after the move: the direct-table form of Σ_k α_k (c'_k − c_k) (gutz_site[r] = α of r's
// Gutzwiller class, jast_pair[a·ns + b] = α of the Jastrow class of (a, b); the form of the
// local energy's projection ratio, observables.rs:1553-1640):
//   − g(source)·n(source) + g(dest)·n↑n↓(dest) + v(source, dest)·(x'_source − x'_dest + 1)
//   + Σ_{k ≠ source, dest} (v(dest, k) − v(source, k))·x_k,   x = n↑ + n↓ − 1.
// Mathematically the counters' sum; the projection counters themselves are not needed
// while the walker moves and are rebuilt from the configuration where a sample is saved.
__device__ __forceinline__ double log_proj_ratio_hop_warp(const DevModel& m, const int* num, int source, int dest) {
  const int lane = threadIdx.x & 31, ns = m.ns;
  double z = 0.0;
  if (m.n_jast > 0) {
    const double* vd = m.jast_pair + static_cast<size_t>(dest) * ns;
    const double* vs = m.jast_pair + static_cast<size_t>(source) * ns;
    // loads outside the branch and unrolled, so that a lane's table loads are all in flight
    // at once (the rows live in L2 for large lattices); the sum is the same as term by term
#pragma unroll 8
    for (int k = lane; k < ns; k += 32) {
      const int x = (k == source || k == dest) ? 0 : num[k] + num[k + ns] - 1;
      const double d = __ldg(vd + k) - __ldg(vs + k);
      if (x != 0) z += d * static_cast<double>(x);
    }
    z = warp_sum(z);
  }
  if (lane == 0) {
    const int xs = num[source] + num[source + ns] - 1, xd = num[dest] + num[dest + ns] - 1;
    z -= __ldg(m.gutz_site + source) * static_cast<double>(num[source] + num[source + ns]);
    z += __ldg(m.gutz_site + dest) * static_cast<double>(num[dest] * num[dest + ns]);
    z += __ldg(m.jast_pair + static_cast<size_t>(source) * ns + dest) * static_cast<double>(xs - xd + 1);
  }
  return z;
}

// Projection counters from the configuration by the whole CTA (make_proj_cnt,
// projection.rs:179): integer sums, so the order of the atomics does not matter.
__device__ void make_proj_cnt_cta(const DevModel& m, const int* jtab, const int* num, int* cnt) {
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  const int ns = m.ns;
  for (int k = tid; k < m.nproj; k += nt) cnt[k] = 0;
  __syncthreads();
  if (m.n_gutz > 0)
    for (int r = tid; r < ns; r += nt) {
      const int g = m.gutz_idx[r];
      const int v = num[r] * num[r + ns];
      if (v && g >= 0 && g < m.nproj) atomicAdd(cnt + g, v);
    }
  if (m.n_jast > 0)
    for (int ri = warp; ri < ns; ri += nwarp) {
      const int xi = num[ri] + num[ri + ns] - 1;
      if (xi == 0) continue;
      for (int rj = ri + 1 + lane; rj < ns; rj += 32) {
        const int j = jtab[ri * ns + rj];
        if (j < 0) continue;
        const int xj = num[rj] + num[rj + ns] - 1;
        if (xj != 0 && m.n_gutz + j < m.nproj) atomicAdd(cnt + m.n_gutz + j, xi * xj);
      }
    }
  __syncthreads();
}

// ---- CalculateMAll on every plane (CTA-wide); returns 0 ok, else the first failure -------
// FP64 planes are swept in place with ws as the ping-pong partner; FP32 planes are swept
// in FP64 in ws/ws2 and rounded into the plane (the FP64 refresh of the mixed path).
// FP64 refresh of every plane (CalculateMAll). The sweep runs in the FP64 buffers: in
// shared memory when they are there (the plane is gathered into the first buffer and the
// result copied to the plane), else in place on an FP64 plane in L2 (rows p, q of each
// pivot step snapshot in the shared GJ rows).
// mask: the planes to recompute (bit q; planes from 64 on always); the others keep their
// Pf and inverse.
template <typename T, int JPL, bool kSmemPlanes, bool kSmemWs>
__device__ int calc_m_all_dev(const DevModel& m, const WalkerSmem<T>& s, unsigned* status,
                              unsigned long long mask = ~0ull) {
  const int n = m.n;
  constexpr bool kFp64Planes = sizeof(T) == sizeof(double);
  // in place: FP64 planes in shared memory, or FP64 planes in L2 without shared buffers
  constexpr bool kInPlace = kFp64Planes && (kSmemPlanes || !kSmemWs);
  constexpr bool kSmemSweep = kInPlace ? kSmemPlanes : kSmemWs;
  constexpr int RB = kSmemSweep ? 1 : (JPL <= 2 ? 4 : (JPL <= 4 ? 2 : 1));
  int info = 0;
  for (int q = 0; q < m.nqp; ++q) {
    if (q < 64 && !((mask >> q) & 1ull)) continue;
    T* P = s.planes + static_cast<size_t>(q) * n * n;
    double* A = kInPlace ? reinterpret_cast<double*>(P) : s.ws;
    double* B = kInPlace ? s.ws : s.ws2;
    for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
      const int i = k / n, j = k - i * n;
      A[k] = __ldg(m.slater + (static_cast<size_t>(q) * m.ns2 + rs_of(m, s.idx, i)) * m.ns2 +
                   rs_of(m, s.idx, j));
    }
    __syncthreads();
    double pfv;
    int st;
    if constexpr (kInPlace && !kSmemPlanes)
      // FP64 plane in L2: swept in place (rows p, q in shared memory), so the resident
      // walkers' refreshes touch their own planes only
      gj_pfinv_ip<double, JPL, RB>(A, s.gj.rowp, n, pfv, st);
    else
      gj_pfinv_pp<double, JPL, RB>(A, B, n, pfv, st);
    if (!kInPlace) {
      for (int k = threadIdx.x; k < n * n; k += blockDim.x) P[k] = static_cast<T>(A[k]);
    }
    __syncthreads();
    if (st != 0) {
      info = st;
      break;
    }
    if (threadIdx.x == 0) s.pf[q] = pfv;
  }
  __syncthreads();
  return info;
}

__device__ __forceinline__ double log_ip_of(const DevModel& m, const double* pf, const double* qpw) {
  double ip = 0.0;
  for (int q = 0; q < m.nqp; ++q) ip += qpw[q] * pf[q];
  return log(fabs(ip));
}

// ---- Pfaffian ratio of a hop: pf_new[q] = -pf[q]·Σ_j InvM[q][msa][j]·S_q[rsa][rs_j] --------
// The gathered Slater row stays in vec slot 0 for the update of an accepted hop.
template <typename T>
__device__ void ratio_hop_dev(const DevModel& m, const WalkerSmem<T>& s, int msa) {
  const int n = m.n, lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int rsa = rs_of(m, s.idx, msa);
  // warps 1.. take the planes (warp 0 forms Δln P meanwhile)
  const int pw = nwarp > 1 ? nwarp - 1 : 1, wi = nwarp > 1 ? warp - 1 : warp;
  if (wi < 0) return;
  for (int q = wi; q < m.nqp; q += pw) {
    const T* row = s.planes + (static_cast<size_t>(q) * n + msa) * n;
    T* slt = s.vec + static_cast<size_t>(q) * 4 * n;
    T r = T(0);
    for (int j = lane; j < n; j += 32) {
      const T sj = slater_at<T>(m, q, rsa, rs_of(m, s.idx, j));
      slt[j] = sj;
      r += row[j] * sj;
    }
    r = warp_sum(r);
    if (lane == 0) s.pfn[q] = -static_cast<double>(r) * s.pf[q];
  }
}

// Column-form products over plane rows, out = Σ_i P[i·n + col]·v[i] (P points at the
// column), with independent accumulators so that several row loads are in flight. A
// thread with two columns walks both together (eight loads in flight).
template <typename T>
__device__ __forceinline__ T col_dot(const T* __restrict__ P, const T* __restrict__ v, int n) {
  T a0 = T(0), a1 = T(0), a2 = T(0), a3 = T(0);
  int i = 0;
  for (; i + 4 <= n; i += 4) {
    a0 += P[(i + 0) * n] * v[i + 0];
    a1 += P[(i + 1) * n] * v[i + 1];
    a2 += P[(i + 2) * n] * v[i + 2];
    a3 += P[(i + 3) * n] * v[i + 3];
  }
  for (; i < n; ++i) a0 += P[i * n] * v[i];
  return (a0 + a1) + (a2 + a3);
}

template <typename T>
__device__ __forceinline__ void col_dot_pair(const T* __restrict__ P0, const T* __restrict__ v0,
                                             const T* __restrict__ P1, const T* __restrict__ v1, int n, T& r0,
                                             T& r1) {
  T a[4], b[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) a[u] = b[u] = T(0);
  int i = 0;
  for (; i + 4 <= n; i += 4) {
    T x[4], y[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      x[u] = P0[(i + u) * n];
      y[u] = P1[(i + u) * n];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a[u] += x[u] * v0[i + u];
      b[u] += y[u] * v1[i + u];
    }
  }
  for (; i < n; ++i) {
    a[0] += P0[i * n] * v0[i];
    b[0] += P1[i * n] * v1[i];
  }
  r0 = (a[0] + a[1]) + (a[2] + a[3]);
  r1 = (b[0] + b[1]) + (b[2] + b[3]);
}

// Column range [i0, i1) of col_dot.
// Sixteen row loads in flight per thread, eight accumulators (planes in L2 are latency
// bound; sixteen against eight: 2D 16x16 FP64 sampling 3 % faster).
template <typename T>
__device__ __forceinline__ T col_dot_range(const T* __restrict__ P, const T* __restrict__ v, int n, int i0,
                                           int i1) {
  T a[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) a[u] = T(0);
  int i = i0;
  for (; i + 16 <= i1; i += 16) {
    T x[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) x[u] = P[(i + u) * n];
#pragma unroll
    for (int u = 0; u < 16; ++u) a[u & 7] += x[u] * v[i + u];
  }
  for (; i + 8 <= i1; i += 8) {
    T x[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) x[u] = P[(i + u) * n];
#pragma unroll
    for (int u = 0; u < 8; ++u) a[u] += x[u] * v[i + u];
  }
  for (; i < i1; ++i) a[0] += P[i * n] * v[i];
  return ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
}

// out[q][j] = −Σ_i P_q[i][j]·vec[q][in][i] → vec[q][out] for every (plane, column), two
// columns per thread where there are enough. With fewer columns than threads (one wide
// plane) each column is split into two row halves on two threads, the second half
// parked in slot 3 and added in order after a barrier. Ends without a barrier.
template <typename T>
__device__ __forceinline__ void planes_col_dot(const DevModel& m, const WalkerSmem<T>& s, int in, int out) {
  const int n = m.n, total = m.nqp * n, nt = blockDim.x;
  if (total <= nt && out != 3 && in != 3) {
    const int half = ((n + 1) / 2 + 3) & ~3;
    for (int k = threadIdx.x; k < 2 * total; k += nt) {
      const int seg = k / total, kk = k - seg * total;
      const int q = kk / n, j = kk - q * n;
      const T* P = s.planes + static_cast<size_t>(q) * n * n + j;
      const int i0 = seg ? min(half, n) : 0, i1 = seg ? n : min(half, n);
      const T r = col_dot_range(P, s.vec + (q * 4 + in) * n, n, i0, i1);
      s.vec[(q * 4 + (seg ? 3 : out)) * n + j] = r;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < total; k += nt) {
      const int q = k / n, j = k - q * n;
      s.vec[(q * 4 + out) * n + j] = -(s.vec[(q * 4 + out) * n + j] + s.vec[(q * 4 + 3) * n + j]);
    }
    return;
  }
  for (int k = threadIdx.x; k < total; k += 2 * nt) {
    const int q = k / n, j = k - q * n;
    const T* P = s.planes + static_cast<size_t>(q) * n * n + j;
    const int k2 = k + nt;
    if (k2 < total) {
      const int q2 = k2 / n, j2 = k2 - q2 * n;
      T r0, r1;
      col_dot_pair(P, s.vec + (q * 4 + in) * n, s.planes + static_cast<size_t>(q2) * n * n + j2,
                   s.vec + (q2 * 4 + in) * n, n, r0, r1);
      s.vec[(q * 4 + out) * n + j] = -r0;
      s.vec[(q2 * 4 + out) * n + j2] = -r1;
    } else {
      s.vec[(q * 4 + out) * n + j] = -col_dot(P, s.vec + (q * 4 + in) * n, n);
    }
  }
}

template <typename T>
__device__ __forceinline__ void col_dot2(const T* __restrict__ P, const T* __restrict__ v,
                                         const T* __restrict__ u, int n, T& pv, T& pu) {
  T a[4], b[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) a[k] = b[k] = T(0);
  int i = 0;
  for (; i + 4 <= n; i += 4) {
    T x[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) x[k] = P[(i + k) * n];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      a[k] += x[k] * v[i + k];
      b[k] += x[k] * u[i + k];
    }
  }
  for (; i < n; ++i) {
    const T x = P[i * n];
    a[0] += x * v[i];
    b[0] += x * u[i];
  }
  pv = (a[0] + a[1]) + (a[2] + a[3]);
  pu = (b[0] + b[1]) + (b[2] + b[3]);
}

// Lane-owned columns: lane l of every warp owns columns j = l + 32c (c < JPL) of every
// plane row it touches, so column vectors of the rank-2/rank-4 updates sit in registers
// and only the row scalars are broadcast from shared memory.

// ---- rank-2 update of an accepted hop (update_one_real, updates.rs:1154-1215) --------------
//   vec1 = −InvMᵀ·slt,  pf ← −pf·vec1[msa],  vec2 = InvM[msa]·(−1/vec1[msa]),
//   InvM += vec1⊗vec2 − vec2⊗vec1, then column msa −= vec2 and row msa += vec2.
// gathered: slt is already in vec slot 0 (ratio_hop_dev of the same proposal, followed by a
// barrier).
template <typename T, int JPL>
__device__ void update_hop_dev(const DevModel& m, const WalkerSmem<T>& s, int msa, bool gathered) {
  const int n = m.n, nq = m.nqp, tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  const int rsa = rs_of(m, s.idx, msa);
  T* vec = s.vec;  // [q][0]=slt, [1]=vec1, [2]=vec2
  if (!gathered) {
    for (int k = tid; k < nq * n; k += nt) {
      const int q = k / n, i = k - q * n;
      vec[(q * 4 + 0) * n + i] = slater_at<T>(m, q, rsa, rs_of(m, s.idx, i));
    }
    __syncthreads();
  }
  planes_col_dot(m, s, 0, 1);  // vec1
  __syncthreads();
  for (int k = tid; k < nq * n; k += nt) {
    const int q = k / n, j = k - q * n;
    const T tmp = vec[(q * 4 + 1) * n + msa];
    const T ia = T(-1) / tmp;
    vec[(q * 4 + 2) * n + j] = s.planes[(static_cast<size_t>(q) * n + msa) * n + j] * ia;
    if (j == 0) s.pf[q] *= -static_cast<double>(tmp);
  }
  __syncthreads();
  const int cmsa = msa >> 5, lmsa = msa & 31;
  for (int q = 0; q < nq; ++q) {
    const T* v1 = vec + (q * 4 + 1) * n;
    const T* v2 = vec + (q * 4 + 2) * n;
    T v1c[JPL], v2c[JPL];
#pragma unroll
    for (int c = 0; c < JPL; ++c) {
      const int j = lane + 32 * c;
      v1c[c] = j < n ? v1[j] : T(0);
      v2c[c] = j < n ? v2[j] : T(0);
    }
    T* P = s.planes + static_cast<size_t>(q) * n * n;
    // rows per batch (their loads are issued before any store), fewer for wide rows so
    // that several walkers fit an SM's register file; two for the widest rows, whose
    // planes live in L2 where one batch of seven loads leaves the SM latency bound
    constexpr int RB = JPL <= 2 ? 4 : 2;
    for (int i0 = warp; i0 < n; i0 += nwarp * RB) {
      T x[RB][JPL];
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const int i = i0 + r * nwarp;
#pragma unroll
        for (int c = 0; c < JPL; ++c) {
          const int j = lane + 32 * c;
          x[r][c] = (i < n && j < n) ? P[static_cast<size_t>(i) * n + j] : T(0);
        }
      }
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const int i = i0 + r * nwarp;
        if (i >= n || i == msa) continue;
        const T v1i = v1[i], v2i = v2[i];
        T* Pi = P + static_cast<size_t>(i) * n;
#pragma unroll
        for (int c = 0; c < JPL; ++c) {
          const int j = lane + 32 * c;
          if (j < n) {
            T y = x[r][c] + (v1i * v2c[c] - v1c[c] * v2i);
            if (c == cmsa && lane == lmsa) y -= v2i;  // column msa of this row
            Pi[j] = y;
          }
        }
      }
    }
    for (int i = warp; i < n; i += nwarp) {
      if (i != msa) continue;
      const T v1i = v1[i], v2i = v2[i];
      T* Pi = P + static_cast<size_t>(i) * n;
      {
#pragma unroll
        for (int c = 0; c < JPL; ++c) {
          const int j = lane + 32 * c;
          if (j < n) {
            T x = Pi[j] + (v1i * v2c[c] - v1c[c] * v2i);
            if (c == cmsa && lane == lmsa) x -= v2i;
            Pi[j] = x + v2c[c];
          }
        }
      }
    }
  }
  __syncthreads();
}

// ---- exchange ratio (two_ratio_real, updates.rs:1539-1622) --------------------------------
//   ratio = InvM_ab·vb_a + InvM_ab·(vbᵀ·InvM·va) + p_a q_b − p_b q_a
template <typename T, int JPL>
__device__ void ratio_exchange_dev(const DevModel& m, const WalkerSmem<T>& s, int msa, int msb) {
  const int n = m.n, nq = m.nqp, tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  const int rsa = rs_of(m, s.idx, msa), rsb = rs_of(m, s.idx, msb);
  T* vec = s.vec;  // [0]=va, [1]=vb, [2]=InvM·va
  for (int k = tid; k < nq * n; k += nt) {
    const int q = k / n, i = k - q * n;
    const int ri = rs_of(m, s.idx, i);
    vec[(q * 4 + 0) * n + i] = slater_at<T>(m, q, rsa, ri);
    vec[(q * 4 + 1) * n + i] = slater_at<T>(m, q, rsb, ri);
  }
  __syncthreads();
  // (InvM·va)[i] = −Σ_j InvM[j][i]·va[j] (skew symmetry)
  planes_col_dot(m, s, 0, 2);
  __syncthreads();
  for (int q = warp; q < nq; q += nwarp) {
    const T* P = s.planes + static_cast<size_t>(q) * n * n;
    const T* va = vec + (q * 4 + 0) * n;
    const T* vb = vec + (q * 4 + 1) * n;
    const T* ia = vec + (q * 4 + 2) * n;
    T pa = 0, pb = 0, qa = 0, qb = 0, bma = 0;
    for (int i = lane; i < n; i += 32) {
      pa += P[msa * n + i] * va[i];
      pb += P[msb * n + i] * va[i];
      qa += P[msa * n + i] * vb[i];
      qb += P[msb * n + i] * vb[i];
      bma += vb[i] * ia[i];
    }
    pa = warp_sum(pa);
    pb = warp_sum(pb);
    qa = warp_sum(qa);
    qb = warp_sum(qb);
    bma = warp_sum(bma);
    if (lane == 0) {
      const T iab = P[msa * n + msb];
      const T ratio = iab * vb[msa] + iab * bma + pa * qb - pb * qa;
      s.pfn[q] = static_cast<double>(ratio) * s.pf[q];
    }
  }
}

// ---- rank-4 update of an accepted exchange (update_two_real, updates.rs:1429-1505) --------
// gathered: va and vb of ratio_exchange_dev (same proposal) are still in vec slots 0 and 1;
// only entry msb of vs differs from va.
template <typename T, int JPL>
__device__ void update_exchange_dev(const DevModel& m, const WalkerSmem<T>& s, int msa, int msb,
                                    int rsa_old, int rsb_old, bool gathered) {
  const int n = m.n, nq = m.nqp, tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  const int rsa = rs_of(m, s.idx, msa), rsb = rs_of(m, s.idx, msb);
  T* vec = s.vec;  // [0]=vs, [1]=vt, [2]=vp, [3]=vq
  if (gathered) {
    for (int q = tid; q < nq; q += nt) vec[(q * 4 + 0) * n + msb] = slater_at<T>(m, q, rsa_old, rsb_old);
  } else {
    for (int k = tid; k < nq * n; k += nt) {
      const int q = k / n, i = k - q * n;
      const int ri = rs_of(m, s.idx, i);
      vec[(q * 4 + 0) * n + i] = (i == msb) ? slater_at<T>(m, q, rsa_old, rsb_old) : slater_at<T>(m, q, rsa, ri);
      vec[(q * 4 + 1) * n + i] = slater_at<T>(m, q, rsb, ri);
    }
  }
  __syncthreads();
  // vp = InvM·vs, vq = InvM·vt in column form (skew symmetry)
  for (int k = tid; k < nq * n; k += nt) {
    const int q = k / n, i = k - q * n;
    const T* P = s.planes + static_cast<size_t>(q) * n * n + i;
    T p, r;
    col_dot2(P, vec + (q * 4 + 0) * n, vec + (q * 4 + 1) * n, n, p, r);
    vec[(q * 4 + 2) * n + i] = -p;
    vec[(q * 4 + 3) * n + i] = -r;
  }
  __syncthreads();
  double* sc = s.pscal;  // per plane: a b c d e f idet det
  for (int q = warp; q < nq; q += nwarp) {
    const T* vt = vec + (q * 4 + 1) * n;
    const T* vp = vec + (q * 4 + 2) * n;
    const T* vq = vec + (q * 4 + 3) * n;
    T bma = T(0);
    for (int i = lane; i < n; i += 32) bma += vt[i] * vp[i];
    bma = warp_sum(bma);
    if (lane == 0) {
      const T* P = s.planes + static_cast<size_t>(q) * n * n;
      const T iab = P[msa * n + msb];
      const T ratio = iab * vt[msa] + iab * bma + vp[msa] * vq[msb] - vp[msb] * vq[msa];
      s.pf[q] *= static_cast<double>(ratio);
      const T a = -vp[msa], b = vp[msb], c = vq[msa], d = -vq[msb];
      const T e = -bma - vt[msa], f = iab;
      const T det = a * d - b * c - e * f;
      const T idet = T(1) / det;
      double* o = sc + q * 8;
      o[0] = a; o[1] = b; o[2] = c; o[3] = d; o[4] = e; o[5] = f; o[6] = idet; o[7] = det;
    }
  }
  __syncthreads();
  // vs <- idet·InvM[msa][:], vt <- idet·InvM[msb][:]
  for (int k = tid; k < nq * n; k += nt) {
    const int q = k / n, i = k - q * n;
    const T idet = static_cast<T>(sc[q * 8 + 6]);
    const T* P = s.planes + static_cast<size_t>(q) * n * n;
    vec[(q * 4 + 0) * n + i] = idet * P[msa * n + i];
    vec[(q * 4 + 1) * n + i] = idet * P[msb * n + i];
  }
  __syncthreads();
  for (int q = 0; q < nq; ++q) {
    const double* o = sc + q * 8;
    const T a = o[0], b = o[1], c = o[2], d = o[3], e = o[4], f = o[5], idet = o[6], det = o[7];
    const T edet = e * det, fidet = f * idet;
    const T* vs = vec + (q * 4 + 0) * n;
    const T* vt = vec + (q * 4 + 1) * n;
    const T* vp = vec + (q * 4 + 2) * n;
    const T* vq = vec + (q * 4 + 3) * n;
    // The rank-4 correction (plus the row/column fixes of slots msa, msb) as four column
    // vectors with per-row coefficients: x_ij += Ct_i·t_j + Cs_i·s_j + Cq_i·q'_j + Cp_i·p'_j,
    // p' = p + e_msa, q' = q + e_msb (the column fixes); the row fixes enter Ct..Cp of rows
    // msa and msb.
    T pc[JPL], qc[JPL], sc_[JPL], tc[JPL];
#pragma unroll
    for (int c2 = 0; c2 < JPL; ++c2) {
      const int j = lane + 32 * c2;
      pc[c2] = j < n ? vp[j] + (j == msa ? T(1) : T(0)) : T(0);
      qc[c2] = j < n ? vq[j] + (j == msb ? T(1) : T(0)) : T(0);
      sc_[c2] = j < n ? vs[j] : T(0);
      tc[c2] = j < n ? vt[j] : T(0);
    }
    T* P = s.planes + static_cast<size_t>(q) * n * n;
    constexpr int RB = JPL <= 2 ? 2 : 1;  // rows per batch: their loads are issued before any store
    for (int i0 = warp; i0 < n; i0 += nwarp * RB) {
      T xl[RB][JPL];
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const int i = i0 + r * nwarp;
#pragma unroll
        for (int c2 = 0; c2 < JPL; ++c2) {
          const int j = lane + 32 * c2;
          xl[r][c2] = (i < n && j < n) ? P[i * n + j] : T(0);
        }
      }
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const int i = i0 + r * nwarp;
        if (i >= n) continue;
        const T pi = vp[i], qi = vq[i], si = vs[i], ti = vt[i];
        T ct = a * qi + c * pi + edet * si;
        T cs = b * qi + d * pi - edet * ti;
        T cq = fidet * pi - a * ti - b * si;
        T cp = -(c * ti + d * si + fidet * qi);
        if (i == msa) {
          ct += c;
          cs += d;
          cq += fidet;
        }
        if (i == msb) {
          ct += a;
          cs += b;
          cp -= fidet;
        }
        T* Pi = P + i * n;
#pragma unroll
        for (int c2 = 0; c2 < JPL; ++c2) {
          const int j = lane + 32 * c2;
          if (j < n) Pi[j] = xl[r][c2] + (ct * tc[c2] + cs * sc_[c2] + cq * qc[c2] + cp * pc[c2]);
        }
      }
    }
  }
  __syncthreads();
}

// ---- serial helpers for thread 0 ------------------------------------------------------------
__device__ __forceinline__ void move_electron(const DevModel& m, int* idx, int* cfg, int* num, int mi,
                                              int ri, int rj, int sp) {
  const int msa = mi + sp * m.ne, ro = ri + sp * m.ns, rn = rj + sp * m.ns;
  idx[msa] = rj;
  cfg[ro] = -1;
  cfg[rn] = mi;
  num[ro] = 0;
  num[rn] = 1;
}
__device__ __forceinline__ void revert_electron(const DevModel& m, int* idx, int* cfg, int* num, int mi,
                                                int ri, int rj, int sp) {
  const int msa = mi + sp * m.ne, ro = ri + sp * m.ns, rn = rj + sp * m.ns;
  idx[msa] = ri;
  cfg[ro] = mi;
  cfg[rn] = -1;
  num[ro] = 1;
  num[rn] = 0;
}

__device__ void make_initial_sample_dev(const DevModel& m, SfmtRef& rng, int* idx, int* cfg, int* num,
                                        int* cnt) {
  for (int k = 0; k < m.n; ++k) idx[k] = -1;
  for (int k = 0; k < m.ns2; ++k) cfg[k] = -1;
  for (int si = 0; si < 2; ++si)
    for (int mi = 0; mi < m.ne; ++mi) {
      int guard = 0;
      while (true) {
        const int ri = static_cast<int>(rng.mod(m.ns));
        if (cfg[ri + si * m.ns] == -1) {
          cfg[ri + si * m.ns] = mi;
          idx[mi + si * m.ne] = ri;
          break;
        }
        if (++guard > (1 << 24)) break;  // unreachable for ne <= nsite
      }
    }
  for (int r = 0; r < m.ns2; ++r) num[r] = cfg[r] < 0 ? 0 : 1;
  make_proj_cnt_serial(m, num, cnt);
}

// Walkers per SM the register budget is sized for: one when the planes are in shared
// memory; with planes in L2, enough CTAs for 16 warps per SM (a tighter budget spills).
template <int NT, bool kSmemPlanes>
struct SampOccupancy {
  static constexpr int kBlocks = kSmemPlanes ? 1 : (512 / NT);
};

template <typename T, int JPL, int NT, bool kSmemPlanes, bool kSmemWs>
__global__ void __launch_bounds__(NT, (SampOccupancy<NT, kSmemPlanes>::kBlocks)) k_sample(DevModel m, DevWalkers w) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int wk = blockIdx.x;
  const int tid = threadIdx.x;
  const SampLayout L = samp_layout<T>(m, kSmemPlanes, kSmemWs);
  WalkerSmem<T> s;
  s.sf = reinterpret_cast<uint32_t*>(smem + L.sf);
  s.ctl = reinterpret_cast<int*>(smem + L.ctl);
  s.dctl = reinterpret_cast<double*>(smem + L.dctl);
  s.idx = reinterpret_cast<int*>(smem + L.idx);
  s.cfg = reinterpret_cast<int*>(smem + L.cfg);
  s.num = reinterpret_cast<int*>(smem + L.num);
  s.cnt = reinterpret_cast<int*>(smem + L.cnt);
  s.pf = reinterpret_cast<double*>(smem + L.pf);
  s.pfn = reinterpret_cast<double*>(smem + L.pfn);
  s.proj = reinterpret_cast<double*>(smem + L.proj);
  s.qpw = reinterpret_cast<double*>(smem + L.qpw);
  if (m.ns <= kJidxSmemSites) {
    int* jt = reinterpret_cast<int*>(smem + L.jidx);
    for (int k = threadIdx.x; k < m.ns * m.ns; k += blockDim.x) jt[k] = m.jast_idx[k];
    s.jidx = jt;
  } else {
    s.jidx = m.jast_idx;
  }
  s.vec = reinterpret_cast<T*>(smem + L.vec);
  s.pscal = reinterpret_cast<double*>(smem + L.vec + sizeof(T) * 4 * static_cast<size_t>(m.nqp) * m.n);
  s.gj = gj_carve<double>(smem + L.gj, m.n);
  const size_t nn = static_cast<size_t>(m.n) * m.n;
  if (kSmemWs) {
    s.ws = reinterpret_cast<double*>(smem + L.ws);
    s.ws2 = s.ws + nn;
  } else {
    s.ws = w.ws64 + static_cast<size_t>(wk) * 2 * nn;
    s.ws2 = s.ws + nn;
  }
  s.planes = kSmemPlanes ? reinterpret_cast<T*>(smem + L.planes)
                         : reinterpret_cast<T*>(w.inv) + static_cast<size_t>(wk) * m.nqp * nn;

  // ---- load the walker ----
  for (int k = tid; k < kSfmtN32; k += blockDim.x) s.sf[k] = w.sfmt[static_cast<size_t>(wk) * kSfmtN32 + k];
  for (int k = tid; k < m.n; k += blockDim.x) s.idx[k] = w.ele_idx[static_cast<size_t>(wk) * m.n + k];
  for (int k = tid; k < m.ns2; k += blockDim.x) {
    s.cfg[k] = w.ele_cfg[static_cast<size_t>(wk) * m.ns2 + k];
    s.num[k] = w.ele_num[static_cast<size_t>(wk) * m.ns2 + k];
  }
  for (int k = tid; k < m.nproj; k += blockDim.x) {
    s.cnt[k] = w.proj_cnt[static_cast<size_t>(wk) * m.nproj + k];
    s.proj[k] = m.proj[k];
  }
  for (int k = tid; k < m.nqp; k += blockDim.x) s.qpw[k] = m.qpw[k];
  // the generator's cursor and word count live in thread 0's registers (only thread 0 draws)
  int sf_idx = 0;
  unsigned long long sf_draws = 0;
  if (tid == 0) {
    sf_idx = w.sfmt_idx[wk];
    sf_draws = w.draws[wk];
    s.ctl[cBurn] = w.burn[wk];
  }
  __syncthreads();
  SfmtRef rng{s.sf, &sf_idx, &sf_draws};
  const int n = m.n, ns = m.ns, ne = m.ne;
  bool burn = s.ctl[cBurn] != 0;

  // ---- initial configuration (makeInitialSample with the C retry rule) ----
  auto initial = [&]() {
    for (int attempt = 1; attempt <= 101; ++attempt) {
      if (tid == 0) make_initial_sample_dev(m, rng, s.idx, s.cfg, s.num, s.cnt);
      __syncthreads();
      const int info = calc_m_all_dev<T, JPL, kSmemPlanes, kSmemWs>(m, s, w.status);
      if (attempt > 100) {
        if (tid == 0) atomicOr(w.status, kDevInitLoops);
        return;
      }
      if (info <= 0) return;
    }
  };
  if (!burn) initial();
  calc_m_all_dev<T, JPL, kSmemPlanes, kSmemWs>(m, s, w.status);
  if (tid == 0) s.dctl[dLogIp] = log_ip_of(m, s.pf, s.qpw);
  __syncthreads();
  if (!isfinite(s.dctl[dLogIp])) {
    initial();
    calc_m_all_dev<T, JPL, kSmemPlanes, kSmemWs>(m, s, w.status);
    if (tid == 0) s.dctl[dLogIp] = log_ip_of(m, s.pf, s.qpw);
    burn = false;
    __syncthreads();
  }
  const int S = m.saved;
  const int n_out = burn ? S + 1 : m.warmup + S;
  const int n_in = m.interval * max(1, ns);
  long long counter[6] = {0, 0, 0, 0, 0, 0};
  int n_acc_win = 0;
  const int refresh_every = (sizeof(T) == sizeof(float) && w.refresh_sweeps > 0) ? w.refresh_sweeps * max(1, ns) : 0;
  long long since_refresh = 0;
  double drift_max = 0.0;
  long long n_sched = 0, n_guard = 0;  // scheduled and guard-triggered refreshes

  long long proposal = 0;
  unsigned long long ph[kPhCount] = {0, 0, 0, 0, 0, 0, 0, 0};
  const bool timing = w.timers != nullptr && tid == 0;
  unsigned long long t_last = timing ? clock64() : 0ULL;
  const unsigned long long t_begin = t_last;
  auto lap = [&](int phase) {
    if (timing) {
      const unsigned long long t = clock64();
      ph[phase] += t - t_last;
      t_last = t;
    }
  };
  for (int out = 0; out < n_out; ++out) {
    for (int step = 0; step < n_in; ++step, ++proposal) {
      // Candidate slots alternate between two banks: a skipped proposal has no later
      // barrier, so the next proposal must not overwrite the bank still being read.
      int* const cc = s.ctl + ((proposal & 1) ? 16 : 0);
      // --- candidate (thread 0) ---
      if (tid == 0) {
        ++since_refresh;  // proposal attempts since the last FP64 refresh (mixed path)
        int type;
        switch (m.nex_path) {
          case 0: type = 0; break;
          case 1: type = rng.real2() < 0.5 ? 1 : 0; break;
          case 2: type = 1; break;
          default: type = 3;
        }
        int skip = 1;
        if (type == 0) {
          counter[0]++;
          const int mi = static_cast<int>(rng.mod(ne));
          const int sp = rng.real2() < 0.5 ? 0 : 1;
          const int ri = s.idx[mi + sp * ne];
          int rj = 0, icnt = 0;
          bool reject = false;
          const int icnt_max = ns * ns;
          while (true) {
            rj = static_cast<int>(rng.mod(ns));
            if (icnt > icnt_max) {
              reject = true;
              break;
            }
            ++icnt;
            if (s.cfg[rj + sp * ns] == -1) break;
          }
          if (!reject) {
            move_electron(m, s.idx, s.cfg, s.num, mi, ri, rj, sp);
            cc[cMi] = mi; cc[cRi] = ri; cc[cRj] = rj; cc[cS] = sp;
            cc[cMsa] = mi + sp * ne;
            skip = 0;
          }
        } else if (type == 1) {
          counter[2]++;
          bool single = false;
          for (int r = 0; r < ns; ++r)
            if (s.num[r] + s.num[r + ns] == 1) {
              single = true;
              break;
            }
          if (single) {
            int mi, sp, ri, mj, rj;
            // The C loops are unbounded; a partner always exists for sz-balanced
            // configurations. The bound only turns a malformed input into a status bit.
            constexpr int kLoopBound = 1 << 22;
            int guard = 0;
            while (true) {
              mi = static_cast<int>(rng.mod(ne));
              sp = rng.real2() < 0.5 ? 0 : 1;
              ri = s.idx[mi + sp * ne];
              if (s.cfg[ri + (1 - sp) * ns] == -1 || ++guard > kLoopBound) break;
            }
            const int t = 1 - sp;
            while (guard <= kLoopBound) {
              mj = static_cast<int>(rng.mod(ne));
              rj = s.idx[mj + t * ne];
              if (s.cfg[rj + sp * ns] == -1 || ++guard > kLoopBound) break;
            }
            if (guard > kLoopBound) {
              atomicOr(w.status, kDevCandidateLoop);  // skip stays 1: no move is made
            } else {
              move_electron(m, s.idx, s.cfg, s.num, mi, ri, rj, sp);
              move_electron(m, s.idx, s.cfg, s.num, mj, rj, ri, t);
              cc[cMi] = mi; cc[cRi] = ri; cc[cRj] = rj; cc[cS] = sp;
              cc[cMj] = mj; cc[cT] = t;
              cc[cMsa] = mi + sp * ne;
              cc[cMsb] = mj + t * ne;
              skip = 0;
            }
          }
        }
        cc[cType] = type;
        cc[cSkip] = skip;
      }
      __syncthreads();
      lap(kPhCandidate);
      if (cc[cSkip]) continue;
      const int type = cc[cType];
      const int ri = cc[cRi], rj = cc[cRj], sp = cc[cS], msa = cc[cMsa];
      // --- Δ ln P (warp 0) and Pfaffian ratios (CTA) ---
      if (type == 0) {
        if (tid < 32) {
          const double z = log_proj_ratio_hop_warp(m, s.num, ri, rj);
          if (tid == 0) s.dctl[dDproj] = z;
        }
        ratio_hop_dev<T>(m, s, msa);
      } else {
        // an exchange keeps every site's charge and double occupancy: every projection
        // counter is unchanged and Σ_k α_k (c'_k − c_k) is exactly 0
        if (tid == 0) s.dctl[dDproj] = 0.0;
        ratio_exchange_dev<T, JPL>(m, s, msa, cc[cMsb]);
      }
      __syncthreads();
      lap(kPhRatio);
      // --- Metropolis (thread 0) ---
      if (tid == 0) {
        double ip = 0.0;
        for (int q = 0; q < m.nqp; ++q) ip += s.qpw[q] * s.pfn[q];
        const double lip_new = log(fabs(ip));
        const double dproj = s.dctl[dDproj];
        double wgt = exp(2.0 * ((dproj + 0.0 + lip_new) - s.dctl[dLogIp]));
        if (!isfinite(wgt)) wgt = -1.0;
        const double u = rng.real2();
        const int acc = wgt > u ? 1 : 0;
        unsigned long long guard = 0ull;  // planes whose ratio tripped the guard
        if (acc) {
          s.dctl[dLogIp] = lip_new;
          ++n_acc_win;
          if (type == 0) counter[1]++;
          else counter[3]++;
          if (w.refresh_guard > 0.0) {
            // a plane whose Pfaffian ratio leaves [g, 1/g] passes near a singular matrix:
            // the rank-2 update amplifies the inverse's rounding error by about 1/|ratio|
            for (int q = 0; q < m.nqp; ++q) {
              const double r = fabs(s.pfn[q] / s.pf[q]);
              if (!(r >= w.refresh_guard && r * w.refresh_guard <= 1.0)) guard |= q < 64 ? (1ull << q) : ~0ull;
            }
          }
        } else if (type == 0) {
          revert_electron(m, s.idx, s.cfg, s.num, cc[cMi], ri, rj, sp);
        } else {
          revert_electron(m, s.idx, s.cfg, s.num, cc[cMj], rj, ri, cc[cT]);
          revert_electron(m, s.idx, s.cfg, s.num, cc[cMi], ri, rj, sp);
        }
        cc[cAccept] = acc;
        int refresh = 0;
        if (refresh_every > 0) {
          // mixed path: FP64 refresh of Pf and X⁻¹ every NRefresh sweeps
          if (since_refresh >= refresh_every) refresh = 2;
        } else if (n_acc_win > ns) {
          refresh = 1;  // C rule: recompute when the accept window exceeds Nsite
          n_acc_win = 0;
        }
        if (guard && !refresh) refresh = 3;
        // a guard refresh recomputes only the planes that tripped it (the others carry no
        // amplified error); a scheduled one recomputes every plane
        reinterpret_cast<unsigned long long*>(s.dctl)[dRefreshMask] = refresh == 3 ? guard : ~0ull;
        // the schedules (accept window, NRefresh) restart only at a refresh of every plane
        if (refresh == 1 || refresh == 2) since_refresh = 0;
        if (refresh == 3) ++n_guard;
        else if (refresh) ++n_sched;
        cc[cRefresh] = refresh;
      }
      __syncthreads();
      lap(kPhMetropolis);
      if (cc[cAccept]) {
        if (type == 0) {
          update_hop_dev<T, JPL>(m, s, msa, true);
        } else {
          update_exchange_dev<T, JPL>(m, s, msa, cc[cMsb], ri + sp * ns, rj + cc[cT] * ns, true);
        }
      }
      lap(kPhUpdate);
      if (cc[cRefresh]) {
        const unsigned long long rmask = reinterpret_cast<const unsigned long long*>(s.dctl)[dRefreshMask];
        const int info = calc_m_all_dev<T, JPL, kSmemPlanes, kSmemWs>(m, s, w.status, rmask);
        if (tid == 0 && info == 0) {
          // drift of the incrementally updated amplitude against the FP64 recomputation
          const double fresh = log_ip_of(m, s.pf, s.qpw);
          const double d = fabs(fresh - s.dctl[dLogIp]);
          if (isfinite(d) && d > drift_max) drift_max = d;
          s.dctl[dLogIp] = fresh;
        }
        __syncthreads();
        lap(kPhRefresh);
      }
    }
    if (out + S >= n_out) {
      make_proj_cnt_cta(m, s.jidx, s.num, s.cnt);
      const size_t sample = static_cast<size_t>(wk) * S + (out + S - n_out);
      for (int k = tid; k < n; k += blockDim.x) w.s_idx[sample * n + k] = s.idx[k];
      for (int k = tid; k < m.ns2; k += blockDim.x) {
        w.s_cfg[sample * m.ns2 + k] = s.cfg[k];
        w.s_num[sample * m.ns2 + k] = s.num[k];
      }
      for (int k = tid; k < m.nproj; k += blockDim.x) w.s_cnt[sample * m.nproj + k] = s.cnt[k];
      if constexpr (sizeof(T) == sizeof(double)) {
        // resident measurement: this sample's Pf and X⁻¹ as the walker holds them
        if (w.s_inv) {
          const size_t nn = static_cast<size_t>(n) * n;
          double* dst = w.s_inv + sample * m.nqp * nn;
          for (size_t k = tid; k < m.nqp * nn; k += blockDim.x) dst[k] = s.planes[k];
          for (int k = tid; k < m.nqp; k += blockDim.x) w.s_pf[sample * m.nqp + k] = s.pf[k];
        }
      }
    }
  }
  __syncthreads();
  make_proj_cnt_cta(m, s.jidx, s.num, s.cnt);
  // ---- store the walker (the final configuration is the burn-in state of the next step) ----
  for (int k = tid; k < kSfmtN32; k += blockDim.x) w.sfmt[static_cast<size_t>(wk) * kSfmtN32 + k] = s.sf[k];
  for (int k = tid; k < n; k += blockDim.x) w.ele_idx[static_cast<size_t>(wk) * n + k] = s.idx[k];
  for (int k = tid; k < m.ns2; k += blockDim.x) {
    w.ele_cfg[static_cast<size_t>(wk) * m.ns2 + k] = s.cfg[k];
    w.ele_num[static_cast<size_t>(wk) * m.ns2 + k] = s.num[k];
  }
  for (int k = tid; k < m.nproj; k += blockDim.x) w.proj_cnt[static_cast<size_t>(wk) * m.nproj + k] = s.cnt[k];
  for (int k = tid; k < m.nqp; k += blockDim.x) w.pf[static_cast<size_t>(wk) * m.nqp + k] = s.pf[k];
  if (tid == 0) {
    w.sfmt_idx[wk] = sf_idx;
    w.draws[wk] = sf_draws;
    w.burn[wk] = 1;
    for (int k = 0; k < 6; ++k) w.counter[static_cast<size_t>(wk) * 6 + k] = counter[k];
    if (w.drift) w.drift[wk] = drift_max;
    if (w.nrefresh) {
      w.nrefresh[2 * static_cast<size_t>(wk)] = n_sched;
      w.nrefresh[2 * static_cast<size_t>(wk) + 1] = n_guard;
    }
    if (timing) {
      ph[kPhTotal] = clock64() - t_begin;
      for (int k = 0; k < kPhCount; ++k) w.timers[static_cast<size_t>(wk) * kPhCount + k] = ph[k];
    }
  }
}

// ---- host launch ---------------------------------------------------------------------------
int smem_limit_bytes();

int walkers_per_sm();

template <typename T, int JPL, int NT, bool kSmemPlanes, bool kSmemWs>
int launch_sample_t(const DevModel& m, const DevWalkers& w, cudaStream_t stream) {
  size_t smem = samp_layout<T>(m, kSmemPlanes, kSmemWs).total;
  auto kernel = k_sample<T, JPL, NT, kSmemPlanes, kSmemWs>;
  if (!kSmemPlanes && walkers_per_sm() > 0) {
    // cap the walkers resident per SM (so that their L2 slices stay in L2) by the
    // shared-memory footprint of each CTA, within the per-block limit
    int dev = 0, per_sm = 0, reserved = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa{};
    MVMCB_CUDA(cudaFuncGetAttributes(&fa, kernel));
    const size_t cap = std::min(static_cast<size_t>(per_sm / walkers_per_sm() - reserved) - fa.sharedSizeBytes,
                                static_cast<size_t>(optin) - fa.sharedSizeBytes);
    smem = std::max(smem, cap);
  }
  MVMCB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  kernel<<<w.W, NT, smem, stream>>>(m, w);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

// Shared-memory residency: planes (and for FP32 the FP64 refresh workspace) in shared
// memory when they fit the per-block opt-in limit.
int residency_policy();
// FP32 planes: several small QP planes (side ≤ 64) go to L2 with two walkers per SM, which
// overlap each other's serial phases (2D 8×8, eight planes of 64: 2.08 against 2.63 s per
// SR step with one walker per SM holding its planes in shared memory); one wide plane stays
// in shared memory (2D 16×16: 68.7 against 84.2 ms in L2).
bool fp32_prefers_l2(const DevModel& m) { return residency_policy() == 0 && m.nqp >= 4 && m.n <= 64; }
bool sample_planes_in_smem(const DevModel& m, int precision, int limit) {
  if (residency_policy() == 1) return false;
  if (precision == 32 && fp32_prefers_l2(m)) return false;
  if (precision == 32) return samp_layout<float>(m, true, true).total <= static_cast<size_t>(limit) ||
                              samp_layout<float>(m, true, false).total <= static_cast<size_t>(limit);
  return samp_layout<double>(m, true, true).total <= static_cast<size_t>(limit);
}

// Plane residency: "shared" keeps a walker's planes in shared memory (one walker per SM
// when they are large), "global" keeps them in the walker's L2-resident slice so several
// walkers share an SM; "auto" (default) prefers shared memory. MVMC_B200_RESIDENCY selects.
int residency_policy() {
  static int policy = -1;
  if (policy < 0) {
    const char* v = std::getenv("MVMC_B200_RESIDENCY");
    policy = 0;
    if (v && std::strcmp(v, "global") == 0) policy = 1;
    if (v && std::strcmp(v, "shared") == 0) policy = 2;
  }
  return policy;
}

// Walkers resident per SM when planes are in L2 (MVMC_B200_WPS=k; 0 = as many as fit).
int walkers_per_sm() {
  static int k = -1;
  if (k < 0) {
    const char* v = std::getenv("MVMC_B200_WPS");
    k = v ? std::max(0, std::atoi(v)) : 0;
  }
  return k;
}

// CTA size for walkers whose planes are in L2 (MVMC_B200_THREADS=128|256|512; 0 = auto).
int global_threads() {
  static int nt = -1;
  if (nt < 0) {
    const char* v = std::getenv("MVMC_B200_THREADS");
    nt = (v && std::strcmp(v, "128") == 0) ? 128 : ((v && std::strcmp(v, "256") == 0) ? 256 : 0);
    if (v && std::strcmp(v, "512") == 0) nt = 512;
  }
  return nt;
}

// Auto CTA size: two 256-thread walkers per SM while their planes stay within ~3/4 of the
// L2, else one 512-thread walker per SM (2D 16×16, 401 KB per walker: 24.2k vs 23.5k
// sweeps/s; 2D 8×8 with 8 planes, 256 KB per walker: 2×256 is 1.6× faster).
template <typename T>
int auto_global_threads(const DevModel& m) {
  if (global_threads() != 0) return global_threads();
  int dev = 0, sms = 0, l2 = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev);
  const double planes = static_cast<double>(sizeof(T)) * m.nqp * m.n * m.n;
  return 2.0 * sms * planes > 0.75 * l2 ? 512 : 256;
}

// Planes in L2: the FP64 sweep buffers of the refresh go to shared memory when they fit
// beside the rest without lowering the walkers per SM that the registers allow.
template <typename T, int JPL>
int launch_sample_global(const DevModel& m, const DevWalkers& w, cudaStream_t stream) {
  const int nt = auto_global_threads<T>(m);
  if (nt == 128) return launch_sample_t<T, JPL, 128, false, false>(m, w, stream);
  if (nt == 512) return launch_sample_t<T, JPL, 512, false, false>(m, w, stream);
  int dev = 0, per_sm = 0, reserved = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
  const size_t budget = static_cast<size_t>(per_sm / SampOccupancy<256, false>::kBlocks - reserved);
  if (samp_layout<T>(m, false, true).total <= budget) return launch_sample_t<T, JPL, 256, false, true>(m, w, stream);
  return launch_sample_t<T, JPL, 256, false, false>(m, w, stream);
}

template <int JPL>
int launch_sample_jpl(const DevModel& m, const DevWalkers& w, int precision, int limit, cudaStream_t stream) {
  // Resident (shared-memory) planes run one walker per SM with 16 warps; planes in global
  // memory run several walkers per SM with 8 warps each.
  if (residency_policy() == 1) {
    if (precision == 32) return launch_sample_global<float, JPL>(m, w, stream);
    return launch_sample_global<double, JPL>(m, w, stream);
  }
  if (precision == 32 && fp32_prefers_l2(m)) return launch_sample_global<float, JPL>(m, w, stream);
  if (precision == 32) {
    if (samp_layout<float>(m, true, true).total <= static_cast<size_t>(limit)) {
      if constexpr (JPL == 1) {
        // small planes: 128 threads per walker, as for FP64 below
        const char* e = std::getenv("MVMC_B200_SMEM_THREADS");
        if (!e || std::atoi(e) == 128) return launch_sample_t<float, JPL, 128, true, true>(m, w, stream);
      }
      return launch_sample_t<float, JPL, 512, true, true>(m, w, stream);
    }
    if (samp_layout<float>(m, true, false).total <= static_cast<size_t>(limit))
      return launch_sample_t<float, JPL, 512, true, false>(m, w, stream);
    return launch_sample_global<float, JPL>(m, w, stream);
  }
  if (samp_layout<double>(m, true, true).total <= static_cast<size_t>(limit)) {
    if constexpr (JPL == 1) {
      // small planes (n ≤ 32): 128 threads per walker (1D L16: 1.95M vs 1.33M sweeps/s
      // with 512, whose barriers cost more than the work they split); MVMC_B200_SMEM_THREADS
      // = 64|128|256|512 overrides
      const char* e = std::getenv("MVMC_B200_SMEM_THREADS");
      const int nt = e ? std::atoi(e) : 128;
      if (nt == 64) return launch_sample_t<double, JPL, 64, true, true>(m, w, stream);
      if (nt == 128) return launch_sample_t<double, JPL, 128, true, true>(m, w, stream);
      if (nt == 256) return launch_sample_t<double, JPL, 256, true, true>(m, w, stream);
    }
    return launch_sample_t<double, JPL, 512, true, true>(m, w, stream);
  }
  return launch_sample_global<double, JPL>(m, w, stream);
}

int launch_sample(const DevModel& m, const DevWalkers& w, int precision, cudaStream_t stream) {
  int dev = 0, limit = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&limit, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const int n = m.n;
  if (n <= 32) return launch_sample_jpl<1>(m, w, precision, limit, stream);
  if (n <= 64) return launch_sample_jpl<2>(m, w, precision, limit, stream);
  if (n <= 128) return launch_sample_jpl<4>(m, w, precision, limit, stream);
  if (n <= 224) return launch_sample_jpl<7>(m, w, precision, limit, stream);
  if (n <= 256) return launch_sample_jpl<8>(m, w, precision, limit, stream);
  return kErrArgument;
}

// ---- one walker's Pfaffian stage (RealPfStage, sampling/stage.rs:56-129) -----------------
// The five stage operations as single-CTA launches on FP64 planes held in global memory, for
// host-driven (teacher-forced) replay: the host owns the chain and passes the candidate
// configuration with every call; the device owns Pf and the inverses.
template <int JPL>
__global__ void __launch_bounds__(kStageThreads)
    k_stage(DevModel m, StageBufs b, int op, int msa, int msb, int rsa_old, int rsb_old, unsigned* status) {
  extern __shared__ __align__(16) unsigned char smem[];
  const SampLayout L = samp_layout<double>(m, false, false);
  WalkerSmem<double> s{};
  s.idx = reinterpret_cast<int*>(smem + L.idx);
  s.pf = reinterpret_cast<double*>(smem + L.pf);
  s.pfn = reinterpret_cast<double*>(smem + L.pfn);
  s.qpw = reinterpret_cast<double*>(smem + L.qpw);
  s.jidx = m.jast_idx;
  s.vec = reinterpret_cast<double*>(smem + L.vec);
  s.pscal = reinterpret_cast<double*>(smem + L.vec + sizeof(double) * 4 * static_cast<size_t>(m.nqp) * m.n);
  s.gj = gj_carve<double>(smem + L.gj, m.n);
  const size_t nn = static_cast<size_t>(m.n) * m.n;
  s.ws = b.ws;
  s.ws2 = b.ws + nn;
  s.planes = b.planes;
  const int tid = threadIdx.x;
  for (int k = tid; k < m.n; k += blockDim.x) s.idx[k] = b.idx[k];
  for (int k = tid; k < m.nqp; k += blockDim.x) {
    s.pf[k] = b.pf[k];
    s.pfn[k] = b.pfn[k];
    s.qpw[k] = m.qpw[k];
  }
  __syncthreads();
  if (op == kStageRecompute) {
    const int info = calc_m_all_dev<double, JPL, false, false>(m, s, status);
    if (tid == 0) b.info[0] = info;
  } else if (op == kStageProposeHop) {
    ratio_hop_dev<double>(m, s, msa);
  } else if (op == kStageAcceptHop) {
    update_hop_dev<double, JPL>(m, s, msa, false);
  } else if (op == kStageProposeExchange) {
    ratio_exchange_dev<double, JPL>(m, s, msa, msb);
  } else if (op == kStageAcceptExchange) {
    update_exchange_dev<double, JPL>(m, s, msa, msb, rsa_old, rsb_old, false);
  }
  __syncthreads();
  for (int k = tid; k < m.nqp; k += blockDim.x) {
    b.pf[k] = s.pf[k];
    b.pfn[k] = s.pfn[k];
  }
}

template <int JPL>
int launch_stage_jpl(const DevModel& m, const StageBufs& b, int op, int msa, int msb, int rsa_old, int rsb_old,
                     unsigned* status, cudaStream_t stream) {
  const size_t smem = samp_layout<double>(m, false, false).total;
  auto kernel = k_stage<JPL>;
  MVMCB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  kernel<<<1, kStageThreads, smem, stream>>>(m, b, op, msa, msb, rsa_old, rsb_old, status);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

int launch_stage(const DevModel& m, const StageBufs& b, int op, int msa, int msb, int rsa_old, int rsb_old,
                 unsigned* status, cudaStream_t stream) {
  const int n = m.n;
  if (n <= 32) return launch_stage_jpl<1>(m, b, op, msa, msb, rsa_old, rsb_old, status, stream);
  if (n <= 64) return launch_stage_jpl<2>(m, b, op, msa, msb, rsa_old, rsb_old, status, stream);
  if (n <= 128) return launch_stage_jpl<4>(m, b, op, msa, msb, rsa_old, rsb_old, status, stream);
  if (n <= 224) return launch_stage_jpl<7>(m, b, op, msa, msb, rsa_old, rsb_old, status, stream);
  if (n <= 256) return launch_stage_jpl<8>(m, b, op, msa, msb, rsa_old, rsb_old, status, stream);
  return kErrArgument;
}

}  // namespace mvmcb
