// K3 + K4: local measurement of saved samples and the SR operand reduction.
//
// One CTA per saved sample (accumulate_observables_local, crates/mvmc-core/src/run.rs:
// 2937-3614 of AtelierArith/mvmc-rs):
//   * CalculateMAll per QP plane (pfaffian.rs:871-927) by the Gauss–Jordan sweep;
//   * IP = Σ_q w_q Pf_q (observables.rs:128) and the skip rules (run.rs:3077,3241,3305);
//   * local energy: CoulombIntra / CoulombInter / Hund diagonal (observables.rs:483) and
//     every Transfer term through the one-electron Pfaffian ratio with the direct
//     projection ratio of the moved configuration (calh1_real_fast, observables.rs:1680);
//   * O = [1, projection counts, ∂lnΨ/∂f_k] (set_projection_diff observables.rs:202 and the
//     adjoint Slater derivative slater_derivative.rs:289-550), written as one row of the
//     SR sample matrix (calculate_oo_store_real, observables.rs:297).
// In the PhysCal form (NVMCCalMode 1) the O row is skipped and the Green functions of
// the sample are evaluated on the same inverse planes instead (ordinary_green_values,
// crates/mvmc-core/src/observables/green_measurements.rs:264-320): one-body terms by the
// one-electron ratio (green_func1, observables.rs:1895-2050), TwoBodyG terms by their
// index-coincidence reductions or the two-hop ratio (green_func2, observables.rs:664-860;
// two_ratio_real, sampling/updates.rs:1539-1567).
// The reductions sum per walker in sample order and then across walkers in walker
// order (the rank-order fold of ThreadReducer, multichain.rs:433), and the Slater
// derivative is gathered per orbital in a fixed order, so reruns are bitwise repeatable
// (a model whose translations are not permutations falls back to an atomic scatter).
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstdlib>
#include <cstring>

#include "common.cuh"
#include "engine.cuh"
#include "pfinv.cuh"

namespace mvmcb {

constexpr int kMeasThreads = 256;
// dense one-body product: destination rows per tile (warps × rows per thread)
constexpr int kGreenRows = 4;
constexpr int kGreenTile = (kMeasThreads / 32) * kGreenRows;

struct MeasLayout {
  size_t idx, cfg, num, cnt, tr, sg, pf, tacc, g1, oacc, cj, gscr, gacc, gempty, gtile, snap, gj, plane, total;
};

__host__ __device__ inline size_t a16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline MeasLayout meas_layout(const DevModel& m, bool smem_plane, bool green = false) {
  MeasLayout L;
  size_t o = 0;
  L.idx = o; o = a16(o + sizeof(int) * m.n);
  L.cfg = o; o = a16(o + sizeof(int) * m.ns2);
  L.num = o; o = a16(o + sizeof(int) * m.ns2);
  L.cnt = o; o = a16(o + sizeof(int) * (m.nproj + 1));
  L.tr = o; o = a16(o + sizeof(int) * m.n);
  L.sg = o; o = a16(o + sizeof(int) * m.n);
  L.pf = o; o = a16(o + sizeof(double) * (m.nqp + 2));
  L.tacc = o; o = a16(o + sizeof(double) * (m.nterm + 1));
  L.g1 = o; o = a16(o + sizeof(double) * (m.nterm + 1));
  L.oacc = o; o = a16(o + sizeof(double) * (m.norb + 1));
  L.cj = o; o = a16(o + sizeof(double) * m.ns);
  // two-hop scratch: the gathered Slater rows u, v of one term per warp
  L.gscr = o;
  if (green && m.nggen > 0) o = a16(o + sizeof(double) * 2 * (kMeasThreads / 32) * static_cast<size_t>(m.n));
  // one-body plane sums (when they fit beside the planes)
  L.gacc = o;
  if (green && m.gacc_smem) o = a16(o + sizeof(double) * static_cast<size_t>(m.ngone));
  // dense one-body product: the empty sites of each spin and one tile of gathered rows
  L.gempty = o;
  if (green && m.gdense) o = a16(o + sizeof(int) * 2 * static_cast<size_t>(m.ns));
  L.gtile = o;
  if (green && m.gdense) o = a16(o + sizeof(double) * kGreenTile * static_cast<size_t>(m.n));
  // rows p and q of the in-place sweep of a plane in global memory
  L.snap = o;
  if (!smem_plane) o = a16(o + 2 * sizeof(double) * static_cast<size_t>(m.n));
  L.gj = o;
  L.plane = o;
  // the plane and its ping-pong partner
  if (smem_plane) o = a16(o + 2 * sizeof(double) * static_cast<size_t>(m.n) * m.n);
  L.total = o;
  return L;
}

// Σ_k α_k Δc_k of moving one electron from site `src` to site `dst` (update_proj_cnt,
// sampling/projection.rs:278, with log_proj_ratio :403), where occ(slot) is the occupation
// of the 2Ns spin-site slots after the move: Gutzwiller −α(src)·n_src + α(dst)·n↑n↓(dst),
// Jastrow α(src,dst)·(n_src − n_dst + 1) + Σ_{k≠src,dst} (α(dst,k) − α(src,k))·(n_k − 1).
template <class Occ>
__device__ double hop_log_proj(const DevModel& m, int src, int dst, Occ occ) {
  const int ns = m.ns;
  const int n_src = occ(src) + occ(src + ns), n_dst = occ(dst) + occ(dst + ns);
  double z = -m.gutz_site[src] * static_cast<double>(n_src);
  z += m.gutz_site[dst] * static_cast<double>(occ(dst) * occ(dst + ns));
  z += m.jast_pair[src * ns + dst] * static_cast<double>(n_src - n_dst + 1);
  for (int k = 0; k < ns; ++k) {
    if (k == src || k == dst) continue;
    z += (m.jast_pair[dst * ns + k] - m.jast_pair[src * ns + k]) * static_cast<double>(occ(k) + occ(k + ns) - 1);
  }
  return z;
}

// Σ_k α_k Δc_k of the hop src → dst (spin-site slots src_slot, dst_slot) from the
// charges before the move and cj[r] = Σ_site J(r, site)·(n_site − 1): the O(1) form of
// calh1_direct_projection_ratio_moved (observables.rs:1680-1758).
__device__ inline double direct_hop_log_proj(const DevModel& m, const int* num, const double* cj, int source,
                                             int dest, int src_slot, int dst_slot) {
  const int ns = m.ns;
  auto occ = [&](int slot) { return slot == src_slot ? 0 : (slot == dst_slot ? 1 : num[slot]); };
  auto chm = [&](int site) { return occ(site) + occ(ns + site) - 1; };
  auto ch = [&](int site) { return num[site] + num[ns + site] - 1; };
  double z = 0.0;
  z -= m.gutz_site[source] * static_cast<double>(occ(source) + occ(ns + source));
  z += m.gutz_site[dest] * static_cast<double>(occ(dest) * occ(ns + dest));
  const double jsd = m.jast_pair[source * ns + dest];
  z += jsd * static_cast<double>(chm(source) - chm(dest) + 1);
  const double sum_dest = cj[dest] - m.jast_pair[dest * ns + source] * static_cast<double>(ch(source));
  const double sum_src = cj[source] - m.jast_pair[source * ns + dest] * static_cast<double>(ch(dest));
  return z + (sum_dest - sum_src);
}

// Julia's complex quotient (pfapack julia_complex.rs:9-75) for a real numerator a and a
// real denominator c: a·(1/c), rescaled by powers of two when |a| or |c| is extreme.
__device__ inline double julia_real_quotient(double a, double c) {
  const double halfov = 0.5 * DBL_MAX, twouneps = DBL_MIN * 2.0 / DBL_EPSILON;
  const double ab = fabs(a), cd = fabs(c);
  if (isinf(c)) return 0.0 * (a == 0.0 ? a : copysign(1.0, a)) * copysign(1.0, c);
  double s = 1.0;
  if (ab >= halfov || ab <= twouneps || cd >= halfov || cd <= twouneps) {
    const double bs = 2.0 / (DBL_EPSILON * DBL_EPSILON);
    if (ab >= halfov) { a *= 0.5; s *= 2.0; }
    else if (ab <= twouneps) { a *= bs; s /= bs; }
    if (cd >= halfov) { c *= 0.5; s *= 0.5; }
    else if (cd <= twouneps) { c *= bs; s *= bs; }
  }
  const double t = 1.0 / c;
  return a * t * s;
}

// Dense one-body product on one plane: for every spin s, every empty site r of spin s and
// every electron m of spin s, R = Σ_k F(r, r_k)·X⁻¹[m][k] with r_k the electron sites, read
// as −Σ_k F(r, r_k)·X⁻¹[k][m] (X⁻¹ is skew) so that lanes take consecutive m; the moved
// electron's own term is corrected to F(r, r)·X⁻¹[m][m] (calculate_new_pf_m2_real_flat with
// the configuration after the hop). Pf' = −Pf·R is added to the one-body term (r s j s), j
// the site of m. Rows are tiled kGreenTile at a time through shared memory.
__device__ void green_dense_plane(const DevModel& m, int q, double wq, double pfv, const double* A, const int* idx,
                                  const int* gempty, double* gtile, double* gacc) {
  const int n = m.n, ns = m.ns, ne = m.ne, ns2 = m.ns2, tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int ce = ns - ne;  // empty sites per spin
  const double* slq = m.slater + static_cast<size_t>(q) * ns2 * ns2;
  for (int s = 0; s < 2; ++s) {
    const int* empty = gempty + s * ns;
    for (int r0 = 0; r0 < ce; r0 += kGreenTile) {
      const int rows = min(kGreenTile, ce - r0);
      for (int k = tid; k < rows * n; k += nt) {
        const int rr = k / n, c = k - rr * n;
        const int rs = empty[r0 + rr] + s * ns;
        gtile[k] = __ldg(slq + static_cast<size_t>(rs) * ns2 + idx[c] + (c >= ne ? ns : 0));
      }
      __syncthreads();
      for (int e0 = 0; e0 < ne; e0 += 32) {
        const int e = e0 + lane;
        const int mcol = s * ne + min(e, ne - 1);
        double acc[kGreenRows];
#pragma unroll
        for (int i = 0; i < kGreenRows; ++i) acc[i] = 0.0;
        const double* g0 = gtile + static_cast<size_t>(warp * kGreenRows) * n;
        for (int k = 0; k < n; ++k) {
          const double a = A[static_cast<size_t>(k) * n + mcol];
#pragma unroll
          for (int i = 0; i < kGreenRows; ++i) acc[i] += g0[i * n + k] * a;
        }
        if (e < ne) {
          const int msj = s * ne + e;
          const int site_j = idx[msj];
          const double amm = A[static_cast<size_t>(msj) * n + msj];
#pragma unroll
          for (int i = 0; i < kGreenRows; ++i) {
            const int rr = warp * kGreenRows + i;
            if (rr >= rows) continue;
            const int site_i = empty[r0 + rr];
            const int t = m.gterm_of[(s * ns + site_i) * ns + site_j];
            if (t < 0) continue;
            const int rs = site_i + s * ns;
            // R over rows m: −acc; the moved electron's slot holds F(r, r) instead of F(r, r_m)
            const double r = -acc[i] + amm * (__ldg(slq + static_cast<size_t>(rs) * ns2 + rs) -
                                              __ldg(slq + static_cast<size_t>(rs) * ns2 + site_j + s * ns));
            gacc[t] += wq * (-r * pfv);
          }
        }
      }
      __syncthreads();
    }
  }
}

// Per-plane Green contributions of one sample: Σ_q w_q·Pf'_q of every one-body hop and of
// every two-hop term, added into the sample's row (plane order).
template <int JPL>
__device__ void green_plane(const DevModel& m, int q, double wq, double pfv, const double* A, const int* idx,
                            const int* cfg, const int* num, double* gacc, double* grow, double* gscr) {
  const int n = m.n, ns = m.ns, ne = m.ne, lane = threadIdx.x & 31, warp = threadIdx.x >> 5,
            nwarp = blockDim.x >> 5;
  // one-body: the electron at rj (spin t) moves to the empty ri: Pf' = −Pf·Σ_k X⁻¹[msj][k]·F(ri, r'_k).
  // Each warp tests 32 terms at once (one per lane) and runs the allowed ones in turn.
  for (int base = warp * 32; base < (m.gdense ? 0 : m.ngone); base += nwarp * 32) {
    const int k = base + lane;
    bool allowed = false;
    int gi = 0, gt = 0, msj = 0;
    if (k < m.ngone) {
      const int4 term = __ldg(reinterpret_cast<const int4*>(m.gone) + k);
      gi = term.x;
      const int gs = term.y, gj = term.z;
      gt = term.w;
      const int dst = gi + gs * ns, src = gj + gt * ns;
      allowed = gs == gt && gi != gj && num[dst] == 0 && num[src] == 1 && cfg[src] >= 0;
      if (allowed) msj = cfg[src] + gt * ne;
    }
    unsigned todo = __ballot_sync(0xffffffffu, allowed);
    while (todo) {
      const int j = __ffs(todo) - 1;
      todo &= todo - 1;
      const int ti = __shfl_sync(0xffffffffu, gi, j), tt = __shfl_sync(0xffffffffu, gt, j);
      const int tm = __shfl_sync(0xffffffffu, msj, j);
      const double* row = A + static_cast<size_t>(tm) * n;
      const double* srow = m.slater + (static_cast<size_t>(q) * m.ns2 + (ti + tt * ns)) * m.ns2;
      double r = 0.0;
      for (int c = lane; c < n; c += 32) {
        const int rc = (c == tm ? ti : idx[c]) + (c >= ne ? ns : 0);
        r += row[c] * __ldg(srow + rc);
      }
      r = warp_sum(r);
      if (lane == j) gacc[k] += wq * (-r * pfv);
    }
  }
  // two-hop: electron msa moves rl → rk (spin u), then msb moves rj → ri (spin s);
  // ratio = X_ab·v_a + X_ab·(vᵀ X u) + p_a q_b − p_b q_a with u, v the moved rows
  double* gu = gscr + static_cast<size_t>(warp) * 2 * n;
  double* gv = gu + n;
  for (int g = warp; g < m.nggen; g += nwarp) {
    const int* t = m.ggen + 6 * g;
    const int ri = t[0], rj = t[1], rk = t[2], rl = t[3], s = t[4], u = t[5];
    if (num[ri + s * ns] != 0 || num[rj + s * ns] != 1 || num[rk + u * ns] != 0 || num[rl + u * ns] != 1) continue;
    const int mj = cfg[rj + s * ns], mi = cfg[rl + u * ns];
    if (mj < 0 || mi < 0) continue;
    const int msa = mi + u * ne, msb = mj + s * ne;
    const double* sa = m.slater + (static_cast<size_t>(q) * m.ns2 + (rk + u * ns)) * m.ns2;
    const double* sb = m.slater + (static_cast<size_t>(q) * m.ns2 + (ri + s * ns)) * m.ns2;
    const double* xa = A + static_cast<size_t>(msa) * n;
    const double* xb = A + static_cast<size_t>(msb) * n;
    double pa = 0.0, pb = 0.0, qa = 0.0, qb = 0.0;
    for (int c = lane; c < n; c += 32) {
      const int rc = (c == msa ? rk : (c == msb ? ri : idx[c])) + (c >= ne ? ns : 0);
      const double va = __ldg(sa + rc), vb = __ldg(sb + rc);
      gu[c] = va;
      gv[c] = vb;
      pa += xa[c] * va;
      pb += xb[c] * va;
      qa += xa[c] * vb;
      qb += xb[c] * vb;
    }
    __syncwarp();
    // vᵀ X u: column sums w_c = Σ_i v_i X[i][c] (lanes on consecutive columns), then Σ_c w_c u_c
    double bma = 0.0;
    for (int c = lane; c < n; c += 32) {
      double w = 0.0;
      for (int i = 0; i < n; ++i) w += gv[i] * A[static_cast<size_t>(i) * n + c];
      bma += w * gu[c];
    }
    pa = warp_sum(pa);
    pb = warp_sum(pb);
    qa = warp_sum(qa);
    qb = warp_sum(qb);
    bma = warp_sum(bma);
    if (lane == 0) {
      const double xab = xa[msb], vba = gv[msa];
      const double ratio = xab * vba + xab * bma + pa * qb - pb * qa;
      grow[m.ngone + m.ngtwo + g] += wq * (ratio * pfv);
    }
    __syncwarp();
  }
}

// Final Green values of one sample from the plane sums (run after the energy, all threads).
__device__ void green_finish(const DevModel& m, double ip, bool ok, const int* cfg, const int* num, const double* cj,
                             const double* gacc, double* grow) {
  const int ns = m.ns, tid = threadIdx.x, nt = blockDim.x;
  for (int k = tid; k < m.ngone; k += nt) {
    const int4 term = __ldg(reinterpret_cast<const int4*>(m.gone) + k);
    const int gi = term.x, gs = term.y, gj = term.z, gt = term.w;
    const int dst = gi + gs * ns, src = gj + gt * ns;
    double v;
    if (ip == 0.0) v = 0.0;
    else if (gs == gt && gi == gj) v = static_cast<double>(num[src]);
    else if (gs != gt || num[dst] == 1 || num[src] == 0 || cfg[src] < 0) v = 0.0;
    else {
      const double a = gacc[m.gdense ? m.gfirst[k] : k];
      v = julia_real_quotient(exp(direct_hop_log_proj(m, num, cj, gj, gi, src, dst)) * a, ip);
    }
    grow[k] = ok ? v : 0.0;
  }
  for (int g = tid; g < m.nggen; g += nt) {
    const int* t = m.ggen + 6 * g;
    const int ri = t[0], rj = t[1], rk = t[2], rl = t[3], s = t[4], u = t[5];
    double v = 0.0;
    if (ip != 0.0 && num[ri + s * ns] == 0 && num[rj + s * ns] == 1 && num[rk + u * ns] == 0 &&
        num[rl + u * ns] == 1 && cfg[rj + s * ns] >= 0 && cfg[rl + u * ns] >= 0) {
      const int a0 = rl + u * ns, a1 = rk + u * ns, b0 = rj + s * ns, b1 = ri + s * ns;
      auto mid = [&](int slot) { return slot == a0 ? 0 : (slot == a1 ? 1 : num[slot]); };
      auto fin = [&](int slot) { return slot == b0 ? 0 : (slot == b1 ? 1 : mid(slot)); };
      const double z = hop_log_proj(m, rl, rk, mid) + hop_log_proj(m, rj, ri, fin);
      v = julia_real_quotient(exp(z) * grow[m.ngone + m.ngtwo + g], ip);
    }
    grow[m.ngone + m.ngtwo + g] = ok ? v : 0.0;
  }
  __syncthreads();
  const double* one = grow;
  const double* gen = grow + m.ngone + m.ngtwo;
  for (int k = tid; k < m.ngtwo; k += nt) {
    const int4 t0 = __ldg(reinterpret_cast<const int4*>(m.gtwo) + 2 * k);
    const int4 t1 = __ldg(reinterpret_cast<const int4*>(m.gtwo) + 2 * k + 1);
    const int ri = t0.x, rj = t0.y, rk = t0.z, rl = t0.w, s = t1.x, u = t1.y, ref = t1.z, gi = t1.w;
    const int rsi = ri + s * ns, rsj = rj + s * ns, rtk = rk + u * ns;
    double v;
    if (s == u) {
      if (rk == rl) v = num[rtk] == 0 ? 0.0 : one[ref];
      else if (rj == rl) v = 0.0;
      else if (ri == rl) v = num[rsi] == 0 ? 0.0 : (rj == rk ? static_cast<double>(1 - num[rsj]) : -one[ref]);
      else if (rj == rk) v = num[rsj] == 1 ? 0.0 : one[ref];
      else if (ri == rk) v = 0.0;
      else if (ri == rj) v = num[rsi] == 0 ? 0.0 : one[ref];
      else v = gen[gi];
    } else if (rk == rl) {
      v = num[rtk] == 0 ? 0.0 : (ri == rj ? static_cast<double>(num[rsi]) : one[ref]);
    } else if (ri == rj) {
      v = num[rsi] == 0 ? 0.0 : one[ref];
    } else {
      v = gen[gi];
    }
    grow[m.ngone + k] = ok ? v : 0.0;
  }
  __syncthreads();
}

template <int JPL, bool kSmemPlane, bool kGreen, int NT = kMeasThreads>
__global__ void __launch_bounds__(NT, (kSmemPlane || NT > kMeasThreads ? 1 : 2))
    k_measure(DevModel m, const int* __restrict__ s_idx, const int* __restrict__ s_cfg,
              const int* __restrict__ s_num, const int* __restrict__ s_cnt, int nsamples,
              double* __restrict__ gws, double* __restrict__ ostore, double* __restrict__ eloc,
              double* __restrict__ lpsi, int* __restrict__ valid, double* __restrict__ gval, unsigned* status) {
  extern __shared__ __align__(16) unsigned char smem[];
  const MeasLayout L = meas_layout(m, kSmemPlane, kGreen);
  int* idx = reinterpret_cast<int*>(smem + L.idx);
  int* cfg = reinterpret_cast<int*>(smem + L.cfg);
  int* num = reinterpret_cast<int*>(smem + L.num);
  int* cnt = reinterpret_cast<int*>(smem + L.cnt);
  int* tr = reinterpret_cast<int*>(smem + L.tr);
  int* sg = reinterpret_cast<int*>(smem + L.sg);
  double* pf = reinterpret_cast<double*>(smem + L.pf);
  double* tacc = reinterpret_cast<double*>(smem + L.tacc);
  double* g1 = reinterpret_cast<double*>(smem + L.g1);
  double* oacc = reinterpret_cast<double*>(smem + L.oacc);
  double* cj = reinterpret_cast<double*>(smem + L.cj);
  double* gscr = reinterpret_cast<double*>(smem + L.gscr);
  const int n = m.n, ns = m.ns, ne = m.ne, tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  const size_t nn = static_cast<size_t>(n) * n;
  double* A = kSmemPlane ? reinterpret_cast<double*>(smem + L.plane) : gws + static_cast<size_t>(blockIdx.x) * 2 * nn;
  double* Bpp = A + nn;
  __shared__ int s_bad;

  for (int sample = blockIdx.x; sample < nsamples; sample += gridDim.x) {
    for (int k = tid; k < n; k += nt) idx[k] = s_idx[static_cast<size_t>(sample) * n + k];
    for (int k = tid; k < m.ns2; k += nt) {
      cfg[k] = s_cfg[static_cast<size_t>(sample) * m.ns2 + k];
      num[k] = s_num[static_cast<size_t>(sample) * m.ns2 + k];
    }
    for (int k = tid; k < m.nproj; k += nt) cnt[k] = s_cnt[static_cast<size_t>(sample) * m.nproj + k];
    for (int k = tid; k < m.nterm; k += nt) tacc[k] = 0.0;
    for (int k = tid; k < m.norb; k += nt) oacc[k] = 0.0;
    double* grow = kGreen ? gval + static_cast<size_t>(sample) * m.gw : nullptr;
    double* gacc = kGreen && m.gacc_smem ? reinterpret_cast<double*>(smem + L.gacc) : grow;
    int* gempty = reinterpret_cast<int*>(smem + L.gempty);
    double* gtile = reinterpret_cast<double*>(smem + L.gtile);
    if (kGreen) {
      for (int k = tid; k < m.gw; k += nt) grow[k] = 0.0;
      if (m.gacc_smem)
        for (int k = tid; k < m.ngone; k += nt) gacc[k] = 0.0;
    }
    if (tid == 0) s_bad = 0;
    __syncthreads();
    // direct projection helper: cj[r] = Σ_site J[r][site]·(n_site − 1)
    for (int r = tid; r < ns; r += nt) {
      double acc = 0.0;
      for (int site = 0; site < ns; ++site)
        acc += __ldg(m.jast_pair + r * ns + site) * static_cast<double>(num[site] + num[site + ns] - 1);
      cj[r] = acc;
    }
    if (kGreen && m.gdense && warp < 2) {
      // empty sites of spin `warp`, in site order (ballot prefix over 32 sites at a time)
      int count = 0;
      for (int b = 0; b < ns; b += 32) {
        const int site = b + lane;
        const bool e = site < ns && s_num[static_cast<size_t>(sample) * m.ns2 + site + warp * ns] == 0;
        const unsigned mask = __ballot_sync(0xffffffffu, e);
        if (e) gempty[warp * ns + count + __popc(mask & ((1u << lane) - 1u))] = site;
        count += __popc(mask);
      }
    }
    if (tid == 0) {
      bool all_zero = true, all_neg = true;
      for (int k = 0; k < n; ++k) {
        all_zero = all_zero && idx[k] == 0;
        all_neg = all_neg && idx[k] < 0;
      }
      if (all_zero || all_neg) s_bad = 1;
    }
    __syncthreads();
    if (s_bad) {
      if (tid == 0) {
        valid[sample] = 0;
        eloc[sample] = 0.0;
        lpsi[sample] = 0.0;
      }
      if (!kGreen)
        for (int k = tid; k < m.sr_size; k += nt) ostore[static_cast<size_t>(sample) * m.sr_size + k] = 0.0;
      __syncthreads();
      continue;
    }
    for (int q = 0; q < m.nqp; ++q) {
      double pfv;
      int st;
      if (m.rinv) {
        // resident measurement: the sampler's Pf and X⁻¹ of this sample
        const double* src = m.rinv + (static_cast<size_t>(sample) * m.nqp + q) * n * n;
        for (int k = tid; k < n * n; k += nt) A[k] = src[k];
        pfv = m.rpf[static_cast<size_t>(sample) * m.nqp + q];
        st = 0;
        __syncthreads();
      } else {
        for (int k = tid; k < n * n; k += nt) {
          const int i = k / n, j = k - i * n;
          const int ri = idx[i] + (i >= ne ? ns : 0), rj = idx[j] + (j >= ne ? ns : 0);
          A[k] = __ldg(m.slater + (static_cast<size_t>(q) * m.ns2 + ri) * m.ns2 + rj);
        }
        __syncthreads();
        // planes in L2: a few rows in flight per warp, fewer for wide rows so that two
        // samples share an SM
        if (kSmemPlane)
          gj_pfinv_pp<double, JPL, 1>(A, Bpp, n, pfv, st);
        else  // in place: one plane per sample block in L2, rows p and q snapshot in shared memory
          gj_pfinv_ip<double, JPL, (JPL <= 2 ? 4 : (JPL <= 4 ? 2 : 1))>(A, reinterpret_cast<double*>(smem + L.snap),
                                                                         n, pfv, st);
      }
      if (st != 0) {
        if (tid == 0) s_bad = 1;
        __syncthreads();
        break;
      }
      if (tid == 0) pf[q] = pfv;
      const double wq = m.qpw[q];
      // transfer terms: one-electron ratio on this plane (warp per term)
      for (int t = warp; t < m.nterm; t += nwarp) {
        const int ti = m.tterm[4 * t], tsi = m.tterm[4 * t + 1], tj = m.tterm[4 * t + 2], tsj = m.tterm[4 * t + 3];
        const int dst = ti + tsi * ns, src = tj + tsj * ns;
        if (tsi != tsj || (ti == tj) || num[dst] == 1 || num[src] == 0 || cfg[src] < 0) continue;
        const int msj = cfg[src] + tsj * ne;
        const int rsa = ti + tsj * ns;
        const double* row = A + static_cast<size_t>(msj) * n;
        double r = 0.0;
        for (int k = lane; k < n; k += 32) {
          const int rk = (k == msj ? ti : idx[k]) + (k >= ne ? ns : 0);
          r += row[k] * __ldg(m.slater + (static_cast<size_t>(q) * m.ns2 + rsa) * m.ns2 + rk);
        }
        r = warp_sum(r);
        if (lane == 0) tacc[t] += wq * (-r * pfv);
      }
      if (kGreen) {
        if (m.gdense) green_dense_plane(m, q, wq, pfv, A, idx, gempty, gtile, gacc);
        green_plane<JPL>(m, q, wq, pfv, A, idx, cfg, num, gacc, grow, gscr);
        __syncthreads();
        continue;  // PhysCal: no O row
      }
      // adjoint Slater derivative: translated sites of the electrons for this plane
      const int trans = q / m.nleg, spidx = q % m.nleg;
      const int mpidx = trans % m.nmp;
      for (int k = tid; k < n; k += nt) {
        tr[k] = m.trans[mpidx * ns + idx[k]];
        sg[k] = m.trans_sgn[mpidx * ns + idx[k]];
      }
      __syncthreads();
      const double cs = pfv * m.spgl[spidx], cc = pfv * m.spgl[m.nleg + spidx], ss = pfv * m.spgl[2 * m.nleg + spidx];
      if (m.orb_off && m.trans_inv) {
        // by orbital: thread k adds the electron pairs on orbital k's translated site pairs in
        // a fixed order, so the O row is bitwise repeatable (no atomics)
        const int* tinv = m.trans_inv + mpidx * ns;
        const int* tsgn = m.trans_sgn + mpidx * ns;
        const double fac[4] = {cs, -cc, ss, -cs};  // (up, up), (up, dn), (dn, up), (dn, dn)
        for (int k = tid; k < m.norb; k += nt) {
          double acc = 0.0;
          const int e1 = __ldg(m.orb_off + k + 1);
          for (int e = __ldg(m.orb_off + k); e < e1; ++e) {
            const int ent = __ldg(m.orb_ent + e);
            const int a = __ldg(tinv + (ent >> 16)), b = __ldg(tinv + ((ent >> 1) & 0x7fff));
            const int sgn = (ent & 1 ? -1 : 1) * __ldg(tsgn + a) * __ldg(tsgn + b);
#pragma unroll
            for (int sa = 0; sa < 2; ++sa) {
              const int ei = cfg[a + sa * ns];
              if (ei < 0) continue;
#pragma unroll
              for (int sb = 0; sb < 2; ++sb) {
                const int ej = cfg[b + sb * ns];
                if (ej < 0) continue;
                acc += (fac[2 * sa + sb] * A[static_cast<size_t>(ei + sa * ne) * n + ej + sb * ne]) *
                       static_cast<double>(sgn);
              }
            }
          }
          oacc[k] += wq * acc;
        }
      } else {
        for (int k = tid; k < n * n; k += nt) {
          const int i = k / n, j = k - i * n;
          const int orb = __ldg(m.orb_idx + tr[i] * ns + tr[j]);
          if (orb < 0 || orb >= m.norb) continue;
          const int sign = sg[i] * sg[j] * __ldg(m.orb_sgn + tr[i] * ns + tr[j]);
          const double first = i < ne ? cs : ss, second = i < ne ? cc : cs;
          const double v = A[k];
          const double value = j < ne ? v * first : -v * second;
          atomicAdd(oacc + orb, wq * (value * static_cast<double>(sign)));
        }
      }
      __syncthreads();
    }
    if (s_bad) {
      if (tid == 0) {
        valid[sample] = 0;
        eloc[sample] = 0.0;
        lpsi[sample] = 0.0;
        atomicOr(status, kDevSingular);
      }
      if (kGreen)
        for (int k = tid; k < m.gw; k += nt) grow[k] = 0.0;
      else
        for (int k = tid; k < m.sr_size; k += nt) ostore[static_cast<size_t>(sample) * m.sr_size + k] = 0.0;
      __syncthreads();
      continue;
    }
    // IP and the term values
    double ip = 0.0;
    for (int q = 0; q < m.nqp; ++q) ip += m.qpw[q] * pf[q];
    for (int t = tid; t < m.nterm; t += nt) {
      const int ti = m.tterm[4 * t], tsi = m.tterm[4 * t + 1], tj = m.tterm[4 * t + 2], tsj = m.tterm[4 * t + 3];
      const int dst = ti + tsi * ns, src = tj + tsj * ns;
      double g;
      if (tsi == tsj && ti == tj) {
        g = static_cast<double>(num[src]);
      } else if (tsi != tsj || num[dst] == 1 || num[src] == 0 || cfg[src] < 0) {
        g = 0.0;
      } else {
        // calh1_direct_projection_ratio_moved: source = tj, dest = ti, spin tsj
        const double z = direct_hop_log_proj(m, num, cj, tj, ti, src, dst);
        g = exp(z) * tacc[t] / ip;
      }
      g1[t] = g;
    }
    __syncthreads();
    if (tid == 0) {
      double e = 0.0;
      for (int k = 0; k < m.nintra; ++k) {
        const int i = m.intra_i[k];
        e += m.intra_v[k] * static_cast<double>(num[i] * num[i + ns]);
      }
      for (int k = 0; k < m.ninter; ++k) {
        const int i = m.inter_ij[2 * k], j = m.inter_ij[2 * k + 1];
        e += m.inter_v[k] * static_cast<double>(num[i] + num[i + ns]) * static_cast<double>(num[j] + num[j + ns]);
      }
      for (int k = 0; k < m.nhund; ++k) {
        const int i = m.hund_ij[2 * k], j = m.hund_ij[2 * k + 1];
        e -= m.hund_v[k] * (static_cast<double>(num[i] * num[j]) + static_cast<double>(num[i + ns] * num[j + ns]));
      }
      double transfer = 0.0;
      for (int t = 0; t < m.nterm; ++t) transfer -= m.tval[t] * g1[t];
      e += transfer;
      const bool ok = fabs(ip) >= 1.0e-100 && isfinite(e);
      valid[sample] = ok ? 1 : 0;
      eloc[sample] = ok ? e : 0.0;
      // ln|Ψ(x)| = Σ_k α_k c_k (Gutzwiller-Jastrow exponent) + ln|IP|
      double lp = 0.0;
      for (int k = 0; k < m.nproj; ++k) lp += m.proj[k] * static_cast<double>(cnt[k]);
      lpsi[sample] = ok ? lp + log(fabs(ip)) : 0.0;
      pf[m.nqp] = ip;
      pf[m.nqp + 1] = ok ? 1.0 : 0.0;
    }
    __syncthreads();
    const bool ok = pf[m.nqp + 1] != 0.0;
    if (kGreen) {
      green_finish(m, ip, ok, cfg, num, cj, gacc, grow);
      continue;
    }
    const double inv_ip = ip / (ip * ip);
    double* orow = ostore + static_cast<size_t>(sample) * m.sr_size;
    for (int k = tid; k < m.sr_size; k += nt) {
      double v;
      if (k == 0) v = 1.0;
      else if (k <= m.nproj) v = static_cast<double>(cnt[k - 1]);
      else v = oacc[k - 1 - m.nproj] * inv_ip;
      orow[k] = ok ? v : 0.0;
    }
    __syncthreads();
  }
}

// ---- planes whose strict upper triangle fits shared memory -----------------------------
// For n where the full FP64 plane does not fit one SM (2D 16×16, n = 224: 401 KB) the
// sample's plane is swept as a packed upper triangle in shared memory (gj_pfinv_packed,
// 195 KB at n = 224), one 512-thread CTA per SM striding over the samples; nothing of the
// sweep touches L2. The transfer terms' per-term sums sit in the block's L2 workspace. The
// Slater derivative is gathered per orbital: thread k walks orbital k's translated site
// pairs in a fixed order and adds the electron pairs on them, so O rows are bitwise
// repeatable (no atomics).
struct PackedLayout {
  size_t idx, cfg, num, cnt, tr, tsg, pf, cj, rs, rowp, rowq, plane, total;
};

__host__ __device__ inline PackedLayout packed_layout(const DevModel& m) {
  PackedLayout L;
  size_t o = 0;
  L.idx = o; o = a16(o + sizeof(int) * m.n);
  L.cfg = o; o = a16(o + sizeof(int) * m.ns2);
  L.num = o; o = a16(o + sizeof(int) * m.ns2);
  L.cnt = o; o = a16(o + sizeof(int) * (m.nproj + 1));
  L.tr = o; o = a16(o + sizeof(int) * m.ns);
  L.tsg = o; o = a16(o + sizeof(int) * m.ns);
  L.pf = o; o = a16(o + sizeof(double) * (m.nqp + 2));
  L.cj = o; o = a16(o + sizeof(double) * m.ns);
  L.rs = o; o = a16(o + sizeof(int) * m.n);
  L.rowp = o; o = a16(o + 2 * sizeof(double) * m.n);
  L.rowq = o; o = a16(o + sizeof(double) * m.n);
  L.plane = o; o = a16(o + sizeof(double) * static_cast<size_t>(m.n) * (m.n - 1) / 2);
  L.total = o;
  return L;
}

constexpr int kPackedThreads = 512;

template <int JPL>
__global__ void __launch_bounds__(kPackedThreads, 1)
    k_measure_packed(DevModel m, const int* __restrict__ s_idx, const int* __restrict__ s_cfg,
                     const int* __restrict__ s_num, const int* __restrict__ s_cnt, int nsamples,
                     double* __restrict__ gws, size_t gws_stride, double* __restrict__ ostore,
                     double* __restrict__ eloc, double* __restrict__ lpsi, int* __restrict__ valid, unsigned* status) {
  extern __shared__ __align__(16) unsigned char smem[];
  const PackedLayout L = packed_layout(m);
  int* idx = reinterpret_cast<int*>(smem + L.idx);
  int* cfg = reinterpret_cast<int*>(smem + L.cfg);
  int* num = reinterpret_cast<int*>(smem + L.num);
  int* cnt = reinterpret_cast<int*>(smem + L.cnt);
  int* tinv = reinterpret_cast<int*>(smem + L.tr);
  int* tsg = reinterpret_cast<int*>(smem + L.tsg);
  double* pf = reinterpret_cast<double*>(smem + L.pf);
  double* cj = reinterpret_cast<double*>(smem + L.cj);
  int* rs = reinterpret_cast<int*>(smem + L.rs);
  double* rowp = reinterpret_cast<double*>(smem + L.rowp);
  double* rowq = reinterpret_cast<double*>(smem + L.rowq);
  double* P = reinterpret_cast<double*>(smem + L.plane);
  const int n = m.n, ns = m.ns, ne = m.ne, tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  double* tacc = gws + static_cast<size_t>(blockIdx.x) * gws_stride;  // [nterm] plane sums
  double* g1 = tacc + m.nterm;                                          // [nterm] term values
  __shared__ int s_bad;
  for (int i = tid; i < n; i += nt) rs[i] = i * n - i * (i + 1) / 2 - i - 1;

  for (int sample = blockIdx.x; sample < nsamples; sample += gridDim.x) {
    for (int k = tid; k < n; k += nt) idx[k] = s_idx[static_cast<size_t>(sample) * n + k];
    for (int k = tid; k < m.ns2; k += nt) {
      cfg[k] = s_cfg[static_cast<size_t>(sample) * m.ns2 + k];
      num[k] = s_num[static_cast<size_t>(sample) * m.ns2 + k];
    }
    for (int k = tid; k < m.nproj; k += nt) cnt[k] = s_cnt[static_cast<size_t>(sample) * m.nproj + k];
    for (int k = tid; k < m.nterm; k += nt) tacc[k] = 0.0;
    double* orow = ostore + static_cast<size_t>(sample) * m.sr_size;
    for (int k = tid; k < m.norb; k += nt) orow[1 + m.nproj + k] = 0.0;
    if (tid == 0) s_bad = 0;
    __syncthreads();
    for (int r = tid; r < ns; r += nt) {  // cj[r] = Σ_site J[r][site]·(n_site − 1)
      double acc = 0.0;
      for (int site = 0; site < ns; ++site)
        acc += __ldg(m.jast_pair + r * ns + site) * static_cast<double>(num[site] + num[site + ns] - 1);
      cj[r] = acc;
    }
    if (tid == 0) {
      bool all_zero = true, all_neg = true;
      for (int k = 0; k < n; ++k) {
        all_zero = all_zero && idx[k] == 0;
        all_neg = all_neg && idx[k] < 0;
      }
      if (all_zero || all_neg) s_bad = 1;
    }
    __syncthreads();
    if (s_bad) {
      if (tid == 0) {
        valid[sample] = 0;
        eloc[sample] = 0.0;
        lpsi[sample] = 0.0;
      }
      for (int k = tid; k < m.sr_size; k += nt) orow[k] = 0.0;
      __syncthreads();
      continue;
    }
    for (int q = 0; q < m.nqp; ++q) {
      double pfv;
      int st;
      if (m.rinv) {
        // resident measurement: the upper triangle of the sampler's X⁻¹ of this sample
        const double* src = m.rinv + (static_cast<size_t>(sample) * m.nqp + q) * n * n;
        for (int i = warp; i < n - 1; i += nwarp)
          for (int j = i + 1 + lane; j < n; j += 32) P[rs[i] + j] = src[static_cast<size_t>(i) * n + j];
        pfv = m.rpf[static_cast<size_t>(sample) * m.nqp + q];
        st = 0;
        __syncthreads();
      } else {
        for (int i = warp; i < n - 1; i += nwarp) {  // X(i, j), i < j, from the Slater table
          const int ri = idx[i] + (i >= ne ? ns : 0);
          const double* srow = m.slater + (static_cast<size_t>(q) * m.ns2 + ri) * m.ns2;
          for (int j = i + 1 + lane; j < n; j += 32) P[rs[i] + j] = __ldg(srow + idx[j] + (j >= ne ? ns : 0));
        }
        __syncthreads();
        gj_pfinv_packed<JPL, (kPackedThreads > 512 ? 1 : 2)>(P, rs, n, rowp, rowq, pfv, st);
      }
      if (st != 0) {
        if (tid == 0) s_bad = 1;
        __syncthreads();
        break;
      }
      if (tid == 0) pf[q] = pfv;
      const double wq = m.qpw[q];
      // transfer terms: one-electron ratio on this plane (warp per term)
      for (int t = warp; t < m.nterm; t += nwarp) {
        const int ti = m.tterm[4 * t], tsi = m.tterm[4 * t + 1], tj = m.tterm[4 * t + 2], tsj = m.tterm[4 * t + 3];
        const int dst = ti + tsi * ns, src = tj + tsj * ns;
        if (tsi != tsj || (ti == tj) || num[dst] == 1 || num[src] == 0 || cfg[src] < 0) continue;
        const int msj = cfg[src] + tsj * ne;
        const int rsa = ti + tsj * ns;
        const double* srow = m.slater + (static_cast<size_t>(q) * m.ns2 + rsa) * m.ns2;
        double sv[JPL];  // the gathered Slater row: every load of the lane in flight at once
#pragma unroll
        for (int c = 0; c < JPL; ++c) {
          const int k = lane + 32 * c;
          sv[c] = k < n ? __ldg(srow + (k == msj ? ti : idx[k]) + (k >= ne ? ns : 0)) : 0.0;
        }
        double r = 0.0;
#pragma unroll
        for (int c = 0; c < JPL; ++c) {
          const int k = lane + 32 * c;
          if (k < n) r += packed_at(P, rs, msj, k) * sv[c];
        }
        r = warp_sum(r);
        if (lane == 0) {
          const double v = wq * (-r * pfv);
          if (q == 0) tacc[t] = v;  // a plain store: no read of the block's workspace
          else tacc[t] += v;
        }
      }
      // Slater derivative by orbital: electron pairs (i, j) on the orbital's site pairs
      const int trans = q / m.nleg, spidx = q % m.nleg, mpidx = trans % m.nmp;
      for (int k = tid; k < ns; k += nt) {
        const int a = m.trans_inv[mpidx * ns + k];
        tinv[k] = a;
        tsg[a] = m.trans_sgn[mpidx * ns + a];
      }
      __syncthreads();
      const double cs = pfv * m.spgl[spidx], cc = pfv * m.spgl[m.nleg + spidx], ss = pfv * m.spgl[2 * m.nleg + spidx];
      const double fac[4] = {cs, -cc, ss, -cs};  // (up, up), (up, dn), (dn, up), (dn, dn)
      for (int k = tid; k < m.norb; k += nt) {
        double acc = 0.0;
        const int e1 = __ldg(m.orb_off + k + 1);
        for (int e = __ldg(m.orb_off + k); e < e1; ++e) {
          const int ent = __ldg(m.orb_ent + e);
          const int a = tinv[ent >> 16], b = tinv[(ent >> 1) & 0x7fff];
          const int sgn = (ent & 1 ? -1 : 1) * tsg[a] * tsg[b];
#pragma unroll
          for (int sa = 0; sa < 2; ++sa) {
            const int ei = cfg[a + sa * ns];
            if (ei < 0) continue;
#pragma unroll
            for (int sb = 0; sb < 2; ++sb) {
              const int ej = cfg[b + sb * ns];
              if (ej < 0) continue;
              const double v = packed_at(P, rs, ei + sa * ne, ej + sb * ne);
              acc += (fac[2 * sa + sb] * v) * static_cast<double>(sgn);
            }
          }
        }
        orow[1 + m.nproj + k] += wq * acc;
      }
      __syncthreads();
    }
    if (s_bad) {
      if (tid == 0) {
        valid[sample] = 0;
        eloc[sample] = 0.0;
        lpsi[sample] = 0.0;
        atomicOr(status, kDevSingular);
      }
      for (int k = tid; k < m.sr_size; k += nt) orow[k] = 0.0;
      __syncthreads();
      continue;
    }
    double ip = 0.0;
    for (int q = 0; q < m.nqp; ++q) ip += m.qpw[q] * pf[q];
    for (int t = tid; t < m.nterm; t += nt) {
      const int ti = m.tterm[4 * t], tsi = m.tterm[4 * t + 1], tj = m.tterm[4 * t + 2], tsj = m.tterm[4 * t + 3];
      const int dst = ti + tsi * ns, src = tj + tsj * ns;
      double g;
      if (tsi == tsj && ti == tj) g = static_cast<double>(num[src]);
      else if (tsi != tsj || num[dst] == 1 || num[src] == 0 || cfg[src] < 0) g = 0.0;
      else g = exp(direct_hop_log_proj(m, num, cj, tj, ti, src, dst)) * tacc[t] / ip;
      // the transfer sum Σ_t −t_t·g_t in a fixed order: per thread over its terms, warps
      // by shuffles, warps in order below
      g1[t] = -m.tval[t] * g;
    }
    double part = 0.0;
    for (int t = tid; t < m.nterm; t += nt) part += g1[t];
    part = warp_sum(part);
    if (lane == 0) rowq[warp] = part;  // the sweep's row buffer is free here
    __syncthreads();
    if (tid == 0) {
      double e = 0.0;
      for (int k = 0; k < m.nintra; ++k) {
        const int i = m.intra_i[k];
        e += m.intra_v[k] * static_cast<double>(num[i] * num[i + ns]);
      }
      for (int k = 0; k < m.ninter; ++k) {
        const int i = m.inter_ij[2 * k], j = m.inter_ij[2 * k + 1];
        e += m.inter_v[k] * static_cast<double>(num[i] + num[i + ns]) * static_cast<double>(num[j] + num[j + ns]);
      }
      for (int k = 0; k < m.nhund; ++k) {
        const int i = m.hund_ij[2 * k], j = m.hund_ij[2 * k + 1];
        e -= m.hund_v[k] * (static_cast<double>(num[i] * num[j]) + static_cast<double>(num[i + ns] * num[j + ns]));
      }
      double transfer = 0.0;
      for (int w = 0; w < nwarp; ++w) transfer += rowq[w];
      e += transfer;
      const bool ok = fabs(ip) >= 1.0e-100 && isfinite(e);
      valid[sample] = ok ? 1 : 0;
      eloc[sample] = ok ? e : 0.0;
      double lp = 0.0;
      for (int k = 0; k < m.nproj; ++k) lp += m.proj[k] * static_cast<double>(cnt[k]);
      lpsi[sample] = ok ? lp + log(fabs(ip)) : 0.0;
      pf[m.nqp + 1] = ok ? 1.0 : 0.0;
    }
    __syncthreads();
    const bool ok = pf[m.nqp + 1] != 0.0;
    const double inv_ip = ip / (ip * ip);
    for (int k = tid; k < m.sr_size; k += nt) {
      double v;
      if (k == 0) v = 1.0;
      else if (k <= m.nproj) v = static_cast<double>(cnt[k - 1]);
      else v = orow[k] * inv_ip;
      orow[k] = ok ? v : 0.0;
    }
    __syncthreads();
  }
}

bool packed_measure_fits(const DevModel& m, int limit) {
  return m.orb_off != nullptr && m.trans_inv != nullptr && m.n <= 256 &&
         packed_layout(m).total <= static_cast<size_t>(limit);
}

template <int JPL>
int launch_measure_packed(const DevModel& m, const int* s_idx, const int* s_cfg, const int* s_num, const int* s_cnt,
                          int nsamples, double* gws, size_t gws_stride, int gws_blocks, double* ostore, double* eloc,
                          double* lpsi, int* valid, unsigned* status, cudaStream_t stream) {
  const size_t smem = packed_layout(m).total;
  auto kernel = k_measure_packed<JPL>;
  MVMCB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  const int grid = std::max(1, std::min({nsamples, gws_blocks, current_device_attr(cudaDevAttrMultiProcessorCount)}));
  kernel<<<grid, kPackedThreads, smem, stream>>>(m, s_idx, s_cfg, s_num, s_cnt, nsamples, gws, gws_stride, ostore,
                                                 eloc, lpsi, valid, status);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

// Per-walker sums in sample order: [Wc, E, E², Sz, Sz²] and HO, ⟨O⟩, ⟨O²⟩ (unnormalised).
__global__ void k_reduce_walker(const DevModel m, const double* __restrict__ ostore,
                                const double* __restrict__ eloc, const int* __restrict__ valid,
                                const int* __restrict__ s_num, int S, double* __restrict__ wsum) {
  const int wk = blockIdx.x;
  const int size = m.sr_size;
  double* out = wsum + static_cast<size_t>(wk) * (5 + 3 * size);
  if (threadIdx.x == 0) {
    double wc = 0, e1 = 0, e2 = 0, z1 = 0, z2 = 0;
    for (int s = 0; s < S; ++s) {
      const size_t smp = static_cast<size_t>(wk) * S + s;
      if (!valid[smp]) continue;
      const double e = eloc[smp];
      double sz = 0.0;
      for (int r = 0; r < m.ns; ++r)
        sz += static_cast<double>(s_num[smp * m.ns2 + r] - s_num[smp * m.ns2 + r + m.ns]);
      wc += 1.0;
      e1 += 1.0 * e;
      e2 += (1.0 * e) * e;
      z1 += 1.0 * sz;
      z2 += 1.0 * sz * sz;
    }
    out[0] = wc;
    out[1] = e1;
    out[2] = e2;
    out[3] = z1;
    out[4] = z2;
  }
  for (int i = threadIdx.x; i < size; i += blockDim.x) {
    double ho = 0.0, mean = 0.0, diag = 0.0;
    for (int s = 0; s < S; ++s) {
      const size_t smp = static_cast<size_t>(wk) * S + s;
      const double o = ostore[smp * size + i];  // invalid rows are zero
      if (valid[smp]) ho += (1.0 * eloc[smp]) * o;
      mean += o;
      diag += o * o;
    }
    out[5 + i] = ho;
    out[5 + size + i] = mean;
    out[5 + 2 * size + i] = diag;
  }
}

// Walker-order fold and weight average: tot = [Wc, E, E², Sz, Sz², HO.., mean.., diag..].
__global__ void k_reduce_total(int W, int size, const double* __restrict__ wsum, double* __restrict__ tot) {
  const int width = 5 + 3 * size;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < width; k += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int w = 0; w < W; ++w) acc += wsum[static_cast<size_t>(w) * width + k];
    tot[k] = acc;
  }
}

__global__ void k_weight_average(int size, double* tot) {
  const double wc = tot[0];
  if (fabs(wc) < 1.0e-15) return;
  const double inv = 1.0 / wc;
  const int width = 5 + 3 * size;
  for (int k = 1 + threadIdx.x + blockIdx.x * blockDim.x; k < width; k += blockDim.x * gridDim.x) tot[k] *= inv;
}

size_t measure_smem(const DevModel& m, bool smem_plane) { return meas_layout(m, smem_plane).total; }

template <int JPL, bool kGreen>
int launch_measure_kind(const DevModel& m_in, const int* s_idx, const int* s_cfg, const int* s_num, const int* s_cnt,
                        int nsamples, double* gws, int gws_blocks, double* ostore, double* eloc, double* lpsi,
                        int* valid, double* gval, unsigned* status, cudaStream_t stream, int limit) {
  DevModel m = m_in;
  // one-body plane sums in shared memory when they fit beside the layout (planes in shared
  // memory if those fit too)
  m.gacc_smem = 0;
  if (kGreen) {
    // One-body plane sums in shared memory only when that costs no co-resident sample: the
    // measurement is latency bound, and two samples per SM with the sums in the L2-resident
    // row beat one sample per SM with them in shared memory (24.8 → 14.6 ms at 2D 8×8 with
    // the 8192-term list). MVMC_B200_GREEN_ACC=smem|global overrides.
    auto per_sm = [&](bool acc) {
      DevModel t = m;
      t.gacc_smem = acc ? 1 : 0;
      size_t total = meas_layout(t, true, true).total;
      if (total > static_cast<size_t>(limit)) total = meas_layout(t, false, true).total;
      return total > static_cast<size_t>(limit) ? 0 : static_cast<int>((limit + 1024) / (total + 1024));
    };
    m.gacc_smem = per_sm(true) >= per_sm(false) && per_sm(true) > 0 ? 1 : 0;
    if (const char* e = std::getenv("MVMC_B200_GREEN_ACC")) {
      if (std::strcmp(e, "global") == 0) m.gacc_smem = 0;
      if (std::strcmp(e, "smem") == 0 && per_sm(true) > 0) m.gacc_smem = 1;
    }
  }
  const bool smem_plane = meas_layout(m, true, kGreen).total <= static_cast<size_t>(limit);
  const size_t smem = meas_layout(m, smem_plane, kGreen).total;
  if (smem > static_cast<size_t>(limit)) return kErrArgument;
  if (smem_plane) {
    auto kernel = k_measure<JPL, true, kGreen>;
    MVMCB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    kernel<<<nsamples, kMeasThreads, smem, stream>>>(m, s_idx, s_cfg, s_num, s_cnt, nsamples, gws, ostore, eloc, lpsi,
                                                     valid, gval, status);
  } else {
    // As many blocks as are co-resident, striding over the samples: each block reuses its
    // own workspace, so the workspaces stay in L2 across samples. When two 256-thread
    // blocks per SM would hold more plane bytes than ~3/4 of the L2 (2D 16×16: 401 KB per
    // sample), one 512-thread block per SM sweeps instead.
    int dev = 0, sms = 0, per = 0, l2 = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev);
    const double plane_bytes = 8.0 * m.n * m.n;
    bool wide = !kGreen && 2.0 * sms * plane_bytes > 0.75 * l2;
    if (const char* e = std::getenv("MVMC_B200_MEAS_THREADS")) wide = !kGreen && std::strcmp(e, "512") == 0;
    if (wide) {
      auto kernel = k_measure<JPL, false, kGreen, 512>;
      MVMCB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
      MVMCB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, 512, smem));
      const int grid = std::max(1, std::min({nsamples, gws_blocks, sms * std::max(1, per)}));
      kernel<<<grid, 512, smem, stream>>>(m, s_idx, s_cfg, s_num, s_cnt, nsamples, gws, ostore, eloc, lpsi, valid,
                                          gval, status);
    } else {
      auto kernel = k_measure<JPL, false, kGreen>;
      MVMCB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
      MVMCB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kMeasThreads, smem));
      const int grid = std::max(1, std::min({nsamples, gws_blocks, sms * std::max(1, per)}));
      kernel<<<grid, kMeasThreads, smem, stream>>>(m, s_idx, s_cfg, s_num, s_cnt, nsamples, gws, ostore, eloc, lpsi,
                                                   valid, gval, status);
    }
  }
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

template <int JPL>
int launch_measure_jpl(const DevModel& m, const int* s_idx, const int* s_cfg, const int* s_num, const int* s_cnt,
                       int nsamples, double* gws, int gws_blocks, double* ostore, double* eloc, double* lpsi,
                       int* valid, double* gval, unsigned* status, cudaStream_t stream, int limit) {
  if (gval)
    return launch_measure_kind<JPL, true>(m, s_idx, s_cfg, s_num, s_cnt, nsamples, gws, gws_blocks, ostore, eloc,
                                          lpsi, valid, gval, status, stream, limit);
  return launch_measure_kind<JPL, false>(m, s_idx, s_cfg, s_num, s_cnt, nsamples, gws, gws_blocks, ostore, eloc,
                                         lpsi, valid, gval, status, stream, limit);
}


// gval != nullptr selects the PhysCal form: Green rows [nsamples][m.gw] instead of O rows.
// Planes that do not fit one SM's shared memory are swept as packed upper triangles in
// shared memory (k_measure_packed) when those fit, else in place in each block's L2
// workspace (MVMC_B200_MEASURE=l2 selects the latter).
int launch_measure(const DevModel& m, const int* s_idx, const int* s_cfg, const int* s_num,
                   const int* s_cnt, int nsamples, double* gws, int gws_blocks, double* ostore,
                   double* eloc, double* lpsi, int* valid, double* gval, unsigned* status, cudaStream_t stream) {
  int dev = 0, limit = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&limit, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const int n = m.n;
  const char* mode = std::getenv("MVMC_B200_MEASURE");
  // planes too large for shared memory whose upper triangle fits: the packed sweep
  // (MVMC_B200_MEASURE=l2 keeps the in-place sweep of full planes in L2)
  const size_t gws_stride = static_cast<size_t>(2) * n * n;
  if (!gval && meas_layout(m, true).total > static_cast<size_t>(limit) && packed_measure_fits(m, limit) &&
      gws_stride >= static_cast<size_t>(2) * m.nterm && !(mode && std::strcmp(mode, "l2") == 0)) {
    if (n <= 224)
      return launch_measure_packed<7>(m, s_idx, s_cfg, s_num, s_cnt, nsamples, gws, gws_stride, gws_blocks, ostore,
                                      eloc, lpsi, valid, status, stream);
    return launch_measure_packed<8>(m, s_idx, s_cfg, s_num, s_cnt, nsamples, gws, gws_stride, gws_blocks, ostore,
                                    eloc, lpsi, valid, status, stream);
  }
#define MVMCB_MEASURE(J) \
  launch_measure_jpl<J>(m, s_idx, s_cfg, s_num, s_cnt, nsamples, gws, gws_blocks, ostore, eloc, lpsi, valid, gval, \
                        status, stream, limit)
  if (n <= 32) return MVMCB_MEASURE(1);
  if (n <= 64) return MVMCB_MEASURE(2);
  if (n <= 128) return MVMCB_MEASURE(4);
  if (n <= 224) return MVMCB_MEASURE(7);
  if (n <= 256) return MVMCB_MEASURE(8);
#undef MVMCB_MEASURE
  return kErrArgument;
}

// PhysCal Green functions of the measured samples: out = [one-body (n_one) | TwoBodyGEx
// (pairs of one-body values, one per ex entry) | TwoBodyG (ngtwo)]. Every walker's sums in
// sample order over its valid samples are scaled by its 1/Wc, summed in walker order and
// scaled by 1/W (normalize_physcal_green run.rs:287-316; average_physcal_rank_contributions
// run.rs:1158-1181; accumulate_two_body_gex_sample observables.rs:110-126). Pass 1: blocks
// (x, y) sum the walkers of chunk y; pass 2 adds the chunks in order.
__global__ void k_green_partial(int W, int S, int nchunk, int gw, int n_one, int two_off, int ngtwo, int nex,
                                const int* __restrict__ ex, const double* __restrict__ gval,
                                const int* __restrict__ valid, double* __restrict__ part) {
  const int width = n_one + nex + ngtwo;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= width) return;
  const int w0 = static_cast<int>(static_cast<long long>(W) * blockIdx.y / nchunk);
  const int w1 = static_cast<int>(static_cast<long long>(W) * (blockIdx.y + 1) / nchunk);
  int a = -1, b = -1, col = k;
  if (k >= n_one && k < n_one + nex) {
    a = ex[2 * (k - n_one)];
    b = ex[2 * (k - n_one) + 1];
  } else if (k >= n_one + nex) {
    col = two_off + (k - n_one - nex);
  }
  double tot = 0.0;
  for (int w = w0; w < w1; ++w) {
    double wc = 0.0, acc = 0.0;
    for (int s = 0; s < S; ++s) {
      const size_t smp = static_cast<size_t>(w) * S + s;
      if (!valid[smp]) continue;
      const double* row = gval + smp * gw;
      wc += 1.0;
      acc += a >= 0 ? (1.0 * row[a]) * row[b] : row[col];
    }
    if (wc != 0.0) acc *= 1.0 / wc;
    tot += acc;
  }
  part[static_cast<size_t>(blockIdx.y) * width + k] = tot;
}

__global__ void k_green_total(int W, int nchunk, int width, const double* __restrict__ part, double* __restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < width; k += gridDim.x * blockDim.x) {
    double tot = 0.0;
    for (int c = 0; c < nchunk; ++c) tot += part[static_cast<size_t>(c) * width + k];
    if (W > 1) tot *= 1.0 / W;
    out[k] = tot;
  }
}

int green_chunks(int W) { return std::max(1, std::min(W, 64)); }

int launch_green_reduce(const DevModel& m, int W, int S, int n_one, int nex, const int* ex, const double* gval,
                        const int* valid, double* part, double* out, cudaStream_t stream) {
  const int width = n_one + nex + m.ngtwo;
  if (width == 0) return kOk;
  const int nchunk = green_chunks(W);
  // the TwoBodyG values sit after all ngone one-body values of the row
  k_green_partial<<<dim3((width + 127) / 128, nchunk), 128, 0, stream>>>(W, S, nchunk, m.gw, n_one, m.ngone, m.ngtwo,
                                                                         nex, ex, gval, valid, part);
  MVMCB_CUDA(cudaGetLastError());
  k_green_total<<<(width + 255) / 256, 256, 0, stream>>>(W, nchunk, width, part, out);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

// Walker-order totals and weight average of per-walker sums already in wsum.
int launch_reduce_totals(const DevModel& m, int W, const double* wsum, double* tot, cudaStream_t stream) {
  const int width = 5 + 3 * m.sr_size;
  k_reduce_total<<<(width + 255) / 256, 256, 0, stream>>>(W, m.sr_size, wsum, tot);
  MVMCB_CUDA(cudaGetLastError());
  k_weight_average<<<(width + 255) / 256, 256, 0, stream>>>(m.sr_size, tot);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

int launch_reduce(const DevModel& m, int W, int S, const double* ostore, const double* eloc,
                  const int* valid, const int* s_num, double* wsum, double* tot, cudaStream_t stream) {
  k_reduce_walker<<<W, 256, 0, stream>>>(m, ostore, eloc, valid, s_num, S, wsum);
  MVMCB_CUDA(cudaGetLastError());
  const int width = 5 + 3 * m.sr_size;
  k_reduce_total<<<(width + 255) / 256, 256, 0, stream>>>(W, m.sr_size, wsum, tot);
  MVMCB_CUDA(cudaGetLastError());
  k_weight_average<<<(width + 255) / 256, 256, 0, stream>>>(m.sr_size, tot);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

}  // namespace mvmcb
