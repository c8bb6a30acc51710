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
// The reductions sum per walker in sample order and then across walkers in walker
// order (the rank-order fold of ThreadReducer, multichain.rs:433), so reruns are
// bitwise repeatable up to the O_k scatter (shared-memory atomics).
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "engine.cuh"
#include "pfinv.cuh"

namespace mvmcb {

constexpr int kMeasThreads = 256;

struct MeasLayout {
  size_t idx, cfg, num, cnt, tr, sg, pf, tacc, g1, oacc, cj, gj, plane, total;
};

__host__ __device__ inline size_t a16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline MeasLayout meas_layout(const DevModel& m, bool smem_plane) {
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
  L.gj = o;
  L.plane = o;
  // the plane and its ping-pong partner
  if (smem_plane) o = a16(o + 2 * sizeof(double) * static_cast<size_t>(m.n) * m.n);
  L.total = o;
  return L;
}

template <int JPL, bool kSmemPlane>
__global__ void __launch_bounds__(kMeasThreads, (kSmemPlane ? 1 : 2))
    k_measure(DevModel m, const int* __restrict__ s_idx, const int* __restrict__ s_cfg,
              const int* __restrict__ s_num, const int* __restrict__ s_cnt, int nsamples,
              double* __restrict__ gws, double* __restrict__ ostore, double* __restrict__ eloc,
              double* __restrict__ lpsi, int* __restrict__ valid, unsigned* status) {
  extern __shared__ __align__(16) unsigned char smem[];
  const MeasLayout L = meas_layout(m, kSmemPlane);
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
    if (tid == 0) s_bad = 0;
    __syncthreads();
    // direct projection helper: cj[r] = Σ_site J[r][site]·(n_site − 1)
    for (int r = tid; r < ns; r += nt) {
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
      for (int k = tid; k < m.sr_size; k += nt) ostore[static_cast<size_t>(sample) * m.sr_size + k] = 0.0;
      __syncthreads();
      continue;
    }
    for (int q = 0; q < m.nqp; ++q) {
      for (int k = tid; k < n * n; k += nt) {
        const int i = k / n, j = k - i * n;
        const int ri = idx[i] + (i >= ne ? ns : 0), rj = idx[j] + (j >= ne ? ns : 0);
        A[k] = __ldg(m.slater + (static_cast<size_t>(q) * m.ns2 + ri) * m.ns2 + rj);
      }
      __syncthreads();
      double pfv;
      int st;
      // planes in L2: a few rows in flight per warp, fewer for wide rows so that two
      // samples share an SM
      gj_pfinv_pp<double, JPL, kSmemPlane ? 1 : (JPL <= 2 ? 4 : (JPL <= 4 ? 2 : 1))>(A, Bpp, n, pfv, st);
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
      // adjoint Slater derivative: translated sites of the electrons for this plane
      const int trans = q / m.nleg, spidx = q % m.nleg;
      const int mpidx = trans % m.nmp;
      for (int k = tid; k < n; k += nt) {
        tr[k] = m.trans[mpidx * ns + idx[k]];
        sg[k] = m.trans_sgn[mpidx * ns + idx[k]];
      }
      __syncthreads();
      const double cs = pfv * m.spgl[spidx], cc = pfv * m.spgl[m.nleg + spidx], ss = pfv * m.spgl[2 * m.nleg + spidx];
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
      __syncthreads();
    }
    if (s_bad) {
      if (tid == 0) {
        valid[sample] = 0;
        eloc[sample] = 0.0;
        lpsi[sample] = 0.0;
        atomicOr(status, kDevSingular);
      }
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
        const int source = tj, dest = ti;
        auto occ = [&](int slot) { return slot == src ? 0 : (slot == dst ? 1 : num[slot]); };
        auto chm = [&](int site) { return occ(site) + occ(ns + site) - 1; };
        auto ch = [&](int site) { return num[site] + num[ns + site] - 1; };
        double z = 0.0;
        z -= m.gutz_site[source] * static_cast<double>(occ(source) + occ(ns + source));
        z += m.gutz_site[dest] * static_cast<double>(occ(dest) * occ(ns + dest));
        const double jsd = m.jast_pair[source * ns + dest];
        z += jsd * static_cast<double>(chm(source) - chm(dest) + 1);
        const double sum_dest = cj[dest] - m.jast_pair[dest * ns + source] * static_cast<double>(ch(source));
        const double sum_src = cj[source] - m.jast_pair[source * ns + dest] * static_cast<double>(ch(dest));
        z += sum_dest - sum_src;
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

template <int JPL>
int launch_measure_jpl(const DevModel& m, const int* s_idx, const int* s_cfg, const int* s_num,
                       const int* s_cnt, int nsamples, double* gws, int gws_blocks, double* ostore,
                       double* eloc, double* lpsi, int* valid, unsigned* status, cudaStream_t stream, int limit) {
  const bool smem_plane = meas_layout(m, true).total <= static_cast<size_t>(limit);
  const size_t smem = meas_layout(m, smem_plane).total;
  if (smem > static_cast<size_t>(limit)) return kErrArgument;
  if (smem_plane) {
    auto kernel = k_measure<JPL, true>;
    MVMCB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    kernel<<<nsamples, kMeasThreads, smem, stream>>>(m, s_idx, s_cfg, s_num, s_cnt, nsamples, gws, ostore, eloc, lpsi,
                                                     valid, status);
  } else {
    auto kernel = k_measure<JPL, false>;
    MVMCB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    // As many blocks as are co-resident, striding over the samples: each block reuses its
    // own ping-pong workspace, so the workspaces stay in L2 across samples.
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    MVMCB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kMeasThreads, smem));
    const int grid = std::max(1, std::min({nsamples, gws_blocks, sms * std::max(1, per)}));
    kernel<<<grid, kMeasThreads, smem, stream>>>(m, s_idx, s_cfg, s_num, s_cnt, nsamples, gws, ostore, eloc, lpsi,
                                                 valid, status);
  }
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

int launch_measure(const DevModel& m, const int* s_idx, const int* s_cfg, const int* s_num,
                   const int* s_cnt, int nsamples, double* gws, int gws_blocks, double* ostore,
                   double* eloc, double* lpsi, int* valid, unsigned* status, cudaStream_t stream) {
  int dev = 0, limit = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&limit, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const int n = m.n;
  if (n <= 32) return launch_measure_jpl<1>(m, s_idx, s_cfg, s_num, s_cnt, nsamples, gws, gws_blocks, ostore, eloc, lpsi, valid, status, stream, limit);
  if (n <= 64) return launch_measure_jpl<2>(m, s_idx, s_cfg, s_num, s_cnt, nsamples, gws, gws_blocks, ostore, eloc, lpsi, valid, status, stream, limit);
  if (n <= 128) return launch_measure_jpl<4>(m, s_idx, s_cfg, s_num, s_cnt, nsamples, gws, gws_blocks, ostore, eloc, lpsi, valid, status, stream, limit);
  if (n <= 224) return launch_measure_jpl<7>(m, s_idx, s_cfg, s_num, s_cnt, nsamples, gws, gws_blocks, ostore, eloc, lpsi, valid, status, stream, limit);
  if (n <= 256) return launch_measure_jpl<8>(m, s_idx, s_cfg, s_num, s_cnt, nsamples, gws, gws_blocks, ostore, eloc, lpsi, valid, status, stream, limit);
  return kErrArgument;
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
