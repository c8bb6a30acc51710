// K3 + K4 for planes larger than one SM's shared memory (2D 16×16: n = 224, 401 KB in
// FP64): one two-CTA thread-block cluster per saved sample. Each CTA keeps half of the
// rows of the plane in its shared memory and the pair sweeps the plane in place with the
// skew Gauss–Jordan step of gj_pfinv_pp (pfinv.cuh); the pivot rows p and q are read
// through distributed shared memory by the CTA that does not own them. Afterwards each CTA
// evaluates the transfer-term ratios of the electrons whose rows it holds and adds the
// adjoint Slater derivative of its rows; rank 0 combines, computes the energy and writes
// the sample's O row (accumulate_observables_local, crates/mvmc-core/src/run.rs:2937-3614;
// CalculateMAll pfaffian.rs:871-927; calh1_real_fast observables.rs:1680; the adjoint
// slater_derivative.rs:289-550; calculate_oo_store_real observables.rs:297).
//
// Every barrier here is a hardware barrier (__syncthreads, barrier.cluster): no spin loop.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "engine.cuh"

namespace cg = cooperative_groups;

namespace mvmcb {

constexpr int kClusterThreads = 512;

struct ClusterLayout {
  size_t rows, rowbuf, idx, cfg, num, cnt, tr, sg, pf, cj, oacc, ctl, total;
};

__host__ __device__ inline size_t c16(size_t x) { return (x + 15) & ~size_t(15); }

// oacc_smem: the O_k sums of this CTA in shared memory (else in the sample's O row). The
// transfer-term plane sums live in a per-CTA slice of global scratch (L2).
__host__ __device__ inline ClusterLayout cluster_layout(const DevModel& m, bool oacc_smem) {
  ClusterLayout L;
  const int h = m.n / 2;
  size_t o = 0;
  L.rows = o; o = c16(o + sizeof(double) * static_cast<size_t>(h) * m.n);
  L.rowbuf = o; o = c16(o + sizeof(double) * 2 * m.n);
  L.idx = o; o = c16(o + sizeof(int) * m.n);
  L.cfg = o; o = c16(o + sizeof(int) * m.ns2);
  L.num = o; o = c16(o + sizeof(int) * m.ns2);
  L.cnt = o; o = c16(o + sizeof(int) * (m.nproj + 1));
  L.tr = o; o = c16(o + sizeof(int) * m.n);
  L.sg = o; o = c16(o + sizeof(int) * m.n);
  L.pf = o; o = c16(o + sizeof(double) * (m.nqp + 4));
  L.cj = o; o = c16(o + sizeof(double) * m.ns);
  L.oacc = o;
  if (oacc_smem) o = c16(o + sizeof(double) * (m.norb + 1));
  L.ctl = o; o = c16(o + sizeof(int) * 8 + sizeof(double) * 8);
  L.total = o;
  return L;
}

size_t cluster_measure_smem(const DevModel& m, bool oacc_smem) { return cluster_layout(m, oacc_smem).total; }

template <int JPL>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kClusterThreads, 1)
    k_measure_cluster(DevModel m, const int* __restrict__ s_idx, const int* __restrict__ s_cfg,
                      const int* __restrict__ s_num, const int* __restrict__ s_cnt, int nsamples, int oacc_smem,
                      double* __restrict__ scratch, double* __restrict__ ostore, double* __restrict__ eloc, double* __restrict__ lpsi,
                      int* __restrict__ valid, unsigned* status) {
  extern __shared__ __align__(16) unsigned char smem[];
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = static_cast<int>(cluster.block_rank());
  const ClusterLayout L = cluster_layout(m, oacc_smem != 0);
  const int n = m.n, ns = m.ns, ne = m.ne, h = n / 2, r0 = rank * h;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  double* rows = reinterpret_cast<double*>(smem + L.rows);  // rows r0 .. r0 + h − 1
  double* rowbuf = reinterpret_cast<double*>(smem + L.rowbuf);
  int* idx = reinterpret_cast<int*>(smem + L.idx);
  int* cfg = reinterpret_cast<int*>(smem + L.cfg);
  int* num = reinterpret_cast<int*>(smem + L.num);
  int* cnt = reinterpret_cast<int*>(smem + L.cnt);
  int* tr = reinterpret_cast<int*>(smem + L.tr);
  int* sg = reinterpret_cast<int*>(smem + L.sg);
  double* pf = reinterpret_cast<double*>(smem + L.pf);
  double* tacc = scratch + static_cast<size_t>(blockIdx.x) * (m.nterm + 1);  // this CTA's term sums
  double* cj = reinterpret_cast<double*>(smem + L.cj);
  int* ictl = reinterpret_cast<int*>(smem + L.ctl);
  double* dctl = reinterpret_cast<double*>(smem + L.ctl + sizeof(int) * 8);
  // the partner's rows (distributed shared memory)
  const double* prow = cluster.map_shared_rank(rows, rank ^ 1);
  const double* ptacc = scratch + static_cast<size_t>(blockIdx.x ^ 1) * (m.nterm + 1);
  const int clusters = gridDim.x / 2;

  for (int sample = blockIdx.x / 2; sample < nsamples; sample += clusters) {
    double* orow = ostore + static_cast<size_t>(sample) * m.sr_size;
    double* oacc = oacc_smem ? reinterpret_cast<double*>(smem + L.oacc) : orow + 1 + m.nproj;
    for (int k = tid; k < n; k += nt) idx[k] = s_idx[static_cast<size_t>(sample) * n + k];
    for (int k = tid; k < m.ns2; k += nt) {
      cfg[k] = s_cfg[static_cast<size_t>(sample) * m.ns2 + k];
      num[k] = s_num[static_cast<size_t>(sample) * m.ns2 + k];
    }
    for (int k = tid; k < m.nproj; k += nt) cnt[k] = s_cnt[static_cast<size_t>(sample) * m.nproj + k];
    for (int k = tid; k < m.nterm; k += nt) tacc[k] = 0.0;
    if (oacc_smem) {
      for (int k = tid; k < m.norb; k += nt) oacc[k] = 0.0;
    } else if (rank == 0) {
      for (int k = tid; k < m.norb; k += nt) oacc[k] = 0.0;  // both CTAs add into the O row
    }
    __syncthreads();
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
      ictl[0] = (all_zero || all_neg) ? 1 : 0;  // bad sample
    }
    cluster.sync();  // the O row is zeroed before either CTA adds to it
    bool bad = ictl[0] != 0;
    for (int q = 0; q < m.nqp && !bad; ++q) {
      const double* slq = m.slater + static_cast<size_t>(q) * m.ns2 * m.ns2;
      for (int k = tid; k < h * n; k += nt) {
        const int il = k / n, j = k - il * n, i = r0 + il;
        const int ri = idx[i] + (i >= ne ? ns : 0), rj = idx[j] + (j >= ne ? ns : 0);
        rows[k] = __ldg(slq + static_cast<size_t>(ri) * m.ns2 + rj);
      }
      unsigned swept = 0;  // bit c: column lane + 32c swept (identical in every warp)
      int p = 0, parity = 0, st = 0;
      double pfv = 1.0;
      cluster.sync();  // both halves gathered
      for (int step = 0; step < n / 2; ++step) {
        // row p into rowbuf[0] (from the CTA that owns it)
        const double* srcp = (p / h == rank ? rows : prow) + static_cast<size_t>(p - (p / h) * h) * n;
        for (int j = tid; j < n; j += nt) rowbuf[j] = srcp[j];
        __syncthreads();
        // pivot search on row p by every warp (identical result), parity of (p, q)
        double rp[JPL];
        double best = -1.0;
        int bi = n;
#pragma unroll
        for (int c = 0; c < JPL; ++c) {
          const int j = lane + 32 * c;
          rp[c] = j < n ? rowbuf[j] : 0.0;
          if (j < n && j != p && !((swept >> c) & 1u)) {
            const double v = fabs(rp[c]);
            if (v > best) {
              best = v;
              bi = j;
            }
          }
        }
        warp_argmax_first(best, bi);
        const int qq = __shfl_sync(0xffffffffu, bi, 0);
        best = __shfl_sync(0xffffffffu, best, 0);
        if (!(best > 0.0)) {
          st = p + 1;
          break;  // every warp of both CTAs sees the same row p: all leave together
        }
        int cntp = 0;
#pragma unroll
        for (int c = 0; c < JPL; ++c) {
          const int j = lane + 32 * c;
          cntp += (j < n && !((swept >> c) & 1u) && j > p && j < qq) ? 1 : 0;
        }
        for (int off = 16; off > 0; off >>= 1) cntp += __shfl_xor_sync(0xffffffffu, cntp, off);
        parity += cntp;
        const double a = rowbuf[qq];
        pfv *= a;
        const double ia = 1.0 / a;
        // row q into rowbuf[1]
        const double* srcq = (qq / h == rank ? rows : prow) + static_cast<size_t>(qq - (qq / h) * h) * n;
        for (int j = tid; j < n; j += nt) rowbuf[n + j] = srcq[j];
        cluster.sync();  // both CTAs hold rows p and q: the in-place update may start
        const double* rowp = rowbuf;
        const double* rowq = rowbuf + n;
        double rq[JPL];
#pragma unroll
        for (int c = 0; c < JPL; ++c) {
          const int j = lane + 32 * c;
          rq[c] = j < n ? rowq[j] : 0.0;
        }
        for (int il = warp; il < h; il += nwarp) {
          const int i = r0 + il;
          const double rpi = rowp[i], rqi = rowq[i];
          double* Ci = rows + static_cast<size_t>(il) * n;
#pragma unroll
          for (int c = 0; c < JPL; ++c) {
            const int j = lane + 32 * c;
            if (j >= n) continue;
            double v;
            if (i == p) v = (j == qq) ? -ia : (j == p ? 0.0 : rq[c] * ia);
            else if (i == qq) v = (j == p) ? ia : (j == qq ? 0.0 : -rp[c] * ia);
            else if (j == p) v = -rqi * ia;
            else if (j == qq) v = rpi * ia;
            else v = Ci[j] + (rqi * rp[c] - rpi * rq[c]) * ia;
            Ci[j] = v;
          }
        }
        // mark p, q; the next pivot row is the smallest unswept index
#pragma unroll
        for (int c = 0; c < JPL; ++c) {
          const int j = lane + 32 * c;
          if (j == p || j == qq) swept |= 1u << c;
        }
        int nxt = n;
#pragma unroll
        for (int c = 0; c < JPL; ++c) {
          const int j = lane + 32 * c;
          if (j < n && !((swept >> c) & 1u)) nxt = min(nxt, j);
        }
        for (int off = 16; off > 0; off >>= 1) nxt = min(nxt, __shfl_xor_sync(0xffffffffu, nxt, off));
        p = nxt < n ? nxt : 0;
        cluster.sync();  // the update is complete in both halves
      }
      if (st == 0 && !isfinite((parity & 1) ? -pfv : pfv)) st = -1;
      if (st != 0) {
        bad = true;
        if (tid == 0 && rank == 0) atomicOr(status, kDevSingular);
        break;
      }
      const double pfq = (parity & 1) ? -pfv : pfv;
      if (tid == 0) pf[q] = pfq;
      const double wq = m.qpw[q];
      // transfer terms whose moved electron's row this CTA holds (warp per term)
      for (int t = warp; t < m.nterm; t += nwarp) {
        const int ti = m.tterm[4 * t], tsi = m.tterm[4 * t + 1], tj = m.tterm[4 * t + 2], tsj = m.tterm[4 * t + 3];
        const int dst = ti + tsi * ns, src = tj + tsj * ns;
        if (tsi != tsj || ti == tj || num[dst] == 1 || num[src] == 0 || cfg[src] < 0) continue;
        const int msj = cfg[src] + tsj * ne;
        if (msj / h != rank) continue;
        const double* row = rows + static_cast<size_t>(msj - r0) * n;
        const double* srow = slq + static_cast<size_t>(ti + tsj * ns) * m.ns2;
        double r = 0.0;
        for (int k = lane; k < n; k += 32) {
          const int rk = (k == msj ? ti : idx[k]) + (k >= ne ? ns : 0);
          r += row[k] * __ldg(srow + rk);
        }
        r = warp_sum(r);
        if (lane == 0) tacc[t] += wq * (-r * pfq);
      }
      // adjoint Slater derivative over this CTA's rows
      const int trans = q / m.nleg, spidx = q % m.nleg;
      const int mpidx = trans % m.nmp;
      for (int k = tid; k < n; k += nt) {
        tr[k] = m.trans[mpidx * ns + idx[k]];
        sg[k] = m.trans_sgn[mpidx * ns + idx[k]];
      }
      __syncthreads();
      const double cs = pfq * m.spgl[spidx], cc = pfq * m.spgl[m.nleg + spidx], ss = pfq * m.spgl[2 * m.nleg + spidx];
      for (int k = tid; k < h * n; k += nt) {
        const int il = k / n, j = k - il * n, i = r0 + il;
        const int orb = __ldg(m.orb_idx + tr[i] * ns + tr[j]);
        if (orb < 0 || orb >= m.norb) continue;
        const int sign = sg[i] * sg[j] * __ldg(m.orb_sgn + tr[i] * ns + tr[j]);
        const double first = i < ne ? cs : ss, second = i < ne ? cc : cs;
        const double v = rows[k];
        const double value = j < ne ? v * first : -v * second;
        atomicAdd(oacc + orb, wq * (value * static_cast<double>(sign)));
      }
      cluster.sync();  // both halves are done with this plane before the next gather
    }
    cluster.sync();  // partner's transfer sums and O_k sums are complete
    if (rank == 0) {
      if (tid == 0) {
        double e = 0.0, ip = 0.0;
        bool ok = !bad;
        if (ok) {
          for (int q = 0; q < m.nqp; ++q) ip += m.qpw[q] * pf[q];
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
            e -= m.hund_v[k] *
                 (static_cast<double>(num[i] * num[j]) + static_cast<double>(num[i + ns] * num[j + ns]));
          }
          double transfer = 0.0;
          for (int t = 0; t < m.nterm; ++t) {
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
              z += m.jast_pair[source * ns + dest] * static_cast<double>(chm(source) - chm(dest) + 1);
              const double sum_dest = cj[dest] - m.jast_pair[dest * ns + source] * static_cast<double>(ch(source));
              const double sum_src = cj[source] - m.jast_pair[source * ns + dest] * static_cast<double>(ch(dest));
              z += sum_dest - sum_src;
              // the row of the moved electron was on one CTA: the other's sum is zero
              const double acc = tacc[t] + ptacc[t];
              g = exp(z) * acc / ip;
            }
            transfer -= m.tval[t] * g;
          }
          e += transfer;
          ok = fabs(ip) >= 1.0e-100 && isfinite(e);
        }
        valid[sample] = ok ? 1 : 0;
        eloc[sample] = ok ? e : 0.0;
        double lp = 0.0;
        for (int k = 0; k < m.nproj; ++k) lp += m.proj[k] * static_cast<double>(cnt[k]);
        lpsi[sample] = ok ? lp + log(fabs(ip)) : 0.0;
        dctl[0] = ip;
        ictl[1] = ok ? 1 : 0;
      }
      __syncthreads();
      const bool ok = ictl[1] != 0;
      const double ip = dctl[0];
      const double inv_ip = ip / (ip * ip);
      const double* poacc = oacc_smem ? cluster.map_shared_rank(oacc, 1) : nullptr;
      for (int k = tid; k < m.sr_size; k += nt) {
        double v;
        if (k == 0) v = 1.0;
        else if (k <= m.nproj) v = static_cast<double>(cnt[k - 1]);
        else {
          const int o = k - 1 - m.nproj;
          v = (oacc_smem ? oacc[o] + poacc[o] : oacc[o]) * inv_ip;
        }
        orow[k] = ok ? v : 0.0;
      }
    }
    cluster.sync();  // rank 1's shared memory is read until here
  }
}

template <int JPL>
int launch_cluster_jpl(const DevModel& m, const int* s_idx, const int* s_cfg, const int* s_num, const int* s_cnt,
                       int nsamples, double* scratch, size_t scratch_len, double* ostore, double* eloc, double* lpsi,
                       int* valid, unsigned* status, bool oacc_smem, cudaStream_t stream) {
  const size_t smem = cluster_layout(m, oacc_smem).total;
  auto kernel = k_measure_cluster<JPL>;
  MVMCB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // one cluster per sample up to the co-resident clusters; clusters stride over samples
  const int clusters = std::max(1, std::min(nsamples, sms / 2));
  if (static_cast<size_t>(2 * clusters) * (m.nterm + 1) > scratch_len) return kErrArgument;
  kernel<<<2 * clusters, kClusterThreads, smem, stream>>>(m, s_idx, s_cfg, s_num, s_cnt, nsamples, oacc_smem ? 1 : 0,
                                                          scratch, ostore, eloc, lpsi, valid, status);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

// Whether the two-CTA form applies: planes that do not fit one SM but whose half does
// (n ≤ 256, n even). Returns false when the layout does not fit.
bool cluster_measure_fits(const DevModel& m, int limit) {
  if (m.n > 256 || (m.n & 1)) return false;
  return cluster_layout(m, false).total <= static_cast<size_t>(limit);
}

int launch_measure_cluster(const DevModel& m, const int* s_idx, const int* s_cfg, const int* s_num,
                           const int* s_cnt, int nsamples, double* scratch, size_t scratch_len, double* ostore,
                           double* eloc, double* lpsi, int* valid, unsigned* status, int limit, cudaStream_t stream) {
  const bool oacc_smem = cluster_layout(m, true).total <= static_cast<size_t>(limit);
  const int n = m.n;
#define MVMCB_CLUSTER(J)                                                                                      \
  launch_cluster_jpl<J>(m, s_idx, s_cfg, s_num, s_cnt, nsamples, scratch, scratch_len, ostore, eloc, lpsi, valid, \
                        status, oacc_smem, stream)
  if (n <= 160) return MVMCB_CLUSTER(5);
  if (n <= 224) return MVMCB_CLUSTER(7);
  return MVMCB_CLUSTER(8);
#undef MVMCB_CLUSTER
}

}  // namespace mvmcb
