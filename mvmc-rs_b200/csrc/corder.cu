// C-order parity mode: the measurement, its sums and the SR-CG solve in the operation
// order of the reference's CPU path, without FMA contraction (this file is compiled with
// --fmad=false).
//
// Why a second form: the reference's ten-step zvo_out.dat gate (1e-8 over ten SR steps,
// crates/mvmc-core/tests/phase5_zvo_gate_hubbard.rs:19-80) holds between implementations
// whose arithmetic is identical. The SR-CG of a step (sr_cg.rs:700-880) stops at
// |r|² < tol²·n_active², so its iterate depends on the rounding of every operand and every
// product: reordering the terms of one dot product inside the CG product moves the next
// step's energy by ~1e-7 on the 1D L = 16 chain. The throughput kernels (k_measure with the
// skew Gauss–Jordan sweep, parallel sums, k_sr_cg) are therefore exact only to rounding;
// this form runs every serial chain of operations of the reference on one thread:
//   CalculateMAll per QP plane with pfapack's dsktf2 (UPLO 'U', Parlett–Reid pivoting,
//     rank-2 update (a + x·t1) − y·t2), utu2pfa and the utu2inv pipeline
//     (crates/mvmc-core/src/pfaffian.rs:871-927,1107-1188; crates/pfapack/src/ltl.rs:61-188,
//     667-705; utu2.rs:52-110,399-600; backend.rs:166-330);
//   IP (observables.rs:128), the local energy with the one-electron Pfaffian ratios
//     (observables.rs:483-560,1680-1758,3447-3610; updates.rs:168), the O vector
//     (observables.rs:202, slater_derivative.rs:75-99,289-430) and the per-walker sums
//     (run.rs:2937-3614, observables.rs:297-367);
//   the SR-CG recurrence with its product z = Σ_walkers Σ_samples O_s (O_s·v)
//     (sr_cg.rs:492,700-1009; sr_backend.rs:518-606).
// The projection ratios' exp is the one libm function on this path. Host libms differ in
// its last bit (glibc's exp is not correctly rounded: it differs from the correctly rounded
// value on ~0.1 % of arguments) and one ulp in one local energy already changes the CG
// iteration count of the step, so this mode computes exp by fixed_exp below, a fixed
// sequence of IEEE operations that any host reproduces bit for bit.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "engine.cuh"

namespace mvmcb {
namespace corder {

// ---- exp --------------------------------------------------------------------------------
// Cody–Waite reduction x = k·ln2 + r with ln2 split so that k·ln2_hi is exact (fdlibm's
// split), e^r by its Taylor polynomial of degree 13 in Horner form (|r| ≤ ln2/2: truncation
// below 2^-60), then 2^k applied in two exact power-of-two steps. Every step is one IEEE
// double operation (no contraction), so any host computes the same bits. Accuracy ~1 ulp.
__device__ __forceinline__ double pow2i(int e) {  // 2^e for e in [-1022, 1023]
  return __longlong_as_double(static_cast<long long>(e + 1023) << 52);
}
__device__ double fixed_exp(double x) {
  if (x != x) return x;
  if (x > 709.782712893384) return __longlong_as_double(0x7ff0000000000000LL);
  if (x < -745.1332191019412) return 0.0;
  const double kd = floor(x * 0x1.71547652b82fep+0 + 0.5);
  const int k = static_cast<int>(kd);
  const double r = (x - kd * 0x1.62e42fee00000p-1) - kd * 0x1.a39ef35793c76p-33;
  double p = 0x1.6124613a86d09p-33;
  p = p * r + 0x1.1eed8eff8d898p-29;
  p = p * r + 0x1.ae64567f544e4p-26;
  p = p * r + 0x1.27e4fb7789f5cp-22;
  p = p * r + 0x1.71de3a556c734p-19;
  p = p * r + 0x1.a01a01a01a01ap-16;
  p = p * r + 0x1.a01a01a01a01ap-13;
  p = p * r + 0x1.6c16c16c16c17p-10;
  p = p * r + 0x1.1111111111111p-7;
  p = p * r + 0x1.5555555555555p-5;
  p = p * r + 0x1.5555555555555p-3;
  p = p * r + 0x1.0000000000000p-1;
  p = p * r + 1.0;
  p = p * r + 1.0;
  const int k1 = k / 2, k2 = k - k1;
  return (p * pow2i(k1)) * pow2i(k2);
}

// ---- pfapack (column-major a[i + j·n]) ---------------------------------------------------
__device__ __forceinline__ double& at(double* a, int n, int i, int j) { return a[i + static_cast<size_t>(j) * n]; }

// dsktf2 with UPLO 'U': for k0 = n−1 … 1 the pivot is the first maximum of |A(j, k0)|,
// j ≤ k0 − 1; a zero column records its 1-based row and continues.
__device__ int ltl_upper(double* a, int n, int* piv) {
  int info = 0;
  for (int i = 0; i < n; ++i) piv[i] = i + 1;
  if (n < 2) return 0;
  for (int k0 = n - 1; k0 >= 1; --k0) {
    const int kk0 = k0 - 1;
    int kp = 0;
    double colmax = 0.0;
    for (int j = 0; j <= kk0; ++j) {
      const double v = fabs(at(a, n, j, k0));
      if (j == 0 || v > colmax) {
        colmax = v;
        kp = j;
      }
    }
    if (colmax == 0.0) {
      if (!info) info = kk0 + 1;
      piv[kk0] = kk0 + 1;
      continue;
    }
    if (kp != kk0) {
      for (int j = 0; j < kp; ++j) {
        const double t = at(a, n, j, kk0);
        at(a, n, j, kk0) = at(a, n, j, kp);
        at(a, n, j, kp) = t;
      }
      for (int j = kp + 1; j < kk0; ++j) {
        const double t = at(a, n, j, kk0);
        at(a, n, j, kk0) = at(a, n, kp, j);
        at(a, n, kp, j) = t;
      }
      for (int j = k0; j < n; ++j) {
        const double t = at(a, n, kk0, j);
        at(a, n, kk0, j) = at(a, n, kp, j);
        at(a, n, kp, j) = t;
      }
      for (int j = kp; j < kk0; ++j) at(a, n, j, kk0) = -at(a, n, j, kk0);
      for (int j = kp + 1; j < kk0; ++j) at(a, n, kp, j) = -at(a, n, kp, j);
    }
    piv[kk0] = kp + 1;
    if (kk0 >= 1) {
      const double alpha = 1.0 / at(a, n, kk0, k0);
      for (int j = 0; j < kk0; ++j) {
        const double t1 = alpha * at(a, n, j, kk0);
        const double t2 = alpha * at(a, n, j, k0);
        for (int i = 0; i < j; ++i)
          at(a, n, i, j) = (at(a, n, i, j) + at(a, n, i, k0) * t1) - at(a, n, i, kk0) * t2;
        at(a, n, j, j) = 0.0;
      }
      for (int i = 0; i < kk0; ++i) at(a, n, i, k0) *= alpha;
    }
  }
  return info;
}

// utu2pfa: product of the superdiagonal, sign of the pivot permutation.
__device__ double ltl_pfaffian(double* a, int n, const int* piv) {
  double pf = 1.0;
  for (int i = 0; i + 1 < n; i += 2) pf *= at(a, n, i, i + 1);
  bool neg = false;
  for (int k = 0; k < n; ++k)
    if (piv[k] != k + 1) neg = !neg;
  return (neg ? -1.0 : 1.0) * pf;
}

// utu2inv: M ← I; trtri of the unit upper block; M's superdiagonal part; the
// skew-tridiagonal solve with true divisions; Mᵀ·A and the column permutation (order by
// n > 64, the 64-column panel path); the row permutation.
__device__ void ltl_inverse(double* a, int n, const int* piv, double* m, double* vt) {
  for (size_t k = 0; k < static_cast<size_t>(n) * n; ++k) m[k] = 0.0;
  for (int i = 0; i < n; ++i) at(m, n, i, i) = 1.0;
  const int nb = n - 1;
  for (int j = 1; j < nb; ++j)
    for (int i = 0; i < j; ++i) {
      double acc = at(a, n, i, j + 1);
      for (int k = i + 1; k < j; ++k) acc += at(a, n, i, k + 1) * at(a, n, k, j + 1);
      at(a, n, i, j + 1) = -acc;
    }
  for (int jr = 0; jr < n - 2; ++jr)
    for (int ir = 0; ir <= jr; ++ir) at(m, n, ir, jr + 1) = at(a, n, ir, jr + 2);
  for (int i = 0; i < n - 1; ++i) vt[i] = -at(a, n, i, i + 1);
  for (int j = 0; j < n; ++j) {
    const double* b = m + static_cast<size_t>(j) * n;
    double* c = a + static_cast<size_t>(j) * n;
    c[1] = b[0] / -vt[0];
    for (int i = 2; i < n; i += 2) c[i + 1] = (b[i] - c[i - 1] * vt[i - 1]) / -vt[i];
    c[n - 2] = b[n - 1] / vt[n - 2];
    for (int i = n - 3; i >= 1; i -= 2) c[i - 1] = (b[i] + c[i + 1] * vt[i]) / vt[i - 1];
  }
  auto trmm = [&]() {  // A ← Mᵀ·A, M unit upper
    for (int i = n - 1; i >= 0; --i)
      for (int j = 0; j < n; ++j) {
        double acc = at(a, n, i, j);
        for (int k = 0; k < i; ++k) acc += at(m, n, k, i) * at(a, n, k, j);
        at(a, n, i, j) = acc;
      }
  };
  auto col_perm = [&]() {
    for (int j = 0; j < n; ++j) {
      const int t = piv[j] - 1;
      if (t != j)
        for (int i = 0; i < n; ++i) {
          const double v = at(a, n, i, j);
          at(a, n, i, j) = at(a, n, i, t);
          at(a, n, i, t) = v;
        }
    }
  };
  if (n > 64) {
    trmm();
    for (int j = 0; j < n; ++j) {
      at(a, n, j, j) = 0.0;
      for (int i = j + 1; i < n; ++i) at(a, n, i, j) = -at(a, n, j, i);
    }
    col_perm();
  } else {
    col_perm();
    trmm();
  }
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      const int t = piv[i] - 1;
      if (t != i) {
        const double v = at(a, n, i, j);
        at(a, n, i, j) = at(a, n, t, j);
        at(a, n, t, j) = v;
      }
    }
}

// ---- CalculateMAll, IP, local energy, O vector ------------------------------------------
struct Scratch {
  double* inv;  // [nqp][n·n]: X column-major during the factorisation, then InvM[a·n + b]
  double* m;    // [n·n]
  double* vt;   // [n]
  double* pf;   // [nqp]
  double* qo;   // [nqp][norb]
  double* o;    // [sr_size]
  int* piv;     // [n]
  int* rsj;     // [n]
  int* tr;      // [n]
  int* sg;      // [n]
};

__device__ __forceinline__ int rs_of(const DevModel& m, const int* idx, int k) {
  return idx[k] + (k >= m.ne ? m.ns : 0);
}
__device__ __forceinline__ double slater(const DevModel& m, int q, int r1, int r2) {
  return m.slater[(static_cast<size_t>(q) * m.ns2 + r1) * m.ns2 + r2];
}

// Returns 0, or the failure of the first failing plane (its zero-pivot row, −1 for a
// non-finite Pfaffian, 1000000 + q for an all-zero plane).
__device__ int calc_m_all(const DevModel& m, const int* idx, const Scratch& s) {
  const int n = m.n;
  const size_t nn = static_cast<size_t>(n) * n;
  for (int q = 0; q < m.nqp; ++q) {
    double* x = s.inv + q * nn;
    double maxabs = 0.0;
    for (int msi = 0; msi < n; ++msi)
      for (int msj = 0; msj < n; ++msj) {
        const double v = -slater(m, q, rs_of(m, idx, msi), rs_of(m, idx, msj));
        x[msj + static_cast<size_t>(msi) * n] = v;
        const double v2 = v * v;
        maxabs = maxabs < v2 ? v2 : maxabs;
      }
    if (maxabs < 1e-300) return 1000000 + q;
    const int info = ltl_upper(x, n, s.piv);
    if (info) return info;
    const double p = ltl_pfaffian(x, n, s.piv);
    if (!isfinite(p)) return -1;
    ltl_inverse(x, n, s.piv, s.m, s.vt);
    s.pf[q] = p;
    for (size_t k = 0; k < nn; ++k) x[k] = -x[k];
  }
  return 0;
}

__device__ double local_energy(const DevModel& m, const int* idx, const int* cfg, const int* num,
                               const Scratch& s, double ip) {
  const int ns = m.ns, ne = m.ne, n = m.n;
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
  if (m.nterm == 0 || fabs(ip) <= 0.0) return e;
  double transfer = 0.0;
  for (int t = 0; t < m.nterm; ++t) {
    const int ri = m.tterm[4 * t], s1 = m.tterm[4 * t + 1], rj = m.tterm[4 * t + 2], s2 = m.tterm[4 * t + 3];
    const int dst = ri + s1 * ns, src = rj + s2 * ns;
    double g1;
    if (s1 == s2 && ri == rj) {
      g1 = static_cast<double>(num[src]);
    } else if (s1 != s2 || num[dst] == 1 || num[src] == 0 || cfg[src] < 0) {
      g1 = 0.0;
    } else {
      const int msj = cfg[src] + s2 * ne;
      auto occ = [&](int slot) -> int { return slot == src ? 0 : (slot == dst ? 1 : num[slot]); };
      const int source = rj, dest = ri;
      double z = 0.0;
      z -= m.gutz_site[source] * static_cast<double>(occ(source) + occ(ns + source));
      z += m.gutz_site[dest] * static_cast<double>(occ(dest) * occ(ns + dest));
      z += m.jast_pair[source * ns + dest] *
           static_cast<double>((occ(source) + occ(ns + source) - 1) - (occ(dest) + occ(ns + dest) - 1) + 1);
      for (int site = 0; site < ns; ++site)
        if (site != source && site != dest)
          z += (m.jast_pair[dest * ns + site] - m.jast_pair[source * ns + site]) *
               static_cast<double>(num[site] + num[ns + site] - 1);
      const double proj_ratio = fixed_exp(z);
      for (int k = 0; k < n; ++k) s.rsj[k] = (k == msj ? ri : idx[k]) + (k >= ne ? ns : 0);
      const int rsa = ri + s2 * ns;
      double new_ip = 0.0;
      for (int q = 0; q < m.nqp; ++q) {
        const double* row = s.inv + static_cast<size_t>(q) * n * n + static_cast<size_t>(msj) * n;
        double r = 0.0;
        for (int k = 0; k < n; ++k) r += row[k] * slater(m, q, rsa, s.rsj[k]);
        new_ip += m.qpw[q] * (-r * s.pf[q]);
      }
      g1 = proj_ratio * new_ip / ip;
    }
    transfer -= m.tval[t] * g1;
  }
  return e + transfer;
}

// O = [1, projection counts, Slater derivatives] (real slots).
__device__ void o_vector(const DevModel& m, const int* idx, const int* cnt, const Scratch& s, double ip) {
  const int n = m.n, ne = m.ne, ns = m.ns, nleg = m.nleg, norb = m.norb;
  double* o = s.o;
  o[0] = 1.0;
  for (int k = 0; k < m.nproj; ++k) o[1 + k] = static_cast<double>(cnt[k]);
  for (size_t k = 0; k < static_cast<size_t>(m.nqp) * norb; ++k) s.qo[k] = 0.0;
  for (int q = 0; q < m.nqp; ++q) {
    const int trans = q / nleg, spidx = q % nleg;
    const int mpidx = trans % m.nmp;
    for (int k = 0; k < n; ++k) {
      s.tr[k] = m.trans[mpidx * ns + idx[k]];
      s.sg[k] = m.trans_sgn[mpidx * ns + idx[k]];
    }
    const double p = s.pf[q];
    const double cs = p * m.spgl[spidx], cc = p * m.spgl[nleg + spidx], ss = p * m.spgl[2 * nleg + spidx];
    const double* inv = s.inv + static_cast<size_t>(q) * n * n;
    double* out = s.qo + static_cast<size_t>(q) * norb;
    for (int msi = 0; msi < n; ++msi) {
      const double first = msi < ne ? cs : ss, second = msi < ne ? cc : cs;
      for (int msj = 0; msj < n; ++msj) {
        const int orb = m.orb_idx[s.tr[msi] * ns + s.tr[msj]];
        if (orb < 0 || orb >= norb) continue;
        const int sign = s.sg[msi] * s.sg[msj] * m.orb_sgn[s.tr[msi] * ns + s.tr[msj]];
        const double v = inv[msi * n + msj];
        const double value = msj < ne ? v * first : -v * second;
        out[orb] += value * static_cast<double>(sign);
      }
    }
  }
  const double inv_ip = ip / (ip * ip);
  for (int k = 0; k < norb; ++k) {
    double acc = 0.0;
    for (int q = 0; q < m.nqp; ++q) acc += m.qpw[q] * s.qo[static_cast<size_t>(q) * norb + k];
    o[1 + m.nproj + k] = acc * inv_ip;
  }
}

// One thread per walker: its saved samples in order, their O rows in the store and the
// walker's sums [Wc, E, E², Sz, Sz², HO(size), ⟨O⟩ sum(size), ⟨O²⟩ sum(size)].
__global__ void k_measure_corder(DevModel m, int W, int S, const int* __restrict__ s_idx,
                                 const int* __restrict__ s_cfg, const int* __restrict__ s_num,
                                 const int* __restrict__ s_cnt, double* __restrict__ ostore,
                                 double* __restrict__ eloc, double* __restrict__ lpsi, int* __restrict__ valid,
                                 double* __restrict__ wsum, double* __restrict__ dscr, int* __restrict__ iscr,
                                 long long dstride, long long istride) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  const int n = m.n, size = m.sr_size;
  const size_t nn = static_cast<size_t>(n) * n;
  Scratch s;
  s.inv = dscr + w * dstride;
  s.m = s.inv + m.nqp * nn;
  s.vt = s.m + nn;
  s.pf = s.vt + n;
  s.qo = s.pf + m.nqp;
  s.o = s.qo + static_cast<size_t>(m.nqp) * m.norb;
  s.piv = iscr + w * istride;
  s.rsj = s.piv + n;
  s.tr = s.rsj + n;
  s.sg = s.tr + n;
  double* out = wsum + static_cast<size_t>(w) * (5 + 3 * size);
  double wc = 0.0, e1 = 0.0, e2 = 0.0, z1 = 0.0, z2 = 0.0;
  double* ho = out + 5;
  for (int i = 0; i < size; ++i) ho[i] = 0.0;
  for (int smp_i = 0; smp_i < S; ++smp_i) {
    const size_t smp = static_cast<size_t>(w) * S + smp_i;
    const int* idx = s_idx + smp * n;
    const int* cfg = s_cfg + smp * m.ns2;
    const int* num = s_num + smp * m.ns2;
    const int* cnt = s_cnt + smp * m.nproj;
    double* st = ostore + smp * size;
    for (int i = 0; i < size; ++i) st[i] = 0.0;
    valid[smp] = 0;
    eloc[smp] = 0.0;
    lpsi[smp] = 0.0;
    bool all_zero = true, all_neg = true;
    for (int k = 0; k < n; ++k) {
      all_zero = all_zero && idx[k] == 0;
      all_neg = all_neg && idx[k] < 0;
    }
    if (all_zero || all_neg) continue;
    if (calc_m_all(m, idx, s) != 0) continue;
    double ip = 0.0;
    for (int q = 0; q < m.nqp; ++q) ip += m.qpw[q] * s.pf[q];
    if (fabs(ip) < 1.0e-100) continue;
    const double e = local_energy(m, idx, cfg, num, s, ip);
    if (!isfinite(e)) continue;
    double sz = 0.0;
    for (int r = 0; r < m.ns; ++r) sz += static_cast<double>(num[r] - num[r + m.ns]);
    wc += 1.0;
    e1 += 1.0 * e;
    e2 += (1.0 * e) * e;
    z1 += 1.0 * sz;
    z2 += 1.0 * sz * sz;
    o_vector(m, idx, cnt, s, ip);
    for (int i = 0; i < size; ++i) {
      st[i] = 1.0 * s.o[i];
      ho[i] += (1.0 * e) * s.o[i];
    }
    valid[smp] = 1;
    eloc[smp] = e;
    double lp = 0.0;
    for (int k = 0; k < m.nproj; ++k) lp += m.proj[k] * static_cast<double>(cnt[k]);
    lpsi[smp] = lp + log(fabs(ip));
  }
  out[0] = wc;
  out[1] = e1;
  out[2] = e2;
  out[3] = z1;
  out[4] = z2;
  for (int i = 0; i < size; ++i) {  // finalize_oo_store_real, diagonal only
    double mean = 0.0, diag = 0.0;
    for (int smp_i = 0; smp_i < S; ++smp_i) {
      const double v = ostore[(static_cast<size_t>(w) * S + smp_i) * size + i];
      mean += v;
      diag += v * v;
    }
    out[5 + size + i] = mean;
    out[5 + 2 * size + i] = diag;
  }
}

// ---- SR-CG ------------------------------------------------------------------------------
constexpr int kCgThreads = 256;

struct CgState {
  double delta;
  double coef;
  int action;  // 0 continue, 1 stop
};

// z = S·v = Wc⁻¹·Σ_w Σ_s O_s (O_s·v) − (⟨O⟩·v)⟨O⟩ + shift·diag ⊙ v (SampledSrOperator::apply,
// sr_cg.rs:952-1009): y_s by one thread each (serial over components), the walker partials
// zl by one thread per component (serial over the walker's samples, walkers in order).
__device__ void apply(const double* __restrict__ O, int W, int S, int na, const double* mean, const double* diag,
                      double inv_w, double shift, const double* v, double* z, double* y, CgState& sh) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const long long ns = static_cast<long long>(W) * S;
  for (long long s = tid; s < ns; s += nt) {
    double acc = 0.0;
    const double* row = O + s * na;
    for (int i = 0; i < na; ++i) acc += row[i] * v[i];
    y[s] = acc;
  }
  __syncthreads();
  for (int i = tid; i < na; i += nt) {
    double zi = 0.0;
    for (int w = 0; w < W; ++w) {
      double zl = 0.0;
      for (int k = 0; k < S; ++k) {
        const long long s = static_cast<long long>(w) * S + k;
        zl += O[s * na + i] * y[s];
      }
      zi += zl;
    }
    z[i] = zi;
  }
  if (tid == 0) {
    double c = 0.0;
    for (int i = 0; i < na; ++i) c += mean[i] * v[i];
    sh.coef = c;
  }
  __syncthreads();
  const double coef = sh.coef;
  for (int i = tid; i < na; i += nt) z[i] = inv_w * z[i] - coef * mean[i] + shift * diag[i] * v[i];
  __syncthreads();
}

__device__ __forceinline__ double sdot(const double* p, const double* q, int n) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += p[i] * q[i];
  return s;
}

__device__ __forceinline__ double precond(double pfac, double diag, double r) {
  double dq = pfac * diag;
  if (!isfinite(dq) || fabs(dq) < 1e-12) dq = dq < 0.0 ? -1e-12 : 1e-12;
  return r / dq;
}

// The CG solve (solve_with_product, sr_cg.rs:700-880) on one CTA: thread 0 runs the scalar
// recurrence (sequential dots, α, β, the stop and failure rules), every thread the
// elementwise updates. scal receives {δ, status, iterations}.
__global__ void __launch_bounds__(kCgThreads)
    k_cg_corder(const double* __restrict__ O, int W, int S, int na, const double* __restrict__ mean,
                const double* __restrict__ diag, const double* __restrict__ g, double inv_w, double shift,
                double tol, int max_iter, int diag_scale, double* x, double* r, double* d, double* q, double* y,
                double* scal) {
  __shared__ CgState sh;
  __shared__ long long status;
  const int tid = threadIdx.x, nt = blockDim.x, n = na;
  const double threshold = tol * tol * static_cast<double>(n) * static_cast<double>(n);
  const double pfac = 1.0 + shift;
  for (int i = tid; i < n; i += nt) {
    x[i] = 0.0;
    r[i] = g[i];
    q[i] = 0.0;
  }
  __syncthreads();
  if (diag_scale) {
    apply(O, W, S, na, mean, diag, inv_w, shift, x, r, y, sh);
    for (int i = tid; i < n; i += nt) {
      r[i] = g[i] - r[i];
      d[i] = precond(pfac, diag[i], r[i]);
    }
    __syncthreads();
    if (tid == 0) sh.delta = sdot(r, d, n);
  } else {
    for (int i = tid; i < n; i += nt) d[i] = g[i];
    __syncthreads();
    if (tid == 0) sh.delta = sdot(r, r, n);
  }
  if (tid == 0) {
    status = 0;
    sh.action = 0;
    if (!isfinite(sh.delta)) {
      status = -1;
      sh.action = 1;
    }
  }
  __syncthreads();
  int iter = 0;
  while (sh.action == 0 && iter < max_iter) {
    __syncthreads();  // every thread has read the flag before thread 0 writes it again
    if (tid == 0) {
      const long long failed = -(static_cast<long long>(iter) + 1);
      if (!isfinite(sh.delta)) {
        status = failed;
        sh.action = 1;
      } else if (fabs(sh.delta) < threshold) {
        sh.action = 2;  // converged
      }
    }
    __syncthreads();
    if (sh.action != 0) break;
    apply(O, W, S, na, mean, diag, inv_w, shift, d, q, y, sh);
    __shared__ double alpha;
    if (tid == 0) {
      const long long failed = -(static_cast<long long>(iter) + 1);
      const double dq = sdot(d, q, n);
      if (!isfinite(dq) || fabs(dq) < 1e-20) {
        status = failed;
        sh.action = 1;
      } else {
        alpha = sh.delta / dq;
        if (!isfinite(alpha)) {
          status = failed;
          sh.action = 1;
        }
      }
    }
    __syncthreads();
    if (sh.action != 0) break;
    const double a = alpha;
    for (int i = tid; i < n; i += nt) x[i] += a * d[i];
    __syncthreads();
    if ((iter + 1) % 20 == 0) {
      apply(O, W, S, na, mean, diag, inv_w, shift, x, r, y, sh);
      for (int i = tid; i < n; i += nt) r[i] = g[i] - r[i];
    } else {
      for (int i = tid; i < n; i += nt) r[i] -= a * q[i];
    }
    __syncthreads();
    if (diag_scale) {
      for (int i = tid; i < n; i += nt) q[i] = precond(pfac, diag[i], r[i]);
      __syncthreads();
    }
    __shared__ double beta;
    if (tid == 0) {
      const long long failed = -(static_cast<long long>(iter) + 1);
      const double delta_new = diag_scale ? sdot(r, q, n) : sdot(r, r, n);
      if (!isfinite(delta_new) || fabs(sh.delta) < 1e-20) {
        status = failed;
        sh.action = 1;
      } else {
        beta = delta_new / sh.delta;
        if (!isfinite(beta)) {
          status = failed;
          sh.action = 1;
        } else if (diag_scale) {
          sh.delta = delta_new;
        } else {
          sh.delta *= beta;
        }
      }
    }
    __syncthreads();
    if (sh.action != 0) break;
    const double b = beta;
    if (diag_scale)
      for (int i = tid; i < n; i += nt) d[i] = q[i] + b * d[i];
    else
      for (int i = tid; i < n; i += nt) d[i] = r[i] + b * d[i];
    ++iter;
    __syncthreads();
  }
  if (tid == 0) {
    if (sh.action != 1) {
      if (iter == max_iter && fabs(sh.delta) >= threshold)
        status = -(static_cast<long long>(max_iter) + 1);
      else
        status = iter;
    }
    scal[0] = sh.delta;
    scal[1] = static_cast<double>(status);
    scal[2] = static_cast<double>(iter);
  }
}

}  // namespace corder

// Scratch per walker of k_measure_corder, in doubles and ints.
void corder_scratch_sizes(const DevModel& m, long long* dstride, long long* istride) {
  const long long nn = static_cast<long long>(m.n) * m.n;
  *dstride = m.nqp * nn + nn + m.n + m.nqp + static_cast<long long>(m.nqp) * m.norb + m.sr_size;
  *dstride = (*dstride + 31) & ~31LL;
  *istride = (4LL * m.n + 31) & ~31LL;
}

int launch_measure_corder(const DevModel& m, int W, int S, const int* s_idx, const int* s_cfg, const int* s_num,
                          const int* s_cnt, double* ostore, double* eloc, double* lpsi, int* valid, double* wsum,
                          double* dscr, int* iscr, cudaStream_t stream) {
  long long ds = 0, is = 0;
  corder_scratch_sizes(m, &ds, &is);
  constexpr int kThreads = 32;
  corder::k_measure_corder<<<(W + kThreads - 1) / kThreads, kThreads, 0, stream>>>(
      m, W, S, s_idx, s_cfg, s_num, s_cnt, ostore, eloc, lpsi, valid, wsum, dscr, iscr, ds, is);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

int launch_cg_corder(const CgArgs& a, int W, int S, cudaStream_t stream) {
  if (static_cast<long long>(W) * S != a.ns) return kErrArgument;
  corder::k_cg_corder<<<1, corder::kCgThreads, 0, stream>>>(a.O, W, S, a.na, a.mean, a.diag, a.g, a.inv_w, a.shift,
                                                              a.tol, a.max_iter, a.diag_scale, a.x, a.r, a.d, a.q,
                                                              a.y, a.scal);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

}  // namespace mvmcb
