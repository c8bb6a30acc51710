// Oracle: CPU restatement of the real, sz-conserved VMC sampling + SR-CG path of
// AtelierArith/mvmc-rs, in the reference's operation order (FP64, no FMA contraction).
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA product. Only tests/,
// __graft_entry__.smoke() and bench.py's CPU baseline legs load it.
//
// Each function cites the reference file:line it restates (paths inside mvmc-rs).
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../mvmc-rs_b200/host/expert.h"

namespace orc {

using mvmc::Model;

// ===================================================================================
// SFMT19937 (crates/sfmt19937/src/{lib,state,init,real}.rs; MEXP 19937, POS1 122,
// SL1 18, SL2 1 byte, SR1 11, SR2 1 byte, little-endian 128-bit lanes)
// ===================================================================================
struct Sfmt {
  static constexpr int N = 156, N32 = 624, POS1 = 122;
  uint32_t w[N32];
  int idx = N32;
  uint64_t draws = 0;

  void seed(uint32_t s) {
    w[0] = s;
    for (int i = 1; i < N32; ++i) w[i] = 1812433253u * (w[i - 1] ^ (w[i - 1] >> 30)) + static_cast<uint32_t>(i);
    idx = N32;
    draws = 0;
    certify();
  }
  void certify() {
    static const uint32_t parity[4] = {0x00000001u, 0x00000000u, 0x00000000u, 0x13c9e684u};
    uint32_t inner = 0;
    for (int i = 0; i < 4; ++i) inner ^= w[i] & parity[i];
    for (int i = 16; i > 0; i >>= 1) inner ^= inner >> i;
    if (inner & 1u) return;
    for (int i = 0; i < 4; ++i) {
      uint32_t work = 1;
      for (int j = 0; j < 32; ++j) {
        if (work & parity[i]) {
          w[i] ^= work;
          return;
        }
        work <<= 1;
      }
    }
  }
  static void recursion(uint32_t* r, const uint32_t* a, const uint32_t* b, const uint32_t* c,
                        const uint32_t* d) {
    static const uint32_t msk[4] = {0xdfffffefu, 0xddfecb7fu, 0xbffaffffu, 0xbffffff6u};
    const uint64_t ah = (static_cast<uint64_t>(a[3]) << 32) | a[2];
    const uint64_t al = (static_cast<uint64_t>(a[1]) << 32) | a[0];
    const uint64_t xh = (ah << 8) | (al >> 56), xl = al << 8;
    const uint64_t ch = (static_cast<uint64_t>(c[3]) << 32) | c[2];
    const uint64_t cl = (static_cast<uint64_t>(c[1]) << 32) | c[0];
    const uint64_t yh = ch >> 8, yl = (cl >> 8) | (ch << 56);
    const uint32_t x[4] = {static_cast<uint32_t>(xl), static_cast<uint32_t>(xl >> 32),
                           static_cast<uint32_t>(xh), static_cast<uint32_t>(xh >> 32)};
    const uint32_t y[4] = {static_cast<uint32_t>(yl), static_cast<uint32_t>(yl >> 32),
                           static_cast<uint32_t>(yh), static_cast<uint32_t>(yh >> 32)};
    for (int k = 0; k < 4; ++k) r[k] = a[k] ^ x[k] ^ ((b[k] >> 11) & msk[k]) ^ y[k] ^ (d[k] << 18);
  }
  void gen_all() {
    uint32_t* s = w;
    const uint32_t* r1 = s + 4 * (N - 2);
    const uint32_t* r2 = s + 4 * (N - 1);
    int i = 0;
    for (; i < N - POS1; ++i) {
      uint32_t out[4];
      recursion(out, s + 4 * i, s + 4 * (i + POS1), r1, r2);
      std::memcpy(s + 4 * i, out, sizeof out);
      r1 = r2;
      r2 = s + 4 * i;
    }
    for (; i < N; ++i) {
      uint32_t out[4];
      recursion(out, s + 4 * i, s + 4 * (i + POS1 - N), r1, r2);
      std::memcpy(s + 4 * i, out, sizeof out);
      r1 = r2;
      r2 = s + 4 * i;
    }
  }
  uint32_t u32() {
    if (idx >= N32) {
      gen_all();
      idx = 0;
    }
    ++draws;
    return w[idx++];
  }
  double real2() { return static_cast<double>(u32()) * (1.0 / 4294967296.0); }
  uint32_t mod(uint32_t n) { return u32() % n; }  // C `gen_rand32() % n`
  void peek(uint32_t* out, int n) const {         // non-destructive dump
    Sfmt copy = *this;
    for (int k = 0; k < n; ++k) out[k] = copy.u32();
  }
};

// ===================================================================================
// pfapack: skew LTL^T (dsktf2, UPLO='U'), Pfaffian and the 8-step inverse
// (crates/pfapack/src/ltl.rs:61-188,667-705; utu2.rs:52-110,399-600; backend.rs:166-330)
// Matrices are column-major a[i + j*n].
// ===================================================================================
#define A_(i, j) a[(i) + static_cast<size_t>(j) * n]

template <typename R>
int ltl_upper(R* a, int n, int* piv) {
  int info = 0;
  for (int i = 0; i < n; ++i) piv[i] = i + 1;
  if (n < 2) return 0;
  for (int k0 = n - 1; k0 >= 1; --k0) {
    const int kk0 = k0 - 1;
    int kp = 0;
    R colmax = 0.0;
    for (int j = 0; j <= kk0; ++j) {
      const R v = std::fabs(A_(j, k0));
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
      for (int j = 0; j < kp; ++j) std::swap(A_(j, kk0), A_(j, kp));
      for (int j = kp + 1; j < kk0; ++j) std::swap(A_(j, kk0), A_(kp, j));
      for (int j = k0; j < n; ++j) std::swap(A_(kk0, j), A_(kp, j));
      for (int j = kp; j < kk0; ++j) A_(j, kk0) = -A_(j, kk0);
      for (int j = kp + 1; j < kk0; ++j) A_(kp, j) = -A_(kp, j);
    }
    piv[kk0] = kp + 1;
    if (kk0 >= 1) {
      const R alpha = 1.0 / A_(kk0, k0);
      for (int j = 0; j < kk0; ++j) {
        const R t1 = alpha * A_(j, kk0);
        const R t2 = alpha * A_(j, k0);
        for (int i = 0; i < j; ++i) A_(i, j) = (A_(i, j) + A_(i, k0) * t1) - A_(i, kk0) * t2;
        A_(j, j) = 0.0;
      }
      for (int i = 0; i < kk0; ++i) A_(i, k0) *= alpha;
    }
  }
  return info;
}

template <typename R>
R ltl_pfaffian(const R* a, int n, const int* piv) {
  R pf = 1.0;
  for (int i = 0; i + 1 < n; i += 2) pf *= A_(i, i + 1);
  bool neg = false;
  for (int k = 0; k < n; ++k)
    if (piv[k] != k + 1) neg = !neg;
  return (neg ? -1.0 : 1.0) * pf;
}

template <typename R>
void ltl_inverse(R* a, int n, const int* piv, std::vector<R>& mw, std::vector<R>& vt) {
  mw.assign(static_cast<size_t>(n) * n, 0.0);
  vt.assign(n > 1 ? n - 1 : 1, 0.0);
  R* m = mw.data();
#define M_(i, j) m[(i) + static_cast<size_t>(j) * n]
  for (int i = 0; i < n; ++i) M_(i, i) = 1.0;
  // trtri of the unit upper block B(i, j) = A(i, j + 1), size n - 1.
  const int nb = n - 1;
  for (int j = 1; j < nb; ++j)
    for (int i = 0; i < j; ++i) {
      R acc = A_(i, j + 1);
      for (int k = i + 1; k < j; ++k) acc += A_(i, k + 1) * A_(k, j + 1);
      A_(i, j + 1) = -acc;
    }
  for (int jr = 0; jr < n - 2; ++jr)
    for (int ir = 0; ir <= jr; ++ir) M_(ir, jr + 1) = A_(ir, jr + 2);
  for (int i = 0; i < n - 1; ++i) vt[i] = -A_(i, i + 1);
  // skew-tridiagonal solve, direct divisions, output into A.
  for (int j = 0; j < n; ++j) {
    const R* b = m + static_cast<size_t>(j) * n;
    R* c = a + static_cast<size_t>(j) * n;
    c[1] = b[0] / -vt[0];
    for (int i = 2; i < n; i += 2) c[i + 1] = (b[i] - c[i - 1] * vt[i - 1]) / -vt[i];
    c[n - 2] = b[n - 1] / vt[n - 2];
    for (int i = n - 3; i >= 1; i -= 2) c[i - 1] = (b[i] + c[i + 1] * vt[i]) / vt[i - 1];
  }
  auto trmm = [&]() {  // A <- M^T A, M unit upper
    for (int i = n - 1; i >= 0; --i)
      for (int j = 0; j < n; ++j) {
        R acc = A_(i, j);
        for (int k = 0; k < i; ++k) acc += M_(k, i) * A_(k, j);
        A_(i, j) = acc;
      }
  };
  auto col_perm = [&]() {
    for (int j = 0; j < n; ++j) {
      const int t = piv[j] - 1;
      if (t != j)
        for (int i = 0; i < n; ++i) std::swap(A_(i, j), A_(i, t));
    }
  };
  if (n > 64) {
    trmm();
    for (int j = 0; j < n; ++j) {
      A_(j, j) = 0.0;
      for (int i = j + 1; i < n; ++i) A_(i, j) = -A_(j, i);
    }
    col_perm();
  } else {
    col_perm();
    trmm();
  }
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      const int t = piv[i] - 1;
      if (t != i) std::swap(A_(i, j), A_(t, j));
    }
#undef M_
}
#undef A_

// In place: column-major X -> X^-1; returns 0 ok, >0 zero-pivot row, -1 non-finite Pf.
template <typename R>
int pfinv(R* a, int n, R* pf) {
  std::vector<int> piv(n);
  std::vector<R> mw, vt;
  const int info = ltl_upper(a, n, piv.data());
  if (info) return info;
  const R p = ltl_pfaffian(a, n, piv.data());
  if (!std::isfinite(p)) return -1;
  *pf = p;
  ltl_inverse(a, n, piv.data(), mw, vt);
  return 0;
}

// ===================================================================================
// Walker state and CalculateMAll (crates/mvmc-core/src/pfaffian.rs:871-927,1107-1188)
// inv[q][a*n + b] = (X_q^-1)(a, b), X_q(a, b) = SlaterElm[q][rs_a][rs_b].
// ===================================================================================
struct Walker {
  Sfmt rng;
  std::vector<int64_t> ele_idx, ele_cfg, ele_num, proj_cnt;
  std::vector<int64_t> b_idx, b_cfg, b_num, b_cnt;
  bool burn = false;
  std::vector<double> inv, pf;
  std::vector<int64_t> s_idx, s_cfg, s_num, s_cnt;  // saved samples
  int64_t counter[6] = {0, 0, 0, 0, 0, 0};
};

struct Ctx {
  const Model& m;
  const std::vector<double>& slater;  // [nqp][2Ns][2Ns]
  int ns, ne, n, ns2, nqp, nproj;
  std::vector<double> proj;       // G then J parameter values
  std::vector<double> gutz_site;  // direct projection tables
  std::vector<double> jast_pair;
  Ctx(const Model& model, const std::vector<double>& s)
      : m(model), slater(s), ns(model.nsite), ne(model.ne), n(2 * model.ne), ns2(2 * model.nsite),
        nqp(model.nqp), nproj(model.nproj()) {
    proj = model.gutz;
    proj.insert(proj.end(), model.jast.begin(), model.jast.end());
    gutz_site.assign(ns, 0.0);
    for (int r = 0; r < ns; ++r) {
      const int g = model.gutz_idx[r];
      if (model.n_gutz > 0 && g >= 0 && g < model.n_gutz) gutz_site[r] = model.gutz[g];
    }
    jast_pair.assign(static_cast<size_t>(ns) * ns, 0.0);
    for (int a = 0; a < ns; ++a)
      for (int b = 0; b < ns; ++b) {
        if (a == b || model.n_jast == 0) continue;
        const int j = model.jast_idx[std::min(a, b) * ns + std::max(a, b)];
        if (j >= 0 && j < model.n_jast) jast_pair[a * ns + b] = model.jast[j];
      }
  }
  double S(int q, int r1, int r2) const {
    return slater[(static_cast<size_t>(q) * ns2 + r1) * ns2 + r2];
  }
  int rs(const int64_t* idx, int msi) const {
    return static_cast<int>(idx[msi]) + (msi >= ne ? ns : 0);
  }
};

// Returns 0 ok; otherwise the plane's failure (pf/inv of later planes untouched).
template <typename R>
int calc_m_all(const Ctx& c, const int64_t* ele_idx, R* inv, R* pf) {
  const int n = c.n;
  std::vector<R> x(static_cast<size_t>(n) * n);
  for (int q = 0; q < c.nqp; ++q) {
    R maxabs = 0.0;
    for (int msi = 0; msi < n; ++msi)
      for (int msj = 0; msj < n; ++msj) {
        const R v = -c.S(q, c.rs(ele_idx, msi), c.rs(ele_idx, msj));
        x[msj + static_cast<size_t>(msi) * n] = v;
        maxabs = std::max(maxabs, v * v);
      }
    if (maxabs < 1e-300) return 1000000 + q;
    R p = 0.0;
    const int st = pfinv(x.data(), n, &p);
    if (st) return st;
    pf[q] = p;
    R* dst = inv + static_cast<size_t>(q) * n * n;
    for (size_t k = 0; k < x.size(); ++k) dst[k] = -x[k];
  }
  return 0;
}

template <typename R>
R ip_of(const Ctx& c, const R* pf) {  // calculate_ip_real (observables.rs:128)
  R ip = 0.0;
  for (int q = 0; q < c.nqp; ++q) ip += c.m.qp_weight[q] * pf[q];
  return ip;
}

// ===================================================================================
// Projection counters (sampling/projection.rs:170-470)
// ===================================================================================
void make_proj_cnt(const Ctx& c, const int64_t* num, int64_t* cnt) {
  const int ns = c.ns;
  for (int k = 0; k < c.nproj; ++k) cnt[k] = 0;
  for (int ri = 0; ri < ns; ++ri) {
    const int g = c.m.gutz_idx[ri];
    if (c.m.n_gutz > 0 && g >= 0 && g < c.nproj) cnt[g] += num[ri] * num[ri + ns];
  }
  if (c.m.n_jast > 0)
    for (int ri = 0; ri < ns; ++ri) {
      const int64_t xi = num[ri] + num[ri + ns] - 1;
      if (xi == 0) continue;
      for (int rj = ri + 1; rj < ns; ++rj) {
        const int j = c.m.jast_idx[ri * ns + rj];
        if (j < 0) continue;
        const int64_t xj = num[rj] + num[rj + ns] - 1;
        if (c.m.n_gutz + j < c.nproj) cnt[c.m.n_gutz + j] += xi * xj;
      }
    }
}

void update_proj_cnt(const Ctx& c, int ri, int rj, int64_t* cnew, const int64_t* cold,
                     const int64_t* num) {
  const int ns = c.ns;
  if (cnew != cold)
    for (int k = 0; k < c.nproj; ++k) cnew[k] = cold[k];
  if (ri == rj) return;
  if (c.m.n_gutz > 0) {
    const int gi = c.m.gutz_idx[ri], gj = c.m.gutz_idx[rj];
    if (gi >= 0 && gi < c.nproj) cnew[gi] -= num[ri] + num[ri + ns];
    if (gj >= 0 && gj < c.nproj) cnew[gj] += num[rj] * num[rj + ns];
  }
  if (c.m.n_jast > 0) {
    auto jidx = [&](int a, int b) { return c.m.jast_idx[std::min(a, b) * ns + std::max(a, b)]; };
    const int64_t xri = num[ri] + num[ri + ns], xrj = num[rj] + num[rj + ns];
    const int off = c.m.n_gutz;
    const int ij = jidx(ri, rj);
    if (ij >= 0) cnew[off + ij] += xri - xrj + 1;
    for (int rk = 0; rk < ns; ++rk) {
      if (rk == ri || rk == rj) continue;
      const int64_t xk = num[rk] + num[rk + ns] - 1;
      const int ik = jidx(ri, rk), jk = jidx(rj, rk);
      if (ik >= 0) cnew[off + ik] -= xk;
      if (jk >= 0) cnew[off + jk] += xk;
    }
  }
}

double log_proj_ratio(const Ctx& c, const int64_t* cnew, const int64_t* cold) {
  double z = 0.0;
  for (int k = 0; k < c.nproj; ++k) z += c.proj[k] * static_cast<double>(cnew[k] - cold[k]);
  return z;
}

void update_ele_config(const Ctx& c, int mi, int ri, int rj, int s, int64_t* idx, int64_t* cfg,
                       int64_t* num) {
  const int msa = mi + s * c.ne, ro = ri + s * c.ns, rn = rj + s * c.ns;
  idx[msa] = rj;
  cfg[ro] = -1;
  cfg[rn] = mi;
  num[ro] = 0;
  num[rn] = 1;
}
void revert_ele_config(const Ctx& c, int mi, int ri, int rj, int s, int64_t* idx, int64_t* cfg,
                       int64_t* num) {
  const int msa = mi + s * c.ne, ro = ri + s * c.ns, rn = rj + s * c.ns;
  idx[msa] = ri;
  cfg[ro] = mi;
  cfg[rn] = -1;
  num[ro] = 1;
  num[rn] = 0;
}

// ===================================================================================
// Ratios and rank-2 / rank-4 updates (sampling/updates.rs:73-160,395-444,588-640,
// 779-835,984-1086,1154-1215,1429-1505,1539-1622)
// ===================================================================================
template <typename R>
void ratio_hop(const Ctx& c, int msa, const int64_t* idx, const R* inv, const R* pf,
               R* pf_new) {
  const int n = c.n;
  const int rsa = c.rs(idx, msa);
  for (int q = 0; q < c.nqp; ++q) {
    const R* row = inv + static_cast<size_t>(q) * n * n + static_cast<size_t>(msa) * n;
    R r = 0.0;
    for (int j = 0; j < n; ++j) r += row[j] * c.S(q, rsa, c.rs(idx, j));
    pf_new[q] = -r * pf[q];
  }
}

template <typename R>
void update_hop(const Ctx& c, int msa, const int64_t* idx, R* inv, R* pf) {
  const int n = c.n;
  const int rsa = c.rs(idx, msa);
  std::vector<R> slt(n), v1(n), v2(n);
  for (int q = 0; q < c.nqp; ++q) {
    R* m = inv + static_cast<size_t>(q) * n * n;
    for (int j = 0; j < n; ++j) slt[j] = c.S(q, rsa, c.rs(idx, j));
    std::fill(v1.begin(), v1.end(), 0.0);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) v1[j] += -m[i * n + j] * slt[i];
    const R tmp = v1[msa];
    pf[q] *= -tmp;
    const R inv_a = -1.0 / tmp;
    for (int j = 0; j < n; ++j) v2[j] = m[msa * n + j] * inv_a;
    for (int i = 0; i < n; ++i) {
      for (int j = 0; j < n; ++j) m[i * n + j] += v1[i] * v2[j] - v1[j] * v2[i];
      m[i * n + msa] -= v2[i];
    }
    for (int j = 0; j < n; ++j) m[msa * n + j] += v2[j];
  }
}

template <typename R>
void ratio_exchange(const Ctx& c, int msa, int msb, const int64_t* idx, const R* inv,
                    const R* pf, R* pf_new) {
  const int n = c.n;
  const int rsa = c.rs(idx, msa), rsb = c.rs(idx, msb);
  std::vector<R> va(n), vb(n);
  for (int q = 0; q < c.nqp; ++q) {
    const R* m = inv + static_cast<size_t>(q) * n * n;
    for (int i = 0; i < n; ++i) {
      va[i] = c.S(q, rsa, c.rs(idx, i));
      vb[i] = c.S(q, rsb, c.rs(idx, i));
    }
    const R vba = vb[msa];
    R pa = 0, pb = 0, qa = 0, qb = 0;
    for (int i = 0; i < n; ++i) {
      pa += m[msa * n + i] * va[i];
      pb += m[msb * n + i] * va[i];
      qa += m[msa * n + i] * vb[i];
      qb += m[msb * n + i] * vb[i];
    }
    const R iab = m[msa * n + msb];
    R bma = 0.0;
    for (int i = 0; i < n; ++i) {
      R t = 0.0;
      for (int j = 0; j < n; ++j) t += m[i * n + j] * va[j];
      bma += vb[i] * t;
    }
    const R ratio = iab * vba + iab * bma + pa * qb - pb * qa;
    pf_new[q] = ratio * pf[q];
  }
}

template <typename R>
void update_exchange(const Ctx& c, int msa, int msb, int ra_old, int rb_old, int sa, int sb,
                     const int64_t* idx, R* inv, R* pf) {
  const int n = c.n;
  const int rsa = c.rs(idx, msa), rsb = c.rs(idx, msb);
  const int rsa_old = ra_old + sa * c.ns, rsb_old = rb_old + sb * c.ns;
  std::vector<R> vs(n), vt(n), vp(n), vq(n);
  for (int qp = 0; qp < c.nqp; ++qp) {
    R* m = inv + static_cast<size_t>(qp) * n * n;
    const R m_old_ab = c.S(qp, rsa_old, rsb_old);
    for (int i = 0; i < n; ++i) {
      vs[i] = c.S(qp, rsa, c.rs(idx, i));
      vt[i] = c.S(qp, rsb, c.rs(idx, i));
    }
    vs[msb] = m_old_ab;
    std::fill(vp.begin(), vp.end(), 0.0);
    std::fill(vq.begin(), vq.end(), 0.0);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        vp[i] += m[i * n + j] * vs[j];
        vq[i] += m[i * n + j] * vt[j];
      }
    R bma = 0.0;
    for (int i = 0; i < n; ++i) bma += vt[i] * vp[i];
    const R iab = m[msa * n + msb];
    const R ratio = iab * vt[msa] + iab * bma + vp[msa] * vq[msb] - vp[msb] * vq[msa];
    pf[qp] *= ratio;
    const R a = -vp[msa], b = vp[msb], cc = vq[msa], d = -vq[msb];
    const R e = -bma - vt[msa], f = iab;
    const R det = a * d - b * cc - e * f;
    const R idet = 1.0 / det;
    for (int i = 0; i < n; ++i) {
      vs[i] = idet * m[msa * n + i];
      vt[i] = idet * m[msb * n + i];
    }
    for (int i = 0; i < n; ++i) {
      const R pi = vp[i], qi = vq[i], si = vs[i], ti = vt[i];
      for (int j = 0; j < n; ++j) {
        const R pj = vp[j], qj = vq[j], sj = vs[j], tj = vt[j];
        m[i * n + j] += a * (qi * tj - qj * ti) + b * (qi * sj - qj * si) + cc * (pi * tj - pj * ti) +
                        d * (pi * sj - pj * si) + e * det * (si * tj - sj * ti) +
                        f * idet * (pi * qj - qi * pj);
      }
      m[i * n + msa] += -cc * ti - d * si - f * idet * qi;
      m[i * n + msb] += -a * ti - b * si + f * idet * pi;
    }
    for (int j = 0; j < n; ++j) {
      const R pj = vp[j], qj = vq[j], sj = vs[j], tj = vt[j];
      m[msa * n + j] += cc * tj + d * sj + f * idet * qj;
      m[msb * n + j] += a * tj + b * sj - f * idet * pj;
    }
    m[msa * n + msb] += f * idet;
    m[msb * n + msa] -= f * idet;
  }
}

// ===================================================================================
// Sampler (sampling/driver.rs:175-438, engine.rs:188-476, candidate.rs:137-380,
// initial.rs:77-139, normal_initial.rs:252, metropolis.rs:42-83)
// ===================================================================================
void make_initial_sample(const Ctx& c, Walker& w) {
  const int ns = c.ns, ne = c.ne;
  std::fill(w.ele_idx.begin(), w.ele_idx.end(), -1);
  std::fill(w.ele_cfg.begin(), w.ele_cfg.end(), -1);
  for (int si = 0; si < 2; ++si)
    for (int mi = 0; mi < ne; ++mi) {
      if (w.ele_idx[mi + si * ne] != -1) continue;
      while (true) {
        const int ri = static_cast<int>(w.rng.mod(ns));
        if (w.ele_cfg[ri + si * ns] == -1 && c.m.loc_spn[ri] != 1) {
          w.ele_cfg[ri + si * ns] = mi;
          w.ele_idx[mi + si * ne] = ri;
          break;
        }
      }
    }
  for (int r = 0; r < 2 * ns; ++r) w.ele_num[r] = w.ele_cfg[r] < 0 ? 0 : 1;
  make_proj_cnt(c, w.ele_num.data(), w.proj_cnt.data());
}

double log_ip(const Ctx& c, const double* pf) { return std::log(std::fabs(ip_of(c, pf))); }

void initial_with_retry(const Ctx& c, Walker& w) {
  for (int attempt = 1; attempt <= 101; ++attempt) {
    make_initial_sample(c, w);
    const int info = calc_m_all(c, w.ele_idx.data(), w.inv.data(), w.pf.data());
    if (attempt > 100) throw std::runtime_error("makeInitialSample: too many loops");
    if (info <= 0) return;
  }
}

// One run_block of n_in proposals.
// Largest |ln|IP|_recomputed − ln|IP|_tracked| seen at a refresh (diagnostic).
double g_refresh_drift = 0.0;
// Diagnostic refresh guard: recompute after an accepted move whose ratio on any QP plane
// lies outside [g, 1/g] (0 = off, the reference's schedule); counts guard refreshes.
double g_guard = 0.0;
long long g_guard_count = 0, g_sched_count = 0;

// Teacher-forced long-double shadow of one FP64 chain (oracle_trace_chain): the same
// proposals, decisions and refresh points as the FP64 chain, with the Pfaffians and inverses
// carried in long double by the same algorithms (64-bit significand: 2^11 times the
// precision of double), and the chain's stage operations recorded for a device replay.
// Record per op (8 doubles): PROPOSE: dproj, u, 2((dproj + ln|IP'|) - ln|IP|) in FP64 and in
// long double, accepted, ln|IP| tracked in FP64 and in long double, min_q |pf'_q/pf_q|;
// RECOMPUTE: ln|IP| tracked in FP64 before, recomputed in FP64, recomputed in long double,
// tracked in long double before.
struct Tracer {
  using LD = long double;
  std::vector<LD> inv, pf, pfn;
  LD lip = 0, lip_new = 0;
  std::vector<int32_t> ops;
  std::vector<int64_t> cands;
  std::vector<double> rec;
  size_t max_ops = 0;
  bool full() const { return ops.size() / 7 >= max_ops; }
  void push(const Ctx& c, int code, int ma, int sa, int mb, int sb, int ra, int rb, const int64_t* idx,
            const double* r) {
    if (full()) return;
    const int32_t o[7] = {code, ma, sa, mb, sb, ra, rb};
    ops.insert(ops.end(), o, o + 7);
    cands.insert(cands.end(), idx, idx + c.n);
    rec.insert(rec.end(), r, r + 8);
  }
  LD log_ip_ld(const Ctx& c, const LD* p) const { return std::log(std::fabs(ip_of(c, p))); }
  void begin(const Ctx& c, const int64_t* idx) {
    inv.assign(static_cast<size_t>(c.nqp) * c.n * c.n, 0);
    pf.assign(c.nqp, 0);
    pfn.assign(c.nqp, 0);
    if (calc_m_all(c, idx, inv.data(), pf.data()) != 0) throw std::runtime_error("trace: singular start");
    lip = log_ip_ld(c, pf.data());
  }
  void propose(const Ctx& c, int type, int msa, int msb, const int64_t* idx, double dproj, double u,
               double lw64, bool acc, double lip64, const double* pf_new64, const double* pf64) {
    if (type == 0) ratio_hop(c, msa, idx, inv.data(), pf.data(), pfn.data());
    else ratio_exchange(c, msa, msb, idx, inv.data(), pf.data(), pfn.data());
    lip_new = log_ip_ld(c, pfn.data());
    const LD lw = 2.0L * ((static_cast<LD>(dproj) + lip_new) - lip);
    double rmin = 1e300;
    for (int q = 0; q < c.nqp; ++q) rmin = std::min(rmin, std::fabs(pf_new64[q] / pf64[q]));
    const double r[8] = {dproj, u, lw64, static_cast<double>(lw), acc ? 1.0 : 0.0, lip64,
                         static_cast<double>(lip), rmin};
    const int ne = c.ne;
    if (type == 0) push(c, 0, msa % ne, msa / ne, 0, 0, 0, 0, idx, r);
    else push(c, 2, msa % ne, msa / ne, msb % ne, msb / ne, 0, 0, idx, r);
  }
  void accept(const Ctx& c, int type, int msa, int msb, int ri, int rj, int sa, int sb, const int64_t* idx) {
    if (type == 0) update_hop(c, msa, idx, inv.data(), pf.data());
    else update_exchange(c, msa, msb, ri, rj, sa, sb, idx, inv.data(), pf.data());
    lip = lip_new;
    const double r[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int ne = c.ne;
    if (type == 0) push(c, 1, msa % ne, msa / ne, 0, 0, 0, 0, idx, r);
    else push(c, 3, msa % ne, msa / ne, msb % ne, msb / ne, ri, rj, idx, r);
  }
  void recompute(const Ctx& c, const int64_t* idx, double tracked64, double fresh64) {
    const LD before = lip;
    if (calc_m_all(c, idx, inv.data(), pf.data()) != 0) throw std::runtime_error("trace: singular refresh");
    lip = log_ip_ld(c, pf.data());
    const double r[8] = {tracked64, fresh64, static_cast<double>(lip), static_cast<double>(before), 0, 0, 0, 0};
    push(c, 4, 0, 0, 0, 0, 0, 0, idx, r);
  }
};
Tracer* g_tracer = nullptr;

bool guard_trips(const Ctx& c, const double* pf_new, const double* pf_old) {
  if (g_guard <= 0.0) return false;
  for (int q = 0; q < c.nqp; ++q) {
    const double r = std::fabs(pf_new[q] / pf_old[q]);
    if (!(r >= g_guard && r * g_guard <= 1.0)) return true;
  }
  return false;
}

void run_block(const Ctx& c, Walker& w, int n_in, double& log_ip_old, int& n_acc_win) {
  const int ns = c.ns, ne = c.ne;
  std::vector<double> pf_new(c.nqp);
  std::vector<int64_t> cnt_new(c.nproj), mid(c.nproj);
  int64_t* idx = w.ele_idx.data();
  int64_t* cfg = w.ele_cfg.data();
  int64_t* num = w.ele_num.data();
  for (int step = 0; step < n_in; ++step) {
    int type;  // 0 hop, 1 exchange, 3 none
    switch (c.m.nex_update_path) {
      case 0: type = 0; break;
      case 1: type = w.rng.real2() < 0.5 ? 1 : 0; break;
      case 2: type = 1; break;
      default: type = 3;
    }
    if (type == 0) {
      w.counter[0]++;
      int mi, s, ri, rj;
      mi = static_cast<int>(w.rng.mod(ne));
      s = w.rng.real2() < 0.5 ? 0 : 1;
      ri = static_cast<int>(idx[mi + s * ne]);
      bool reject = false;
      const int icnt_max = ns * ns;
      int icnt = 0;
      while (true) {
        rj = static_cast<int>(w.rng.mod(ns));
        if (icnt > icnt_max) {
          reject = true;
          break;
        }
        ++icnt;
        if (cfg[rj + s * ns] == -1 && c.m.loc_spn[rj] != 1) break;
      }
      if (reject) continue;
      update_ele_config(c, mi, ri, rj, s, idx, cfg, num);
      update_proj_cnt(c, ri, rj, cnt_new.data(), w.proj_cnt.data(), num);
      const int msa = mi + s * ne;
      ratio_hop(c, msa, idx, w.inv.data(), w.pf.data(), pf_new.data());
      const double lip_new = log_ip(c, pf_new.data());
      const double dproj = log_proj_ratio(c, cnt_new.data(), w.proj_cnt.data());
      double wgt = std::exp(2.0 * ((dproj + 0.0 + lip_new) - log_ip_old));
      if (!std::isfinite(wgt)) wgt = -1.0;
      const double u = w.rng.real2();
      if (g_tracer)
        g_tracer->propose(c, 0, msa, 0, idx, dproj, u, 2.0 * ((dproj + 0.0 + lip_new) - log_ip_old), wgt > u,
                          log_ip_old, pf_new.data(), w.pf.data());
      if (wgt > u) {
        const bool trip = guard_trips(c, pf_new.data(), w.pf.data());
        update_hop(c, msa, idx, w.inv.data(), w.pf.data());
        if (g_tracer) g_tracer->accept(c, 0, msa, 0, ri, rj, s, s, idx);
        w.proj_cnt = cnt_new;
        log_ip_old = lip_new;
        ++n_acc_win;
        w.counter[1]++;
        if (trip && n_acc_win <= ns) {
          n_acc_win = ns + 1;
          ++g_guard_count;
          --g_sched_count;
        }
      } else {
        revert_ele_config(c, mi, ri, rj, s, idx, cfg, num);
      }
    } else if (type == 1) {
      w.counter[2]++;
      bool has_single = false;
      for (int r = 0; r < ns; ++r)
        if (num[r] + num[r + ns] == 1) {
          has_single = true;
          break;
        }
      if (!has_single) continue;
      int mi, s, ri, mj, rj;
      while (true) {
        mi = static_cast<int>(w.rng.mod(ne));
        s = w.rng.real2() < 0.5 ? 0 : 1;
        ri = static_cast<int>(idx[mi + s * ne]);
        if (cfg[ri + (1 - s) * ns] == -1) break;
      }
      const int t = 1 - s;
      while (true) {
        mj = static_cast<int>(w.rng.mod(ne));
        rj = static_cast<int>(idx[mj + t * ne]);
        if (cfg[rj + s * ns] == -1) break;
      }
      update_ele_config(c, mi, ri, rj, s, idx, cfg, num);
      update_proj_cnt(c, ri, rj, cnt_new.data(), w.proj_cnt.data(), num);
      update_ele_config(c, mj, rj, ri, t, idx, cfg, num);
      mid = cnt_new;
      update_proj_cnt(c, rj, ri, cnt_new.data(), mid.data(), num);
      const int msa = mi + s * ne, msb = mj + t * ne;
      ratio_exchange(c, msa, msb, idx, w.inv.data(), w.pf.data(), pf_new.data());
      const double lip_new = log_ip(c, pf_new.data());
      const double dproj = log_proj_ratio(c, cnt_new.data(), w.proj_cnt.data());
      double wgt = std::exp(2.0 * ((dproj + 0.0 + lip_new) - log_ip_old));
      if (!std::isfinite(wgt)) wgt = -1.0;
      const double u = w.rng.real2();
      if (g_tracer)
        g_tracer->propose(c, 1, msa, msb, idx, dproj, u, 2.0 * ((dproj + 0.0 + lip_new) - log_ip_old), wgt > u,
                          log_ip_old, pf_new.data(), w.pf.data());
      if (wgt > u) {
        const bool trip = guard_trips(c, pf_new.data(), w.pf.data());
        update_exchange(c, msa, msb, ri, rj, s, t, idx, w.inv.data(), w.pf.data());
        if (g_tracer) g_tracer->accept(c, 1, msa, msb, ri, rj, s, t, idx);
        w.proj_cnt = cnt_new;
        log_ip_old = lip_new;
        ++n_acc_win;
        w.counter[3]++;
        if (trip && n_acc_win <= ns) {
          n_acc_win = ns + 1;
          ++g_guard_count;
          --g_sched_count;
        }
      } else {
        revert_ele_config(c, mj, rj, ri, t, idx, cfg, num);
        revert_ele_config(c, mi, ri, rj, s, idx, cfg, num);
      }
    }
    if (n_acc_win > ns) {
      ++g_sched_count;
      const int info = calc_m_all(c, idx, w.inv.data(), w.pf.data());
      if (info == 0) {
        const double fresh = log_ip(c, w.pf.data());
        const double d = std::fabs(fresh - log_ip_old);
        if (std::isfinite(d) && d > g_refresh_drift) g_refresh_drift = d;
        if (g_tracer) g_tracer->recompute(c, idx, log_ip_old, fresh);
        log_ip_old = fresh;
      }
      n_acc_win = 0;
    }
  }
}

void make_sample(const Ctx& c, Walker& w) {
  const int nsamp = c.m.nvmc_sample;
  if (w.burn) {
    w.ele_idx = w.b_idx;
    w.ele_cfg = w.b_cfg;
    w.ele_num = w.b_num;
    w.proj_cnt = w.b_cnt;
  } else {
    initial_with_retry(c, w);
  }
  calc_m_all(c, w.ele_idx.data(), w.inv.data(), w.pf.data());
  double lip = log_ip(c, w.pf.data());
  bool burn = w.burn;
  if (!std::isfinite(lip)) {
    initial_with_retry(c, w);
    calc_m_all(c, w.ele_idx.data(), w.inv.data(), w.pf.data());
    lip = log_ip(c, w.pf.data());
    burn = false;
  }
  const int n_out = burn ? nsamp + 1 : c.m.nvmc_warmup + nsamp;
  const int n_in = c.m.nvmc_interval * std::max(1, c.ns);
  int n_acc_win = 0;
  std::fill(std::begin(w.counter), std::end(w.counter), 0);
  const int n = c.n, ns2 = c.ns2;
  for (int out = 0; out < n_out; ++out) {
    run_block(c, w, n_in, lip, n_acc_win);
    if (out + nsamp >= n_out) {
      const int sample = out + nsamp - n_out;
      std::copy(w.ele_idx.begin(), w.ele_idx.end(), w.s_idx.begin() + static_cast<size_t>(sample) * n);
      std::copy(w.ele_cfg.begin(), w.ele_cfg.end(), w.s_cfg.begin() + static_cast<size_t>(sample) * ns2);
      std::copy(w.ele_num.begin(), w.ele_num.end(), w.s_num.begin() + static_cast<size_t>(sample) * ns2);
      std::copy(w.proj_cnt.begin(), w.proj_cnt.end(),
                w.s_cnt.begin() + static_cast<size_t>(sample) * c.nproj);
    }
  }
  w.b_idx = w.ele_idx;
  w.b_cfg = w.ele_cfg;
  w.b_num = w.ele_num;
  w.b_cnt = w.proj_cnt;
  w.burn = true;
}

void init_walker(const Ctx& c, Walker& w) {
  w.ele_idx.assign(c.n, -1);
  w.ele_cfg.assign(c.ns2, -1);
  w.ele_num.assign(c.ns2, 0);
  w.proj_cnt.assign(c.nproj, 0);
  w.inv.assign(static_cast<size_t>(c.nqp) * c.n * c.n, 0.0);
  w.pf.assign(c.nqp, 0.0);
  const size_t ns = static_cast<size_t>(c.m.nvmc_sample);
  w.s_idx.assign(ns * c.n, 0);
  w.s_cfg.assign(ns * c.ns2, 0);
  w.s_num.assign(ns * c.ns2, 0);
  w.s_cnt.assign(ns * c.nproj, 0);
}

// ===================================================================================
// exp of the local energy's projection ratios. The reference calls the platform libm
// (mvmc-expert-parsers/src/utils/c_math.rs): std::exp here. For the bitwise C-order parity
// gate with the device, oracle_set_fixed_exp(1) switches to fixed_exp: Cody–Waite reduction
// x = k·ln2 + r (fdlibm's ln2 split, k·ln2_hi exact), the Taylor polynomial of degree 13 in
// Horner form, 2^k in two exact power-of-two steps; every step one IEEE double operation,
// so that any host computes the same bits (libm exps differ in the last bit on some
// arguments; glibc's is not correctly rounded on ~0.1 % of them).
// ===================================================================================
bool g_fixed_exp = false;

double pow2i(int e) {
  const uint64_t bits = static_cast<uint64_t>(e + 1023) << 52;
  double v;
  std::memcpy(&v, &bits, sizeof(v));
  return v;
}

double fixed_exp(double x) {
  if (x != x) return x;
  if (x > 709.782712893384) return std::numeric_limits<double>::infinity();
  if (x < -745.1332191019412) return 0.0;
  const double kd = std::floor(x * 0x1.71547652b82fep+0 + 0.5);
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

double energy_exp(double z) { return g_fixed_exp ? fixed_exp(z) : std::exp(z); }

// ===================================================================================
// Measurement (run.rs:2937-3614; observables.rs:202-330,483-560,1553-1760,3447-3610;
// slater_derivative.rs:75-99,196-430,490-550)
// ===================================================================================
double local_energy(const Ctx& c, const int64_t* idx, const int64_t* cfg, const int64_t* num,
                    const double* inv, const double* pf, double ip) {
  const int ns = c.ns, ne = c.ne, n = c.n;
  double e = 0.0;
  for (const auto& t : c.m.coulomb_intra) e += t.v * static_cast<double>(num[t.i] * num[t.i + ns]);
  for (const auto& t : c.m.coulomb_inter)
    e += t.v * static_cast<double>(num[t.i] + num[t.i + ns]) * static_cast<double>(num[t.j] + num[t.j + ns]);
  for (const auto& t : c.m.hund)
    e -= t.v * (static_cast<double>(num[t.i] * num[t.j]) + static_cast<double>(num[t.i + ns] * num[t.j + ns]));
  if (c.m.transfer.empty() || std::fabs(ip) <= 0.0) return e;
  std::vector<int> rsj(n);
  double transfer = 0.0;
  for (const auto& t : c.m.transfer) {
    const int ri = t.i, rj = t.j, s1 = t.si, s2 = t.sj;
    const int dst = ri + s1 * ns, src = rj + s2 * ns;
    double g1;
    if (s1 == s2 && ri == rj) {
      g1 = static_cast<double>(num[src]);
    } else if (s1 != s2 || num[dst] == 1 || num[src] == 0 || cfg[src] < 0) {
      g1 = 0.0;
    } else {
      const int mj = static_cast<int>(cfg[src]);
      const int msj = mj + s2 * ne;
      // projection ratio of the moved configuration (calh1_direct_projection_ratio_moved)
      auto occ = [&](int slot) -> int64_t {
        if (slot == src) return 0;
        if (slot == dst) return 1;
        return num[slot];
      };
      auto charge_m = [&](int site) { return occ(site) + occ(ns + site) - 1; };
      auto charge = [&](int site) { return num[site] + num[ns + site] - 1; };
      const int source = rj, dest = ri;
      double z = 0.0;
      z -= c.gutz_site[source] * static_cast<double>(occ(source) + occ(ns + source));
      z += c.gutz_site[dest] * static_cast<double>(occ(dest) * occ(ns + dest));
      z += c.jast_pair[source * ns + dest] * static_cast<double>(charge_m(source) - charge_m(dest) + 1);
      for (int site = 0; site < ns; ++site)
        if (site != source && site != dest)
          z += (c.jast_pair[dest * ns + site] - c.jast_pair[source * ns + site]) *
               static_cast<double>(charge(site));
      const double proj_ratio = energy_exp(z);
      for (int k = 0; k < n; ++k) rsj[k] = (k == msj ? ri : static_cast<int>(idx[k])) + (k >= ne ? ns : 0);
      const int rsa = ri + s2 * ns;
      double new_ip = 0.0;
      for (int q = 0; q < c.nqp; ++q) {
        const double* row = inv + static_cast<size_t>(q) * n * n + static_cast<size_t>(msj) * n;
        double r = 0.0;
        for (int k = 0; k < n; ++k) r += row[k] * c.S(q, rsa, rsj[k]);
        new_ip += c.m.qp_weight[q] * (-r * pf[q]);
      }
      g1 = proj_ratio * new_ip / ip;
    }
    transfer -= t.t * g1;
  }
  return e + transfer;
}

// ===================================================================================
// PhysCal Green functions (observables.rs:558-950,1398,1895-2050; green_measurements.rs:
// 264-320; run.rs:3352-3420). The PhysCal form of green_func1 / green_func2: projection
// counts rebuilt by update_proj_cnt, the ratio exp(Σ α Δc) through libm exp, and the
// Julia complex quotient (pfapack julia_complex.rs:9-75), which for a real numerator a and
// real denominator c evaluates a·(1/c) (with its power-of-two rescaling at the extremes).
// ===================================================================================
double julia_real_quotient(double a, double c) {
  const double halfov = 0.5 * std::numeric_limits<double>::max();
  const double twouneps = std::numeric_limits<double>::min() * 2.0 / std::numeric_limits<double>::epsilon();
  const double ab = std::fabs(a), cd = std::fabs(c);
  if (std::isinf(c)) return 0.0 * (a == 0.0 ? a : std::copysign(1.0, a)) * std::copysign(1.0, c);
  double s = 1.0;
  if (ab >= halfov || ab <= twouneps || cd >= halfov || cd <= twouneps) {
    const double bs = 2.0 / (std::numeric_limits<double>::epsilon() * std::numeric_limits<double>::epsilon());
    if (ab >= halfov) {
      a *= 0.5;
      s *= 2.0;
    } else if (ab <= twouneps) {
      a *= bs;
      s /= bs;
    }
    if (cd >= halfov) {
      c *= 0.5;
      s *= 0.5;
    } else if (cd <= twouneps) {
      c *= bs;
      s *= bs;
    }
  }
  const double r = 0.0 / c;
  const double t = 1.0 / (c + 0.0 * r);
  return (a + 0.0 * (0.0 / c)) * t * s;
}

struct GreenSample {
  const int64_t *idx, *cfg, *num, *cnt;
  const double *inv, *pf;
  double ip;
};

// <c†_{ri,s} c_{rj,t}> of one sample (green_func1_impl, observables.rs:1895-2050).
double green_one(const Ctx& c, const GreenSample& g, int ri, int rj, int s, int t) {
  const int ns = c.ns, ne = c.ne, n = c.n;
  if (g.ip == 0.0) return 0.0;
  const int dst = ri + s * ns, src = rj + t * ns;
  if (s == t && ri == rj) return static_cast<double>(g.num[src]);
  if (s != t) return 0.0;
  if (g.num[dst] == 1 || g.num[src] == 0) return 0.0;
  if (g.cfg[src] < 0) return 0.0;
  const int mj = static_cast<int>(g.cfg[src]);
  const int msj = mj + t * ne;
  std::vector<int64_t> idx(g.idx, g.idx + n), num(g.num, g.num + c.ns2), cnt(c.nproj);
  idx[msj] = ri;
  num[dst] = 1;
  num[src] = 0;
  update_proj_cnt(c, rj, ri, cnt.data(), g.cnt, num.data());
  const double proj_ratio = c.nproj > 0 ? std::exp(log_proj_ratio(c, cnt.data(), g.cnt)) : 1.0;
  std::vector<double> pf_new(c.nqp);
  ratio_hop(c, msj, idx.data(), g.inv, g.pf, pf_new.data());
  const double new_ip = ip_of(c, pf_new.data());
  return julia_real_quotient(proj_ratio * new_ip, g.ip);
}

// <c†_{ri,s} c_{rj,s} c†_{rk,u} c_{rl,u}> of one sample (green_func2_impl,
// observables.rs:664-860): index coincidences reduce to one-body values or occupations;
// the general case applies the hop rl→rk (spin u) before rj→ri (spin s).
double green_two(const Ctx& c, const GreenSample& g, int ri, int rj, int rk, int rl, int s, int u) {
  const int ns = c.ns, ne = c.ne, n = c.n;
  if (ne == 0 || ns == 0) return 0.0;
  auto one = [&](int a, int b, int sp) { return green_one(c, g, a, b, sp, sp); };
  const int rsi = ri + s * ns, rsj = rj + s * ns, rtk = rk + u * ns;
  if (s == u) {
    if (rk == rl) return g.num[rtk] == 0 ? 0.0 : one(ri, rj, s);
    if (rj == rl) return 0.0;
    if (ri == rl) {
      if (g.num[rsi] == 0) return 0.0;
      if (rj == rk) return static_cast<double>(1 - g.num[rsj]);
      return -one(rk, rj, s);
    }
    if (rj == rk) return g.num[rsj] == 1 ? 0.0 : one(ri, rl, s);
    if (ri == rk) return 0.0;
    if (ri == rj) return g.num[rsi] == 0 ? 0.0 : one(rk, rl, s);
  } else if (rk == rl) {
    if (g.num[rtk] == 0) return 0.0;
    if (ri == rj) return static_cast<double>(g.num[rsi]);
    return one(ri, rj, s);
  } else if (ri == rj) {
    return g.num[rsi] == 0 ? 0.0 : one(rk, rl, u);
  }
  if (g.num[ri + s * ns] != 0 || g.num[rj + s * ns] != 1 || g.num[rk + u * ns] != 0 || g.num[rl + u * ns] != 1)
    return 0.0;
  const int64_t mj = g.cfg[rj + s * ns], mi = g.cfg[rl + u * ns];
  if (mj < 0 || mi < 0) return 0.0;
  const int msj = static_cast<int>(mj) + s * ne, msi = static_cast<int>(mi) + u * ne;
  std::vector<int64_t> idx(g.idx, g.idx + n), num(g.num, g.num + c.ns2), mid(c.nproj), fin(c.nproj);
  idx[msi] = rk;
  num[rl + u * ns] = 0;
  num[rk + u * ns] = 1;
  update_proj_cnt(c, rl, rk, mid.data(), g.cnt, num.data());
  idx[msj] = ri;
  num[rj + s * ns] = 0;
  num[ri + s * ns] = 1;
  update_proj_cnt(c, rj, ri, fin.data(), mid.data(), num.data());
  const double proj_ratio = std::exp(log_proj_ratio(c, fin.data(), g.cnt));
  std::vector<double> pf_new(c.nqp);
  // calculate_new_pf_m_two2_real_flat(mi, u, mj, s): electron msa = msi, partner msb = msj
  if (msi == msj)
    ratio_hop(c, msj, idx.data(), g.inv, g.pf, pf_new.data());
  else
    ratio_exchange(c, msi, msj, idx.data(), g.inv, g.pf, pf_new.data());
  const double new_ip = ip_of(c, pf_new.data());
  return julia_real_quotient(proj_ratio * new_ip, g.ip);
}

// O vector (real slots): [1, proj counts, Slater derivatives].
void o_vector(const Ctx& c, const int64_t* idx, const int64_t* cnt, const double* inv,
              const double* pf, double ip, double* o) {
  const int n = c.n, ne = c.ne, ns = c.ns, nleg = std::max(1, c.m.nsp_gauss_leg);
  const int norb = c.m.n_orb;
  o[0] = 1.0;
  for (int k = 0; k < c.nproj; ++k) o[1 + k] = static_cast<double>(cnt[k]);
  std::vector<double> qo(static_cast<size_t>(c.nqp) * norb, 0.0);
  std::vector<int> tr(n), sg(n);
  for (int q = 0; q < c.nqp; ++q) {
    const int trans = q / nleg, spidx = q % nleg;
    const int mpidx = trans % c.m.mp_trans();
    for (int k = 0; k < n; ++k) mvmc::translated_site(c.m, static_cast<int>(idx[k]), mpidx, &tr[k], &sg[k]);
    const double p = pf[q];
    const double cs = p * c.m.spgl_cs[spidx], cc = p * c.m.spgl_cc[spidx], ss = p * c.m.spgl_ss[spidx];
    const double* m = inv + static_cast<size_t>(q) * n * n;
    double* out = qo.data() + static_cast<size_t>(q) * norb;
    for (int msi = 0; msi < n; ++msi) {
      const double first = msi < ne ? cs : ss, second = msi < ne ? cc : cs;
      for (int msj = 0; msj < n; ++msj) {
        const int orb = c.m.orb_idx[tr[msi] * ns + tr[msj]];
        if (orb < 0 || orb >= norb) continue;
        const int sign = sg[msi] * sg[msj] * c.m.orb_sgn[tr[msi] * ns + tr[msj]];
        const double v = m[msi * n + msj];
        const double value = msj < ne ? v * first : -v * second;
        out[orb] += value * static_cast<double>(sign);
      }
    }
  }
  const double inv_ip = ip / (ip * ip);
  for (int k = 0; k < norb; ++k) {
    double acc = 0.0;
    for (int q = 0; q < c.nqp; ++q) acc += c.m.qp_weight[q] * qo[static_cast<size_t>(q) * norb + k];
    o[1 + c.nproj + k] = acc * inv_ip;
  }
}

struct Accum {
  double wc = 0, etot = 0, etot2 = 0, sztot = 0, sztot2 = 0;
  std::vector<double> ho, oo, store, o_last;  // store: [NS][size]
};

void measure(const Ctx& c, Walker& w, Accum& a) {
  const int n = c.n, ns2 = c.ns2, size = c.m.sr_size();
  const int nsamp = c.m.nvmc_sample;
  a.ho.assign(size, 0.0);
  a.oo.assign(2 * static_cast<size_t>(size), 0.0);
  a.store.assign(static_cast<size_t>(nsamp) * size, 0.0);
  a.o_last.assign(size, 0.0);
  std::vector<double> inv(static_cast<size_t>(c.nqp) * n * n), pf(c.nqp), o(size);
  for (int s = 0; s < nsamp; ++s) {
    const int64_t* idx = w.s_idx.data() + static_cast<size_t>(s) * n;
    bool all_zero = true, all_neg = true;
    for (int k = 0; k < n; ++k) {
      all_zero = all_zero && idx[k] == 0;
      all_neg = all_neg && idx[k] < 0;
    }
    if (all_zero || all_neg) continue;
    if (calc_m_all(c, idx, inv.data(), pf.data()) != 0) continue;
    const int64_t* cfg = w.s_cfg.data() + static_cast<size_t>(s) * ns2;
    const int64_t* num = w.s_num.data() + static_cast<size_t>(s) * ns2;
    const int64_t* cnt = w.s_cnt.data() + static_cast<size_t>(s) * c.nproj;
    const double ip = ip_of(c, pf.data());
    if (std::fabs(ip) < 1.0e-100) continue;
    const double e = local_energy(c, idx, cfg, num, inv.data(), pf.data(), ip);
    if (!std::isfinite(e)) continue;
    double sz = 0.0;
    for (int r = 0; r < c.ns; ++r) sz += static_cast<double>(num[r] - num[r + c.ns]);
    a.wc += 1.0;
    a.etot += 1.0 * e;
    a.etot2 += (1.0 * e) * e;
    a.sztot += 1.0 * sz;
    a.sztot2 += 1.0 * sz * sz;
    o_vector(c, idx, cnt, inv.data(), pf.data(), ip, o.data());
    a.o_last = o;
    double* st = a.store.data() + static_cast<size_t>(s) * size;
    for (int i = 0; i < size; ++i) {
      st[i] = 1.0 * o[i];
      a.ho[i] += (1.0 * e) * o[i];
    }
  }
  for (int i = 0; i < size; ++i) {  // finalize_oo_store_real, diagonal only
    double mean = 0.0, diag = 0.0;
    for (int s = 0; s < nsamp; ++s) {
      const double v = a.store[static_cast<size_t>(s) * size + i];
      mean += v;
      diag += v * v;
    }
    a.oo[i] = mean;
    a.oo[size + i] = diag;
  }
}

// ===================================================================================
// SR-CG (sr_cg.rs:201-490,492,538-1009; sr_backend.rs:518-606; sr.rs:439)
// ===================================================================================
struct CgResult {
  std::vector<double> x;
  long long status;
};

double sdot(const std::vector<double>& p, const std::vector<double>& q) {
  double s = 0.0;
  for (size_t i = 0; i < p.size(); ++i) s += p[i] * q[i];
  return s;
}

struct SrOperator {
  int na = 0;
  std::vector<double> mean, diag;
  std::vector<std::vector<double>> samples;  // per walker [NS][na]
  double inv_w = 1.0, shift = 0.0;
  void apply(std::vector<double>& z, const std::vector<double>& x) const {
    std::fill(z.begin(), z.end(), 0.0);
    std::vector<double> zl(na);
    for (const auto& smp : samples) {
      const size_t ns = smp.size() / std::max(1, na);
      std::vector<double> y(ns, 0.0);
      for (size_t s = 0; s < ns; ++s) {
        double acc = 0.0;
        for (int i = 0; i < na; ++i) acc += smp[s * na + i] * x[i];
        y[s] = acc;
      }
      std::fill(zl.begin(), zl.end(), 0.0);
      for (size_t s = 0; s < ns; ++s)
        for (int i = 0; i < na; ++i) zl[i] += smp[s * na + i] * y[s];
      for (int i = 0; i < na; ++i) z[i] += zl[i];
    }
    const double coef = sdot(mean, x);
    for (int i = 0; i < na; ++i) z[i] = inv_w * z[i] - coef * mean[i] + shift * diag[i] * x[i];
  }
};

CgResult cg_solve(const SrOperator& op, const std::vector<double>& g, double tol, int max_iter,
                  bool diag_scale) {
  const int n = op.na;
  const double threshold = tol * tol * static_cast<double>(n) * static_cast<double>(n);
  const double pfac = 1.0 + op.shift;
  auto precond = [&](int i, double r) {
    double dq = pfac * op.diag[i];
    if (!std::isfinite(dq) || std::fabs(dq) < 1e-12) dq = dq < 0.0 ? -1e-12 : 1e-12;
    return r / dq;
  };
  CgResult res;
  res.x.assign(n, 0.0);
  std::vector<double> r = g, q(n, 0.0), d;
  double delta;
  if (diag_scale) {
    op.apply(r, res.x);
    for (int i = 0; i < n; ++i) r[i] = g[i] - r[i];
    d.assign(n, 0.0);
    for (int i = 0; i < n; ++i) d[i] = precond(i, r[i]);
    delta = sdot(r, d);
  } else {
    d = g;
    delta = sdot(r, r);
  }
  if (!std::isfinite(delta)) {
    res.status = -1;
    return res;
  }
  int iter = 0;
  while (iter < max_iter) {
    const long long failed = -(static_cast<long long>(iter) + 1);
    if (!std::isfinite(delta)) {
      res.status = failed;
      return res;
    }
    if (std::fabs(delta) < threshold) break;
    op.apply(q, d);
    const double dq = sdot(d, q);
    if (!std::isfinite(dq) || std::fabs(dq) < 1e-20) {
      res.status = failed;
      return res;
    }
    const double alpha = delta / dq;
    if (!std::isfinite(alpha)) {
      res.status = failed;
      return res;
    }
    for (int i = 0; i < n; ++i) res.x[i] += alpha * d[i];
    if ((iter + 1) % 20 == 0) {
      op.apply(r, res.x);
      for (int i = 0; i < n; ++i) r[i] = g[i] - r[i];
    } else {
      for (int i = 0; i < n; ++i) r[i] -= alpha * q[i];
    }
    double delta_new;
    if (diag_scale) {
      for (int i = 0; i < n; ++i) q[i] = precond(i, r[i]);
      delta_new = sdot(r, q);
    } else {
      delta_new = sdot(r, r);
    }
    if (!std::isfinite(delta_new) || std::fabs(delta) < 1e-20) {
      res.status = failed;
      return res;
    }
    const double beta = delta_new / delta;
    if (!std::isfinite(beta)) {
      res.status = failed;
      return res;
    }
    if (diag_scale) {
      delta = delta_new;
      for (int i = 0; i < n; ++i) d[i] = q[i] + beta * d[i];
    } else {
      delta *= beta;
      for (int i = 0; i < n; ++i) d[i] = r[i] + beta * d[i];
    }
    ++iter;
  }
  if (iter == max_iter && std::fabs(delta) >= threshold) {
    res.status = -(static_cast<long long>(max_iter) + 1);
    return res;
  }
  res.status = iter;
  return res;
}

// Returns 0 ok (parameters updated), 1 non-finite update (skipped); throws on abort.
int stochastic_opt_cg(Model& m, const Accum& tot, const std::vector<const Accum*>& walkers,
                      mvmc::SrInfoRow* row, bool* wrote_row) {
  *wrote_row = false;
  const int size = m.sr_size(), npara = m.npara();
  if (m.rescale_smat) throw std::runtime_error("RescaleSmat is outside the oracle's scope");
  const std::vector<double>& oo = tot.oo;
  const std::vector<double>& ho = tot.ho;
  std::vector<double> var(npara);
  for (int pi = 0; pi < npara; ++pi) var[pi] = oo[size + pi + 1] - oo[pi + 1] * oo[pi + 1];
  double vmax = -INFINITY, vmin = INFINITY;
  bool any_nan = false;
  for (double v : var) {
    if (std::isnan(v)) any_nan = true;
    vmax = std::fmax(vmax, v);
    vmin = std::fmin(vmin, v);
  }
  if (any_nan) vmax = vmin = NAN;
  const double threshold = vmax * m.red_cut;
  std::vector<int> mapping;
  int opt_cut = 0, diag_cut = 0;
  for (int pi = 0; pi < npara; ++pi) {
    const bool optimised = static_cast<size_t>(2 * pi) < m.opt_flags.size() && m.opt_flags[2 * pi] == 1;
    if (!optimised) ++opt_cut;
    else if (var[pi] < threshold) ++diag_cut;
    else mapping.push_back(pi);
  }
  if (mapping.empty()) return 0;
  const int na = static_cast<int>(mapping.size());
  SrOperator op;
  op.na = na;
  op.mean.resize(na);
  op.diag.resize(na);
  std::vector<double> g(na);
  const double dt = 2.0 * m.step_dt;
  for (int si = 0; si < na; ++si) {
    const int idx = mapping[si] + 1;
    op.mean[si] = oo[idx];
    op.diag[si] = var[mapping[si]];
    g[si] = -dt * (ho[idx] - ho[0] * oo[idx]);
  }
  const int nsamp = m.nvmc_sample;
  for (const Accum* a : walkers) {
    std::vector<double> smp(static_cast<size_t>(nsamp) * na);
    for (int s = 0; s < nsamp; ++s)
      for (int si = 0; si < na; ++si)
        smp[static_cast<size_t>(s) * na + si] = a->store[static_cast<size_t>(s) * size + mapping[si] + 1];
    op.samples.push_back(std::move(smp));
  }
  op.inv_w = 1.0 / tot.wc;
  op.shift = m.sta_del;
  const int max_iter = m.cg_max_iter > 0 ? m.cg_max_iter : na;
  CgResult res = cg_solve(op, g, m.cg_tol, max_iter, m.diag_scale);
  long long info = res.status;
  if (res.status < 0) {
    const long long fallback_iter = std::max(-res.status - 1, 0LL);
    if (m.cg_fallback) {
      res = cg_solve(op, g, m.cg_tol, max_iter, !m.diag_scale);
      info = -(fallback_iter + 1);
      if (res.status < 0 && m.cg_abort) throw std::runtime_error("fallback SR-CG failed");
    } else {
      if (m.cg_abort) throw std::runtime_error("SR-CG failed and fallback is disabled");
      info = -(fallback_iter + 1);
    }
  }
  int imax = 0;
  for (int i = 1; i < na; ++i)
    if (std::fabs(res.x[imax]) < std::fabs(res.x[i])) imax = i;
  *row = {npara, na, opt_cut, diag_cut, vmax, vmin, res.x[imax], mapping[imax], static_cast<int>(info)};
  *wrote_row = true;
  for (double v : res.x)
    if (!std::isfinite(v)) {
      if (m.cg_abort) throw std::runtime_error("SR-CG produced non-finite updates");
      return 1;
    }
  std::vector<double> p = mvmc::all_parameters(m);
  for (int si = 0; si < na; ++si) p[mapping[si]] += res.x[si];
  mvmc::set_all_parameters(m, p);
  return 0;
}

// Direct SR (NSRCG = 0; sr.rs:77-160, stochastic_opt_real_with_sr_info_timed): the Gram
// OO = Σ_s O_s O_sᵀ / Wc of the stored rows (finalize_oo_store_real + c_order_gram_real,
// sample order here), the active set by the redundancy cut on ⟨O²⟩ − ⟨O⟩²
// (collect_active_real), S_ij = OO_ij − OO_0i OO_0j with the diagonal × (1 + DSROptStaDel)
// and g_i = −2Δt (HO_i − HO_0 OO_0i) (sr_backend.rs:484-511), then the Cholesky solve
// (LAPACK dpotrf('U') + dpotrs, sr.rs:535) and the update x_pi += x_si.
int cholesky_solve_upper(std::vector<double>& a, std::vector<double>& b, int n) {
  // a: row-major symmetric; U stored in the upper triangle, a = Uᵀ U
  for (int j = 0; j < n; ++j) {
    double d = a[static_cast<size_t>(j) * n + j];
    for (int k = 0; k < j; ++k) d -= a[static_cast<size_t>(k) * n + j] * a[static_cast<size_t>(k) * n + j];
    if (!(d > 0.0) || !std::isfinite(d)) return j + 1;
    const double ujj = std::sqrt(d);
    a[static_cast<size_t>(j) * n + j] = ujj;
    for (int i = j + 1; i < n; ++i) {
      double t = a[static_cast<size_t>(j) * n + i];
      for (int k = 0; k < j; ++k) t -= a[static_cast<size_t>(k) * n + j] * a[static_cast<size_t>(k) * n + i];
      a[static_cast<size_t>(j) * n + i] = t / ujj;
    }
  }
  for (int i = 0; i < n; ++i) {  // Uᵀ y = b
    double t = b[i];
    for (int k = 0; k < i; ++k) t -= a[static_cast<size_t>(k) * n + i] * b[k];
    b[i] = t / a[static_cast<size_t>(i) * n + i];
  }
  for (int i = n - 1; i >= 0; --i) {  // U x = y
    double t = b[i];
    for (int k = i + 1; k < n; ++k) t -= a[static_cast<size_t>(i) * n + k] * b[k];
    b[i] = t / a[static_cast<size_t>(i) * n + i];
  }
  for (double v : b)
    if (!std::isfinite(v)) return -1;
  return 0;
}

int stochastic_opt_direct(Model& m, const Accum& tot, const std::vector<const Accum*>& walkers,
                          mvmc::SrInfoRow* row, bool* wrote_row) {
  *wrote_row = false;
  const int size = m.sr_size(), npara = m.npara();
  if (m.rescale_smat) throw std::runtime_error("RescaleSmat is outside the oracle's scope");
  std::vector<double> oo(static_cast<size_t>(size) * size, 0.0);
  const int nsamp = m.nvmc_sample;
  for (const Accum* a : walkers)
    for (int smp = 0; smp < nsamp; ++smp) {
      const double* o = a->store.data() + static_cast<size_t>(smp) * size;
      for (int i = 0; i < size; ++i)
        for (int j = 0; j < size; ++j) oo[static_cast<size_t>(i) * size + j] += o[i] * o[j];
    }
  const double inv = 1.0 / tot.wc;
  for (double& v : oo) v *= inv;
  std::vector<double> s_diag(npara);
  for (int pi = 0; pi < npara; ++pi)
    s_diag[pi] = oo[static_cast<size_t>(pi + 1) * size + pi + 1] - oo[pi + 1] * oo[pi + 1];
  bool any_nan = false;
  double vmax = 0.0;
  for (double v : s_diag) {
    if (std::isnan(v)) any_nan = true;
    vmax = std::fmax(vmax, v);
  }
  if (any_nan) vmax = NAN;
  const double cut = vmax * m.red_cut;
  auto optimised = [&](int c) { return static_cast<size_t>(c) < m.opt_flags.size() && m.opt_flags[c] == 1; };
  std::vector<int> mapping;
  for (int pi = 0; pi < npara; ++pi) {
    if (!optimised(2 * pi)) continue;
    if (s_diag[pi] < cut) continue;
    mapping.push_back(pi);
  }
  if (mapping.empty()) return 0;
  const int na = static_cast<int>(mapping.size());
  std::vector<double> smat(static_cast<size_t>(na) * na), g(na);
  for (int si = 0; si < na; ++si) {
    const int pi = mapping[si] + 1;
    for (int sj = 0; sj < na; ++sj) {
      const int pj = mapping[sj] + 1;
      double v = oo[static_cast<size_t>(pi) * size + pj] - oo[pi] * oo[pj];
      if (si == sj) v *= 1.0 + m.sta_del;
      smat[static_cast<size_t>(si) * na + sj] = v;
    }
    g[si] = -2.0 * m.step_dt * (tot.ho[pi] - tot.ho[0] * oo[pi]);
  }
  if (cholesky_solve_upper(smat, g, na) != 0) return 1;
  // SRinfo in the complex index space of C (real value, zero imaginary variance)
  double smax = s_diag[0], smin = s_diag[0];
  int opt_num = 0, cut_num = 0;
  for (int c = 0; c < 2 * npara; ++c) {
    const double d = (c & 1) ? 0.0 : s_diag[c / 2];
    if (d > smax) smax = d;
    if (d < smin) smin = d;
  }
  for (int c = 0; c < 2 * npara; ++c) {
    const double d = (c & 1) ? 0.0 : s_diag[c / 2];
    if (!optimised(c)) ++opt_num;
    else if (d < smax * m.red_cut) ++cut_num;
  }
  int imax = 0;
  for (int i = 1; i < na; ++i)
    if (std::fabs(g[imax]) < std::fabs(g[i])) imax = i;
  *row = {npara, na, opt_num, cut_num, smax, smin, g[imax], 2 * mapping[imax], 0};
  *wrote_row = true;
  std::vector<double> p = mvmc::all_parameters(m);
  for (int si = 0; si < na; ++si) p[mapping[si]] += g[si];
  mvmc::set_all_parameters(m, p);
  return 0;
}

// ===================================================================================
// Drivers
// ===================================================================================
struct OptRun {
  Model m;
  std::vector<Walker> walkers;
};

void seed_walkers(Model& m, std::vector<Walker>& ws, long long base_seed) {
  for (size_t w = 0; w < ws.size(); ++w) {
    const long long s = base_seed + static_cast<long long>(w);
    if (s < 0 || s > 0xffffffffLL) throw std::runtime_error("seed outside the UInt32 range");
    ws[w].rng.seed(static_cast<uint32_t>(s));
    Model tmp = m;
    mvmc::init_parameter(tmp, [&]() { return ws[w].rng.real2(); });
    if (w == 0) {
      m.gutz = tmp.gutz;
      m.jast = tmp.jast;
      m.slater = tmp.slater;
    }
  }
}

// One optimisation step through measurement; returns the rank-ordered reduction.
void sample_and_measure(Model& m, std::vector<Walker>& ws, std::vector<Accum>& acc, Accum& tot) {
  std::vector<double> slater;
  mvmc::build_slater_table(m, slater);
  Ctx c(m, slater);
  const int size = m.sr_size();
  acc.assign(ws.size(), Accum());
  for (size_t w = 0; w < ws.size(); ++w) {
    if (ws[w].inv.empty()) init_walker(c, ws[w]);
    make_sample(c, ws[w]);
    measure(c, ws[w], acc[w]);
  }
  tot = Accum();
  tot.ho.assign(size, 0.0);
  tot.oo.assign(2 * static_cast<size_t>(size), 0.0);
  for (const Accum& a : acc) {
    tot.wc += a.wc;
    tot.etot += a.etot;
    tot.etot2 += a.etot2;
    tot.sztot += a.sztot;
    tot.sztot2 += a.sztot2;
    for (int i = 0; i < size; ++i) tot.ho[i] += a.ho[i];
    for (int i = 0; i < 2 * size; ++i) tot.oo[i] += a.oo[i];
  }
  tot.o_last = acc.back().o_last;
  if (std::fabs(tot.wc) >= 1.0e-15) {
    const double inv = 1.0 / tot.wc;
    tot.etot *= inv;
    tot.etot2 *= inv;
    tot.sztot *= inv;
    tot.sztot2 *= inv;
    for (double& v : tot.oo) v *= inv;
    for (double& v : tot.ho) v *= inv;
  }
}

void copy_err(const std::exception& e, char* err, int len) {
  if (err && len > 0) {
    std::snprintf(err, len, "%s", e.what());
  }
}

}  // namespace orc

// ===================================================================================
// C ABI
// ===================================================================================
extern "C" {

void oracle_sfmt_words(uint32_t seed, int count, uint32_t* out) {
  orc::Sfmt r;
  r.seed(seed);
  for (int i = 0; i < count; ++i) out[i] = r.u32();
}

void oracle_pfinv_batch(const double* x, int n, int planes, double* pf, double* inv, int* status) {
  const size_t nn = static_cast<size_t>(n) * n;
  for (int p = 0; p < planes; ++p) {
    std::vector<double> a(x + p * nn, x + (p + 1) * nn);
    double v = 0.0;
    status[p] = orc::pfinv(a.data(), n, &v);
    pf[p] = status[p] == 0 ? v : 0.0;
    std::copy(a.begin(), a.end(), inv + p * nn);
  }
}

int oracle_model_dims(const char* namelist, int* dims, char* err, int err_len) {
  try {
    mvmc::Model m = mvmc::read_expert(namelist);
    mvmc::init_qp_weight(m);
    dims[0] = m.nsite;
    dims[1] = m.ne;
    dims[2] = m.nqp;
    dims[3] = m.nproj();
    dims[4] = m.npara();
    dims[5] = m.nvmc_sample;
    dims[6] = m.data_qty_smp;
    dims[7] = m.n_orb;
    return 0;
  } catch (const std::exception& e) {
    orc::copy_err(e, err, err_len);
    return 1;
  }
}

int oracle_run_opt(const char* namelist, const char* initial_def, const char* out_dir, int walkers,
                   int nsteps, long long seed_override, char* err, int err_len) {
  try {
    mvmc::Model m = mvmc::read_expert(namelist);
    if (nsteps > 0) {
      m.nsr_opt_itr_step = nsteps;
      m.nsr_opt_itr_smp = std::min(m.nsr_opt_itr_smp, nsteps);
    }
    const long long base = seed_override >= 0 ? seed_override : m.rnd_seed;
    std::vector<orc::Walker> ws(std::max(1, walkers));
    orc::seed_walkers(m, ws, base);
    if (initial_def && *initial_def) {
      std::string why;
      if (!mvmc::read_para_triples(m, initial_def, &why)) throw std::runtime_error("initial.def: " + why);
    }
    mvmc::sync_modified_parameter(m, true);
    mvmc::init_qp_weight(m);
    const int window_start = m.nsr_opt_itr_step - m.nsr_opt_itr_smp;
    std::vector<mvmc::OptPoint> window;
    bool first_info = true;
    for (int step = 0; step < m.nsr_opt_itr_step; ++step) {
      std::vector<orc::Accum> acc;
      orc::Accum tot;
      orc::sample_and_measure(m, ws, acc, tot);
      mvmc::StepEnergy se{tot.etot, tot.etot2, tot.sztot, tot.sztot2};
      mvmc::write_out_row(m, out_dir, step, se);
      std::vector<const orc::Accum*> ptrs;
      for (const auto& a : acc) ptrs.push_back(&a);
      mvmc::SrInfoRow row;
      bool wrote = false;
      const int info = m.nsrcg != 0 ? orc::stochastic_opt_cg(m, tot, ptrs, &row, &wrote)
                                    : orc::stochastic_opt_direct(m, tot, ptrs, &row, &wrote);
      if (wrote) {
        mvmc::write_srinfo_row(out_dir, m, first_info, row);
        first_info = false;
      }
      if (info != 0) throw std::runtime_error("SR failed at step " + std::to_string(step));
      mvmc::sync_modified_parameter(m, true);
      if (step >= window_start) window.push_back({tot.etot, tot.etot2, mvmc::all_parameters(m)});
    }
    mvmc::write_opt_files(m, out_dir, window);
    return 0;
  } catch (const std::exception& e) {
    orc::copy_err(e, err, err_len);
    return 1;
  }
}

int oracle_step1_operands(const char* namelist, int cg, int store, long long seed, double* energy,
                          double* ho, double* oo, double* o_last, int sr_size, char* err,
                          int err_len) {
  try {
    mvmc::Model m = mvmc::read_expert(namelist);
    m.nsrcg = cg;
    m.nstore = store;
    m.nsr_opt_itr_step = 1;
    m.nsr_opt_itr_smp = 1;
    if (!cg) throw std::runtime_error("direct SR operands are not covered");
    if (m.sr_size() != sr_size) throw std::runtime_error("sr_size mismatch");
    std::vector<orc::Walker> ws(1);
    orc::seed_walkers(m, ws, seed);
    mvmc::sync_modified_parameter(m, true);
    mvmc::init_qp_weight(m);
    std::vector<orc::Accum> acc;
    orc::Accum tot;
    orc::sample_and_measure(m, ws, acc, tot);
    energy[0] = tot.etot;
    std::copy(tot.ho.begin(), tot.ho.end(), ho);
    std::copy(tot.oo.begin(), tot.oo.end(), oo);
    std::copy(tot.o_last.begin(), tot.o_last.end(), o_last);
    return 0;
  } catch (const std::exception& e) {
    orc::copy_err(e, err, err_len);
    return 1;
  }
}

int oracle_physcal_samples(const char* namelist, const char* zqp_opt, long long seed,
                           int64_t* ele_idx, int64_t* ele_cfg, int64_t* ele_num, int64_t* proj_cnt,
                           int64_t* counters, int64_t* draws, uint32_t* next624, double* energies,
                           char* err, int err_len) {
  try {
    mvmc::Model m = mvmc::read_expert(namelist);
    std::string why;
    if (!mvmc::read_para_triples(m, zqp_opt, &why)) throw std::runtime_error("zqp_opt.dat: " + why);
    mvmc::sync_modified_parameter(m, false);
    std::vector<orc::Walker> ws(1);
    ws[0].rng.seed(static_cast<uint32_t>(seed));
    {
      mvmc::Model tmp = m;  // PhysCal consumes the initial-parameter draws on a clone
      mvmc::init_parameter(tmp, [&]() { return ws[0].rng.real2(); });
    }
    if (m.nmp_trans < 0) m.nmp_trans = -m.nmp_trans;
    mvmc::init_qp_weight(m);
    std::vector<double> slater;
    mvmc::build_slater_table(m, slater);
    orc::Ctx c(m, slater);
    orc::init_walker(c, ws[0]);
    const size_t nsamp = static_cast<size_t>(m.nvmc_sample);
    for (int b = 0; b < m.data_qty_smp; ++b) {
      orc::Walker& w = ws[0];
      orc::make_sample(c, w);
      std::copy(w.s_idx.begin(), w.s_idx.end(), ele_idx + b * nsamp * c.n);
      std::copy(w.s_cfg.begin(), w.s_cfg.end(), ele_cfg + b * nsamp * c.ns2);
      std::copy(w.s_num.begin(), w.s_num.end(), ele_num + b * nsamp * c.ns2);
      std::copy(w.s_cnt.begin(), w.s_cnt.end(), proj_cnt + b * nsamp * c.nproj);
      for (int k = 0; k < 6; ++k) counters[b * 6 + k] = w.counter[k];
      draws[b] = static_cast<int64_t>(w.rng.draws);
      w.rng.peek(next624 + b * 624, 624);
      orc::Accum a;
      orc::measure(c, w, a);
      energies[2 * b] = a.etot / a.wc;
      energies[2 * b + 1] = a.etot2 / a.wc;
    }
    return 0;
  } catch (const std::exception& e) {
    orc::copy_err(e, err, err_len);
    return 1;
  }
}

int oracle_green_dims(const char* namelist, int* dims, char* err, int err_len) {
  try {
    const mvmc::Model m = mvmc::read_expert(namelist);
    dims[0] = static_cast<int>(m.green_one.size());
    dims[1] = static_cast<int>(m.green_two_ex.size());
    dims[2] = static_cast<int>(m.green_two.size());
    dims[3] = m.data_qty_smp;
    dims[4] = m.data_idx_start;
    return 0;
  } catch (const std::exception& e) {
    orc::copy_err(e, err, err_len);
    return 1;
  }
}

int oracle_physcal_green(const char* namelist, const char* zqp_opt, long long seed, int walkers,
                         double* energy, double* one, double* ex, double* two, const char* out_dir,
                         char* err, int err_len) {
  try {
    mvmc::Model m = mvmc::read_expert(namelist);
    std::string why;
    if (!mvmc::read_para_triples(m, zqp_opt, &why)) throw std::runtime_error("zqp_opt.dat: " + why);
    mvmc::sync_modified_parameter(m, false);
    const int W = std::max(1, walkers);
    std::vector<orc::Walker> ws(W);
    for (int w = 0; w < W; ++w) {
      const long long sd = seed + w;
      if (sd < 0 || sd > 0xffffffffLL) throw std::runtime_error("seed outside the UInt32 range");
      ws[w].rng.seed(static_cast<uint32_t>(sd));
      mvmc::Model tmp = m;  // the initial-parameter draws are consumed on a clone
      mvmc::init_parameter(tmp, [&]() { return ws[w].rng.real2(); });
    }
    if (m.nmp_trans < 0) m.nmp_trans = -m.nmp_trans;
    mvmc::init_qp_weight(m);
    std::vector<double> slater;
    mvmc::build_slater_table(m, slater);
    orc::Ctx c(m, slater);
    for (auto& w : ws) orc::init_walker(c, w);
    const int n1 = static_cast<int>(m.green_one.size()), nx = static_cast<int>(m.green_two_ex.size()),
              n2 = static_cast<int>(m.green_two.size());
    const int n = c.n, nsamp = m.nvmc_sample;
    std::vector<double> inv(static_cast<size_t>(c.nqp) * n * n), pf(c.nqp), loc(n1);
    for (int b = 0; b < m.data_qty_smp; ++b) {
      double tot[5] = {0, 0, 0, 0, 0};
      std::vector<double> g1(n1, 0.0), gx(nx, 0.0), g2(n2, 0.0);
      for (int wi = 0; wi < W; ++wi) {
        orc::Walker& w = ws[wi];
        orc::make_sample(c, w);
        double acc[5] = {0, 0, 0, 0, 0};
        std::vector<double> s1(n1, 0.0), sx(nx, 0.0), s2(n2, 0.0);
        for (int s = 0; s < nsamp; ++s) {
          const int64_t* idx = w.s_idx.data() + static_cast<size_t>(s) * n;
          bool all_zero = true, all_neg = true;
          for (int k = 0; k < n; ++k) {
            all_zero = all_zero && idx[k] == 0;
            all_neg = all_neg && idx[k] < 0;
          }
          if (all_zero || all_neg) continue;
          if (orc::calc_m_all(c, idx, inv.data(), pf.data()) != 0) continue;
          const int64_t* cfg = w.s_cfg.data() + static_cast<size_t>(s) * c.ns2;
          const int64_t* num = w.s_num.data() + static_cast<size_t>(s) * c.ns2;
          const int64_t* cnt = w.s_cnt.data() + static_cast<size_t>(s) * c.nproj;
          const double ip = orc::ip_of(c, pf.data());
          if (std::fabs(ip) < 1.0e-100) continue;
          const double e = orc::local_energy(c, idx, cfg, num, inv.data(), pf.data(), ip);
          if (!std::isfinite(e)) continue;
          double sz = 0.0;
          for (int r = 0; r < c.ns; ++r) sz += static_cast<double>(num[r] - num[r + c.ns]);
          acc[0] += 1.0;
          acc[1] += 1.0 * e;
          acc[2] += (1.0 * e) * e;
          acc[3] += 1.0 * sz;
          acc[4] += 1.0 * sz * sz;
          const orc::GreenSample gs{idx, cfg, num, cnt, inv.data(), pf.data(), ip};
          for (int k = 0; k < n1; ++k) {
            const auto& t = m.green_one[k];
            loc[k] = orc::green_one(c, gs, t.i, t.j, t.si, t.sj);
            s1[k] += loc[k];
          }
          for (int k = 0; k < nx; ++k) sx[k] += (1.0 * loc[m.green_two_ex[k].first]) * loc[m.green_two_ex[k].second];
          for (int k = 0; k < n2; ++k) {
            const auto& t = m.green_two[k];
            s2[k] += orc::green_two(c, gs, t.i, t.j, t.k, t.l, t.si, t.sk);
          }
        }
        // per-chain normalisation by its own weight, then the chain-order sum
        const double inv_w = acc[0] != 0.0 ? 1.0 / acc[0] : 1.0;
        for (int k = 0; k < n1; ++k) g1[k] += s1[k] * inv_w;
        for (int k = 0; k < nx; ++k) gx[k] += sx[k] * inv_w;
        for (int k = 0; k < n2; ++k) g2[k] += s2[k] * inv_w;
        for (int k = 0; k < 5; ++k) tot[k] += acc[k];
      }
      if (W > 1) {
        const double inv_r = 1.0 / W;
        for (auto& v : g1) v *= inv_r;
        for (auto& v : gx) v *= inv_r;
        for (auto& v : g2) v *= inv_r;
      }
      mvmc::StepEnergy se;
      if (std::fabs(tot[0]) >= 1.0e-15) {
        const double iw = 1.0 / tot[0];
        se.etot = tot[1] * iw;
        se.etot2 = tot[2] * iw;
        se.sztot = tot[3] * iw;
        se.sztot2 = tot[4] * iw;
      } else {
        se.etot = tot[1];
        se.etot2 = tot[2];
        se.sztot = tot[3];
        se.sztot2 = tot[4];
      }
      energy[4 * b] = se.etot;
      energy[4 * b + 1] = se.etot2;
      energy[4 * b + 2] = se.sztot;
      energy[4 * b + 3] = se.sztot2;
      std::copy(g1.begin(), g1.end(), one + static_cast<size_t>(b) * n1);
      std::copy(gx.begin(), gx.end(), ex + static_cast<size_t>(b) * nx);
      std::copy(g2.begin(), g2.end(), two + static_cast<size_t>(b) * n2);
      if (out_dir && *out_dir)
        mvmc::write_physcal_block(m, out_dir, m.data_idx_start + b, se, g1.data(), gx.data(), g2.data());
    }
    return 0;
  } catch (const std::exception& e) {
    orc::copy_err(e, err, err_len);
    return 1;
  }
}

int oracle_green_identity(const char* namelist, const char* zqp_opt, long long seed, double* out, char* err,
                          int err_len) {
  try {
    mvmc::Model m = mvmc::read_expert(namelist);
    std::string why;
    if (!mvmc::read_para_triples(m, zqp_opt, &why)) throw std::runtime_error("zqp_opt.dat: " + why);
    mvmc::sync_modified_parameter(m, false);
    orc::Walker w;
    w.rng.seed(static_cast<uint32_t>(seed));
    {
      mvmc::Model tmp = m;
      mvmc::init_parameter(tmp, [&]() { return w.rng.real2(); });
    }
    if (m.nmp_trans < 0) m.nmp_trans = -m.nmp_trans;
    mvmc::init_qp_weight(m);
    std::vector<double> slater;
    mvmc::build_slater_table(m, slater);
    orc::Ctx c(m, slater);
    orc::init_walker(c, w);
    orc::make_sample(c, w);
    const int n = c.n, ns = c.ns, ne = c.ne;
    std::vector<double> inv(static_cast<size_t>(c.nqp) * n * n), pf(c.nqp), inv2(inv.size()), pf2(c.nqp);
    double worst = 0.0;
    long long n1 = 0, n2 = 0;
    // ratio by recomputation: exp(Σ α (c' − c)) · IP(x') / IP(x)
    auto direct = [&](const std::vector<int64_t>& idx2, const std::vector<int64_t>& num2, const int64_t* cnt,
                      double ip) {
      std::vector<int64_t> cnt2(c.nproj);
      orc::make_proj_cnt(c, num2.data(), cnt2.data());
      if (orc::calc_m_all(c, idx2.data(), inv2.data(), pf2.data()) != 0) return std::nan("");
      return std::exp(orc::log_proj_ratio(c, cnt2.data(), cnt)) * orc::ip_of(c, pf2.data()) / ip;
    };
    auto note = [&](double a, double b) {
      if (!std::isfinite(b)) return;
      worst = std::max(worst, std::fabs(a - b) / std::max(std::fabs(b), 1e-300));
    };
    for (int s = 0; s < m.nvmc_sample; ++s) {
      const int64_t* idx = w.s_idx.data() + static_cast<size_t>(s) * n;
      const int64_t* cfg = w.s_cfg.data() + static_cast<size_t>(s) * c.ns2;
      const int64_t* num = w.s_num.data() + static_cast<size_t>(s) * c.ns2;
      const int64_t* cnt = w.s_cnt.data() + static_cast<size_t>(s) * c.nproj;
      if (orc::calc_m_all(c, idx, inv.data(), pf.data()) != 0) continue;
      const double ip = orc::ip_of(c, pf.data());
      if (std::fabs(ip) < 1.0e-100) continue;
      const orc::GreenSample gs{idx, cfg, num, cnt, inv.data(), pf.data(), ip};
      for (const auto& t : m.green_one) {
        if (t.si != t.sj || t.i == t.j) continue;
        const int dst = t.i + t.si * ns, src = t.j + t.sj * ns;
        if (num[dst] == 1 || num[src] == 0) continue;
        std::vector<int64_t> idx2(idx, idx + n), num2(num, num + c.ns2);
        idx2[cfg[src] + t.sj * ne] = t.i;
        num2[dst] = 1;
        num2[src] = 0;
        note(orc::green_one(c, gs, t.i, t.j, t.si, t.sj), direct(idx2, num2, cnt, ip));
        ++n1;
      }
      for (const auto& t : m.green_two) {
        const int ri = t.i, rj = t.j, rk = t.k, rl = t.l, sp = t.si, u = t.sk;
        const bool coincident = sp == u ? (rk == rl || rj == rl || ri == rl || rj == rk || ri == rk || ri == rj)
                                        : (rk == rl || ri == rj);
        if (coincident) continue;
        if (num[ri + sp * ns] != 0 || num[rj + sp * ns] != 1 || num[rk + u * ns] != 0 || num[rl + u * ns] != 1)
          continue;
        std::vector<int64_t> idx2(idx, idx + n), num2(num, num + c.ns2);
        idx2[cfg[rl + u * ns] + u * ne] = rk;
        idx2[cfg[rj + sp * ns] + sp * ne] = ri;
        num2[rl + u * ns] = 0;
        num2[rk + u * ns] = 1;
        num2[rj + sp * ns] = 0;
        num2[ri + sp * ns] = 1;
        note(orc::green_two(c, gs, ri, rj, rk, rl, sp, u), direct(idx2, num2, cnt, ip));
        ++n2;
      }
    }
    out[0] = worst;
    out[1] = static_cast<double>(n1);
    out[2] = static_cast<double>(n2);
    return 0;
  } catch (const std::exception& e) {
    orc::copy_err(e, err, err_len);
    return 1;
  }
}

int oracle_opt_step1_walkers(const char* namelist, const char* initial_def, int walkers,
                             long long seed, int64_t* ele_idx, int64_t* proj_cnt, int64_t* counters,
                             int64_t* draws, double* energy, double* ho, double* oo, double* ostore,
                             char* err, int err_len) {
  try {
    mvmc::Model m = mvmc::read_expert(namelist);
    if (m.nsrcg == 0) m.nsrcg = 1;
    std::vector<orc::Walker> ws(std::max(1, walkers));
    orc::seed_walkers(m, ws, seed >= 0 ? seed : m.rnd_seed);
    if (initial_def && *initial_def) {
      std::string why;
      if (!mvmc::read_para_triples(m, initial_def, &why)) throw std::runtime_error("initial.def: " + why);
    }
    mvmc::sync_modified_parameter(m, true);
    mvmc::init_qp_weight(m);
    std::vector<orc::Accum> acc;
    orc::Accum tot;
    orc::sample_and_measure(m, ws, acc, tot);
    const int n = m.nsize(), size = m.sr_size(), S = m.nvmc_sample, np = m.nproj();
    for (size_t w = 0; w < ws.size(); ++w) {
      std::copy(ws[w].s_idx.begin(), ws[w].s_idx.end(), ele_idx + w * S * n);
      std::copy(ws[w].s_cnt.begin(), ws[w].s_cnt.end(), proj_cnt + w * S * np);
      for (int k = 0; k < 6; ++k) counters[w * 6 + k] = ws[w].counter[k];
      draws[w] = static_cast<int64_t>(ws[w].rng.draws);
      std::copy(acc[w].store.begin(), acc[w].store.end(), ostore + w * S * size);
    }
    energy[0] = tot.wc;
    energy[1] = tot.etot;
    energy[2] = tot.etot2;
    energy[3] = tot.sztot;
    energy[4] = tot.sztot2;
    std::copy(tot.ho.begin(), tot.ho.end(), ho);
    std::copy(tot.oo.begin(), tot.oo.end(), oo);
    return 0;
  } catch (const std::exception& e) {
    orc::copy_err(e, err, err_len);
    return 1;
  }
}

int oracle_trace_chain(const char* namelist, const char* initial_def, long long seed, int walker, int blocks,
                       int max_ops, int64_t* idx0, int32_t* ops, int64_t* cands, double* rec, int* nops,
                       char* err, int err_len) {
  orc::Tracer tr;
  try {
    mvmc::Model m = mvmc::read_expert(namelist);
    if (m.nsrcg == 0) m.nsrcg = 1;
    std::vector<orc::Walker> ws(static_cast<size_t>(std::max(0, walker)) + 1);
    orc::seed_walkers(m, ws, seed >= 0 ? seed : m.rnd_seed);
    if (initial_def && *initial_def) {
      std::string why;
      if (!mvmc::read_para_triples(m, initial_def, &why)) throw std::runtime_error("initial.def: " + why);
    }
    mvmc::sync_modified_parameter(m, true);
    mvmc::init_qp_weight(m);
    std::vector<double> slater;
    mvmc::build_slater_table(m, slater);
    orc::Ctx c(m, slater);
    orc::Walker& w = ws.back();
    orc::init_walker(c, w);
    orc::initial_with_retry(c, w);
    orc::calc_m_all(c, w.ele_idx.data(), w.inv.data(), w.pf.data());
    double lip = orc::log_ip(c, w.pf.data());
    if (!std::isfinite(lip)) throw std::runtime_error("trace: non-finite initial amplitude");
    std::copy(w.ele_idx.begin(), w.ele_idx.end(), idx0);
    tr.max_ops = static_cast<size_t>(std::max(0, max_ops));
    tr.begin(c, w.ele_idx.data());
    const int n_out = std::min(blocks, c.m.nvmc_warmup + c.m.nvmc_sample);
    const int n_in = c.m.nvmc_interval * std::max(1, c.ns);
    int n_acc_win = 0;
    orc::g_tracer = &tr;
    for (int out = 0; out < n_out && !tr.full(); ++out) orc::run_block(c, w, n_in, lip, n_acc_win);
    orc::g_tracer = nullptr;
    std::copy(tr.ops.begin(), tr.ops.end(), ops);
    std::copy(tr.cands.begin(), tr.cands.end(), cands);
    std::copy(tr.rec.begin(), tr.rec.end(), rec);
    *nops = static_cast<int>(tr.ops.size() / 7);
    return 0;
  } catch (const std::exception& e) {
    orc::g_tracer = nullptr;
    orc::copy_err(e, err, err_len);
    return 1;
  }
}

int oracle_qp_weights(const char* namelist, double* out, char* err, int err_len) {
  try {
    mvmc::Model m = mvmc::read_expert(namelist);
    mvmc::init_qp_weight(m);
    std::copy(m.qp_weight.begin(), m.qp_weight.end(), out);
    return 0;
  } catch (const std::exception& e) {
    orc::copy_err(e, err, err_len);
    return 1;
  }
}

int oracle_cholesky_solve(double* a, double* b, int n) {
  std::vector<double> av(a, a + static_cast<size_t>(n) * n), bv(b, b + n);
  const int info = orc::cholesky_solve_upper(av, bv, n);
  std::copy(av.begin(), av.end(), a);
  std::copy(bv.begin(), bv.end(), b);
  return info;
}

void oracle_set_refresh_guard(double g) { orc::g_guard = g; }

void oracle_set_fixed_exp(int on) { orc::g_fixed_exp = on != 0; }

double oracle_fixed_exp(double x) { return orc::fixed_exp(x); }

void oracle_refresh_counts(long long* sched, long long* guard, int reset) {
  *sched = orc::g_sched_count;
  *guard = orc::g_guard_count;
  if (reset) orc::g_sched_count = orc::g_guard_count = 0;
}

double oracle_refresh_drift(int reset) {
  const double d = orc::g_refresh_drift;
  if (reset) orc::g_refresh_drift = 0.0;
  return d;
}

int oracle_cg_fixed(int n, int samples, const double* mean, const double* diag, const double* smp,
                    const double* g, double inv_w, double shift, double tol, int max_iter,
                    int diag_scale, double* x_out, double* z_apply) {
  orc::SrOperator op;
  op.na = n;
  op.mean.assign(mean, mean + n);
  op.diag.assign(diag, diag + n);
  op.samples.emplace_back(smp, smp + static_cast<size_t>(n) * samples);
  op.inv_w = inv_w;
  op.shift = shift;
  if (z_apply) {
    std::vector<double> z(n), gv(g, g + n);
    op.apply(z, gv);
    std::copy(z.begin(), z.end(), z_apply);
  }
  orc::CgResult r = orc::cg_solve(op, std::vector<double>(g, g + n), tol, max_iter, diag_scale != 0);
  std::copy(r.x.begin(), r.x.end(), x_out);
  return static_cast<int>(r.status);
}

// Teacher-forced replay of the RealPfStage operations (sampling/stage.rs:56-129) with the
// CPU stage arithmetic above (CpuStage, stage.rs:134-240): the Slater table of `params`
// (projection then Slater parameters), the inverses of idx0, then nops calls, each row of
// ops = {code, ma, sa, mb, sb, ra_old, rb_old}; code 0 propose hop, 1 accept hop (the
// current Pf become the last proposal's, stage.rs:182), 2 propose exchange, 3 accept
// exchange, 4 recompute. idx_seq holds the ele_idx of every call. out[k*nqp..]: pf_new of
// a proposal, else the current Pf (NaN after a failed recompute); inv_out: the final InvM.
int oracle_stage_replay(const char* namelist, const double* params, int npara, const int64_t* idx0, int nops,
                        const int* ops, const int64_t* idx_seq, double* out, double* inv_out, char* err,
                        int err_len) {
  try {
    mvmc::Model m = mvmc::read_expert(namelist);
    if (npara != m.npara()) throw std::runtime_error("parameter count mismatch");
    mvmc::set_all_parameters(m, std::vector<double>(params, params + npara));
    mvmc::init_qp_weight(m);
    std::vector<double> slater;
    mvmc::build_slater_table(m, slater);
    orc::Ctx c(m, slater);
    const int n = c.n, nqp = c.nqp, ne = c.ne;
    std::vector<double> inv(static_cast<size_t>(nqp) * n * n), pf(nqp), pfn(nqp);
    if (orc::calc_m_all(c, idx0, inv.data(), pf.data()) != 0) throw std::runtime_error("singular start");
    for (int k = 0; k < nops; ++k) {
      const int* o = ops + 7 * k;
      const int64_t* idx = idx_seq + static_cast<size_t>(k) * n;
      const int msa = o[1] + o[2] * ne, msb = o[3] + o[4] * ne;
      double* dst = out + static_cast<size_t>(k) * nqp;
      switch (o[0]) {
        case 0:
          orc::ratio_hop(c, msa, idx, inv.data(), pf.data(), pfn.data());
          std::copy(pfn.begin(), pfn.end(), dst);
          break;
        case 1:
          orc::update_hop(c, msa, idx, inv.data(), pf.data());
          pf = pfn;
          std::copy(pf.begin(), pf.end(), dst);
          break;
        case 2:
          orc::ratio_exchange(c, msa, msb, idx, inv.data(), pf.data(), pfn.data());
          std::copy(pfn.begin(), pfn.end(), dst);
          break;
        case 3:
          orc::update_exchange(c, msa, msb, o[5], o[6], o[2], o[4], idx, inv.data(), pf.data());
          std::copy(pf.begin(), pf.end(), dst);
          break;
        case 4:
          if (orc::calc_m_all(c, idx, inv.data(), pf.data()) != 0) std::fill(dst, dst + nqp, NAN);
          else std::copy(pf.begin(), pf.end(), dst);
          break;
        default:
          throw std::runtime_error("unknown stage op");
      }
    }
    std::copy(inv.begin(), inv.end(), inv_out);
    return 0;
  } catch (const std::exception& e) {
    orc::copy_err(e, err, err_len);
    return 1;
  }
}

}  // extern "C"
