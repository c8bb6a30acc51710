// Walker-ensemble engine behind the C ABI: model upload, the Slater table (K0), and the
// sample → measure → SR-CG stages of one optimisation step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/mvmc_b200.h"
#include "../host/abi_common.h"
#include "../host/expert.h"
#include "common.cuh"
#include "engine.cuh"
#include "sfmt.cuh"

namespace mvmcb {

int launch_sample(const DevModel& m, const DevWalkers& w, int precision, cudaStream_t stream);
bool sample_planes_in_smem(const DevModel& m, int precision, int limit);
int launch_measure(const DevModel& m, const int* s_idx, const int* s_cfg, const int* s_num,
                   const int* s_cnt, int nsamples, double* gws, int gws_blocks, double* ostore,
                   double* eloc, double* lpsi, int* valid, double* gval, unsigned* status, cudaStream_t stream);
int launch_green_reduce(const DevModel& m, int W, int S, int n_one, int nex, const int* ex, const double* gval,
                        const int* valid, double* part, double* out, cudaStream_t stream);
int green_chunks(int W);
int launch_reduce(const DevModel& m, int W, int S, const double* ostore, const double* eloc,
                  const int* valid, const int* s_num, double* wsum, double* tot, cudaStream_t stream);
int launch_reduce_totals(const DevModel& m, int W, const double* wsum, double* tot, cudaStream_t stream);
void corder_scratch_sizes(const DevModel& m, long long* dstride, long long* istride);
int launch_measure_corder(const DevModel& m, int W, int S, const int* s_idx, const int* s_cfg, const int* s_num,
                          const int* s_cnt, double* ostore, double* eloc, double* lpsi, int* valid, double* wsum,
                          double* dscr, int* iscr, cudaStream_t stream);
int launch_cg_corder(const CgArgs& a, int W, int S, cudaStream_t stream);
void gram_tc_dims(int na, long long ns, int precision, int* na_pad, long long* ld);
int launch_gram_stage(const double* store, int sr_size, long long ns, const int* map, int na, const double* mean,
                      const double* cs, int precision, void* staged, cudaStream_t stream);
int launch_gram_tc(const void* staged, int na, long long ns, int precision, float* G, int ldg, unsigned* status,
                   cudaStream_t stream);
int launch_gather_active(const double* store, int sr_size, long long ns, const int* map, int na,
                         double* oa, cudaStream_t stream);
int launch_sr_cg(CgArgs a, cudaStream_t stream);
int cg_grid_blocks(long long ns, int na);
int low_lda(int na, int kind);
int cg_grid_blocks_kind(long long ns, int na, int kind);
int cg_nchunk(long long ns, int na, int kind, int blocks);
int launch_gather_active_low(const double* store, int sr_size, long long ns, const int* map, int na,
                             const double* mean, const double* cs, int kind, void* out, cudaStream_t stream);
int launch_stage(const DevModel& m, const StageBufs& b, int op, int msa, int msb, int rsa_old, int rsb_old,
                 unsigned* status, cudaStream_t stream);
int launch_gram(const double* store, int n, long long ns, double inv_w, double* oo, cudaStream_t stream);
int launch_assemble_s_gram(const float* g, int ldg, const double* cs, const double* var, int na, double inv_wc,
                           double sta_del, double* s, cudaStream_t stream);
int launch_assemble_s(const double* oo, int n, const int* map, int na, double ratio_diag, double* s,
                      cudaStream_t stream);
int launch_cholesky_solve(double* a, int n, double* b, int* info_dev, cudaStream_t stream);
int local_product_chunks(long long ns, int na);
int launch_local_product(const double* oa, long long ns, int na, const double* v, double* z, double* y,
                         double* part, cudaStream_t stream);

// K0: SlaterElm[q][rs_i][rs_j] from the Slater parameters (update_slater_elm,
// crates/mvmc-core/src/slater_update.rs:17-120).
__global__ void k_slater_table(int ns, int nqp, int nleg, int nmp, const double* __restrict__ f,
                               const int* __restrict__ orb_idx, const int* __restrict__ orb_sgn,
                               const int* __restrict__ trans, const int* __restrict__ trans_sgn,
                               const double* __restrict__ spgl, double* __restrict__ out,
                               float* __restrict__ out32) {
  const int ns2 = 2 * ns;
  const long long total = static_cast<long long>(nqp) * ns * ns;
  for (long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; k < total;
       k += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int qp = static_cast<int>(k / (static_cast<long long>(ns) * ns));
    const int rem = static_cast<int>(k - static_cast<long long>(qp) * ns * ns);
    const int ri = rem / ns, rj = rem - ri * ns;
    const int mpidx = (qp % (nleg * nmp)) / nleg, spidx = qp % nleg;
    const double cs = spgl[spidx], cc = spgl[nleg + spidx], ss = spgl[2 * nleg + spidx];
    const int tri = trans[mpidx * ns + ri], trj = trans[mpidx * ns + rj];
    const int qpsgn = trans_sgn[mpidx * ns + ri] * trans_sgn[mpidx * ns + rj];
    const int iij = orb_idx[tri * ns + trj], iji = orb_idx[trj * ns + tri];
    double* p = out + static_cast<size_t>(qp) * ns2 * ns2;
    float* p32 = out32 + static_cast<size_t>(qp) * ns2 * ns2;
    double v00 = 0, v01 = 0, v10 = 0, v11 = 0;
    if (iij >= 0 && iji >= 0) {
      // separately rounded products and sums (no FMA): the table equals the host's
      // build_slater_table bit for bit
      const double sij = __dmul_rn(f[iij], static_cast<double>(orb_sgn[tri * ns + trj] * qpsgn));
      const double sji = __dmul_rn(f[iji], static_cast<double>(orb_sgn[trj * ns + tri] * qpsgn));
      v00 = __dmul_rn(-__dsub_rn(sij, sji), cs);
      v01 = __dadd_rn(__dmul_rn(sij, cc), __dmul_rn(sji, ss));
      v10 = __dsub_rn(__dmul_rn(-sij, ss), __dmul_rn(sji, cc));
      v11 = __dmul_rn(__dsub_rn(sij, sji), cs);
    }
    p[ri * ns2 + rj] = v00;
    p[ri * ns2 + rj + ns] = v01;
    p[(ri + ns) * ns2 + rj] = v10;
    p[(ri + ns) * ns2 + rj + ns] = v11;
    p32[ri * ns2 + rj] = static_cast<float>(v00);
    p32[ri * ns2 + rj + ns] = static_cast<float>(v01);
    p32[(ri + ns) * ns2 + rj] = static_cast<float>(v10);
    p32[(ri + ns) * ns2 + rj + ns] = static_cast<float>(v11);
  }
}

}  // namespace mvmcb

using namespace mvmcb;

struct mvmc_b200_ctx {
  mvmc::Model m;
  mvmc_b200_options opt;
  int W = 1, S = 1;
  cudaStream_t stream = nullptr;
  DevModel dm{};
  DevWalkers dw{};
  std::vector<void*> allocs;
  double* d_f = nullptr;
  double* d_proj = nullptr;
  double* d_gsite = nullptr;
  double* d_jpair = nullptr;
  double* d_slater = nullptr;
  float* d_slater32 = nullptr;
  double* d_ostore = nullptr;
  double* d_eloc = nullptr;
  double* d_lpsi = nullptr;
  int* d_valid = nullptr;
  double* d_wsum = nullptr;
  double* d_tot = nullptr;
  double* d_gws = nullptr;
  double* d_cscr = nullptr;  // C-order measurement scratch (per walker), allocated on first use
  cudaEvent_t join_event = nullptr;  // orders device-buffer calls against the caller's stream
  void* d_staged = nullptr;  // Gram form: centred, column-scaled, transposed active samples
  size_t staged_cap = 0;
  float* d_gram = nullptr;   // Gram form: G = OᵀO (FP32, na × na)
  size_t gram_cap = 0;
  int* d_cscr_i = nullptr;
  int gws_blocks = 0;
  // SR-CG buffers
  double* d_oa = nullptr;
  size_t oa_cap = 0;  // doubles
  size_t y_cap = 0;
  double* d_cgvec = nullptr;  // mean, diag, g, x, r, d, q
  size_t cgvec_cap = 0;
  double* d_y = nullptr;
  double* d_part = nullptr;
  size_t part_cap = 0;
  double* d_red = nullptr;
  double* d_scal = nullptr;
  int* d_map = nullptr;
  size_t map_cap = 0;
  // direct SR buffers
  double* d_oo = nullptr;
  size_t oo_cap = 0;
  double* d_smat = nullptr;
  size_t smat_cap = 0;
  int* d_info = nullptr;
  // walker-sharded SR: compact active columns and the product buffers
  int shard_na = 0;
  double* d_shard_vec = nullptr;  // v, z (2·na)
  size_t shard_vec_cap = 0;
  double* d_shard_part = nullptr;
  size_t shard_part_cap = 0;
  // PhysCal Green functions: per-sample rows, the TwoBodyGEx factor pairs and the result
  double* d_gval = nullptr;
  size_t gval_cap = 0;
  int* d_gex = nullptr;
  double* d_gout = nullptr;
  double* d_gpart = nullptr;  // [chunks][outputs] walker-chunk partial sums
  int n_one = 0, n_ex = 0;
  std::vector<double> tot;  // host copy of the last reduction
  long long h2d = 0, d2h = 0;  // bytes copied across the host boundary
  bool sampled = false, measured = false;

  template <typename T>
  T* alloc(size_t count) {
    void* p = nullptr;
    if (count == 0) count = 1;
    if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess)
      throw std::runtime_error("cudaMalloc of " + std::to_string(count * sizeof(T)) + " bytes failed");
    allocs.push_back(p);
    return static_cast<T*>(p);
  }
  template <typename T>
  T* upload(const std::vector<T>& v) {
    T* p = alloc<T>(v.size());
    if (!v.empty() && cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
      throw std::runtime_error("cudaMemcpy upload failed");
    return p;
  }
  ~mvmc_b200_ctx() {
    for (void* p : allocs) cudaFree(p);
    if (join_event) cudaEventDestroy(join_event);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

void upload_parameters(mvmc_b200_ctx* c) {
  const mvmc::Model& m = c->m;
  const int ns = m.nsite;
  std::vector<double> proj = m.gutz;
  proj.insert(proj.end(), m.jast.begin(), m.jast.end());
  std::vector<double> gsite(ns, 0.0), jpair(static_cast<size_t>(ns) * ns, 0.0);
  for (int r = 0; r < ns; ++r) {
    const int g = m.gutz_idx[r];
    if (m.n_gutz > 0 && g >= 0 && g < m.n_gutz) gsite[r] = m.gutz[g];
  }
  for (int a = 0; a < ns; ++a)
    for (int b = 0; b < ns; ++b) {
      if (a == b || m.n_jast == 0) continue;
      const int j = m.jast_idx[std::min(a, b) * ns + std::max(a, b)];
      if (j >= 0 && j < m.n_jast) jpair[static_cast<size_t>(a) * ns + b] = m.jast[j];
    }
  check(cudaMemcpyAsync(c->d_f, m.slater.data(), sizeof(double) * std::max<size_t>(1, m.slater.size()),
                        cudaMemcpyHostToDevice, c->stream), "upload f");
  if (!proj.empty())
    check(cudaMemcpyAsync(c->d_proj, proj.data(), sizeof(double) * proj.size(), cudaMemcpyHostToDevice, c->stream),
          "upload proj");
  check(cudaMemcpyAsync(c->d_gsite, gsite.data(), sizeof(double) * ns, cudaMemcpyHostToDevice, c->stream), "upload gsite");
  check(cudaMemcpyAsync(c->d_jpair, jpair.data(), sizeof(double) * jpair.size(), cudaMemcpyHostToDevice, c->stream),
        "upload jpair");
  c->h2d += static_cast<long long>(sizeof(double)) *
            (std::max<size_t>(1, m.slater.size()) + proj.size() + gsite.size() + jpair.size());
  const long long total = static_cast<long long>(m.nqp) * ns * ns;
  const int grid = static_cast<int>(std::min<long long>((total + 255) / 256, 148LL * 16));
  k_slater_table<<<std::max(1, grid), 256, 0, c->stream>>>(
      ns, m.nqp, std::max(1, m.nsp_gauss_leg), m.mp_trans(), c->d_f, c->dm.orb_idx, c->dm.orb_sgn, c->dm.trans,
      c->dm.trans_sgn, c->dm.spgl, c->d_slater, c->d_slater32);
  check(cudaGetLastError(), "slater table kernel");
  check(cudaStreamSynchronize(c->stream), "parameter upload");
}

// Green tables of the PhysCal measurement. The one-body list is the output list followed
// by the one-body values that TwoBodyG terms with coincident indices reduce to (the one(...)
// calls of green_func2_impl, observables.rs:700-745); TwoBodyG terms without a coincidence
// get a two-hop slot.
void build_green_tables(mvmc_b200_ctx* c) {
  const mvmc::Model& m = c->m;
  std::vector<mvmc::GreenOneTerm> one = m.green_one;
  auto ref_of = [&](int a, int b, int sp) {
    const mvmc::GreenOneTerm t{a, sp, b, sp};
    auto it = std::find(one.begin(), one.end(), t);
    if (it != one.end()) return static_cast<int>(it - one.begin());
    one.push_back(t);
    return static_cast<int>(one.size()) - 1;
  };
  std::vector<int> gtwo, ggen;
  for (const auto& t : m.green_two) {
    const int ri = t.i, rj = t.j, rk = t.k, rl = t.l, s = t.si, u = t.sk;
    int ref = -1, gen = -1;
    bool general = false;
    if (s == u) {
      if (rk == rl) ref = ref_of(ri, rj, s);
      else if (rj == rl) {}
      else if (ri == rl) { if (rj != rk) ref = ref_of(rk, rj, s); }
      else if (rj == rk) ref = ref_of(ri, rl, s);
      else if (ri == rk) {}
      else if (ri == rj) ref = ref_of(rk, rl, s);
      else general = true;
    } else if (rk == rl) {
      if (ri != rj) ref = ref_of(ri, rj, s);
    } else if (ri == rj) {
      ref = ref_of(rk, rl, u);
    } else {
      general = true;
    }
    if (general) {
      gen = static_cast<int>(ggen.size() / 6);
      ggen.insert(ggen.end(), {ri, rj, rk, rl, s, u});
    }
    gtwo.insert(gtwo.end(), {ri, rj, rk, rl, s, u, ref, gen});
  }
  std::vector<int> gone, gex;
  for (const auto& t : one) gone.insert(gone.end(), {t.i, t.si, t.j, t.sj});
  // dense one-body lists (at least half of the Ns² same-spin pairs of a spin on average):
  // the per-plane product over all (empty site, electron) pairs
  const int ns = m.nsite;
  std::vector<int> term_of(2 * static_cast<size_t>(ns) * ns, -1), first(one.size());
  int distinct = 0;
  for (size_t k = 0; k < one.size(); ++k) {
    const auto& t = one[k];
    first[k] = static_cast<int>(k);
    if (t.si != t.sj || t.i == t.j) continue;
    int& slot = term_of[(static_cast<size_t>(t.si) * ns + t.i) * ns + t.j];
    if (slot < 0) {
      slot = static_cast<int>(k);
      ++distinct;
    } else {
      first[k] = slot;
    }
  }
  DevModel& dmg = c->dm;
  dmg.gdense = 2 * distinct >= ns * ns ? 1 : 0;
  if (const char* f = std::getenv("MVMC_B200_GREEN_DENSE")) dmg.gdense = std::atoi(f) != 0 ? 1 : 0;
  dmg.gterm_of = c->upload(term_of);
  dmg.gfirst = c->upload(first);
  for (const auto& p : m.green_two_ex) gex.insert(gex.end(), {p.first, p.second});
  DevModel& dm = c->dm;
  dm.ngone = static_cast<int>(one.size());
  dm.ngtwo = static_cast<int>(m.green_two.size());
  dm.nggen = static_cast<int>(ggen.size() / 6);
  dm.gw = dm.ngone + dm.ngtwo + dm.nggen;
  dm.gone = c->upload(gone);
  dm.gtwo = c->upload(gtwo);
  dm.ggen = c->upload(ggen);
  c->d_gex = c->upload(gex);
  c->n_one = static_cast<int>(m.green_one.size());
  c->n_ex = static_cast<int>(m.green_two_ex.size());
  c->d_gout = c->alloc<double>(c->n_one + c->n_ex + dm.ngtwo);
  c->d_gpart = c->alloc<double>(static_cast<size_t>(green_chunks(c->W)) * (c->n_one + c->n_ex + dm.ngtwo));
}

// physcal_zqp (PhysCal, prepare_phys_cal_from_namelist run.rs:555-737): every walker still
// consumes its initial-parameter draws, then the fixed parameters are read from zqp_opt.dat
// and synchronised without the Gutzwiller/Jastrow shift, and NMPTrans is taken by magnitude.
void build_context(mvmc_b200_ctx* c, const char* namelist, const char* initial_def, const mvmc_b200_options& opt,
                   const char* physcal_zqp = nullptr) {
  c->opt = opt;
  check(cudaSetDevice(opt.device), "cudaSetDevice");
  check(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  mvmc::Model& m = c->m;
  m = mvmc::read_expert(namelist);
  c->W = std::max(1, opt.walkers);
  c->S = opt.saved_per_walker > 0 ? opt.saved_per_walker : m.nvmc_sample;
  if (opt.precision != 64 && opt.precision != 32) throw std::runtime_error("precision must be 64 or 32");
  if (opt.sr_precision != 0 && opt.sr_precision != 64 && opt.sr_precision != 32 && opt.sr_precision != 16)
    throw std::runtime_error("sr_precision must be 0, 64, 32 or 16");
  if (!(opt.refresh_guard >= 0.0 && opt.refresh_guard < 1.0))
    throw std::runtime_error("refresh_guard must lie in [0, 1)");
  // walker streams: seed RndSeed + w, each consuming init_parameter draws (multichain.rs:88)
  const long long base = opt.seed >= 0 ? opt.seed : m.rnd_seed;
  std::vector<uint32_t> sf(static_cast<size_t>(c->W) * kSfmtN32);
  std::vector<int> sf_idx(c->W);
  std::vector<unsigned long long> draws(c->W);
  for (int w = 0; w < c->W; ++w) {
    const long long s = base + w;
    if (s < 0 || s > 0xffffffffLL) throw std::runtime_error("walker seed outside the UInt32 range");
    uint32_t* st = sf.data() + static_cast<size_t>(w) * kSfmtN32;
    sfmt_seed(st, &sf_idx[w], static_cast<uint32_t>(s));
    SfmtRef rng{st, &sf_idx[w], &draws[w]};
    mvmc::Model tmp = m;
    mvmc::init_parameter(tmp, [&]() { return rng.real2(); });
    if (w == 0) {
      m.gutz = tmp.gutz;
      m.jast = tmp.jast;
      m.slater = tmp.slater;
    }
  }
  if (physcal_zqp) {
    std::string why;
    if (!mvmc::read_para_triples(m, physcal_zqp, &why)) throw std::runtime_error(std::string("zqp_opt.dat: ") + why);
    mvmc::sync_modified_parameter(m, false);
    if (m.nmp_trans < 0) m.nmp_trans = -m.nmp_trans;
    m.calc_mode = 1;
  } else {
    if (initial_def && *initial_def) {
      std::string why;
      if (!mvmc::read_para_triples(m, initial_def, &why)) throw std::runtime_error(std::string("initial.def: ") + why);
    }
    mvmc::sync_modified_parameter(m, true);
  }
  mvmc::init_qp_weight(m);

  const int ns = m.nsite, n = m.nsize(), ns2 = 2 * ns, nqp = m.nqp, nproj = m.nproj();
  DevModel& dm = c->dm;
  dm.ns = ns; dm.ne = m.ne; dm.n = n; dm.ns2 = ns2; dm.nqp = nqp; dm.nproj = nproj;
  dm.n_gutz = m.n_gutz; dm.n_jast = m.n_jast; dm.norb = m.n_orb;
  dm.nleg = std::max(1, m.nsp_gauss_leg); dm.nmp = m.mp_trans(); dm.nex_path = m.nex_update_path;
  dm.warmup = m.nvmc_warmup; dm.interval = m.nvmc_interval; dm.saved = c->S;
  dm.sr_size = m.sr_size();
  // projection / orbital / translation tables
  std::vector<int> trans(static_cast<size_t>(dm.nmp) * ns), trans_sgn(trans.size());
  for (int mp = 0; mp < dm.nmp; ++mp)
    for (int r = 0; r < ns; ++r) mvmc::translated_site(m, r, mp, &trans[mp * ns + r], &trans_sgn[mp * ns + r]);
  std::vector<double> spgl;
  spgl.insert(spgl.end(), m.spgl_cs.begin(), m.spgl_cs.end());
  spgl.insert(spgl.end(), m.spgl_cc.begin(), m.spgl_cc.end());
  spgl.insert(spgl.end(), m.spgl_ss.begin(), m.spgl_ss.end());
  std::vector<int> tterm;
  std::vector<double> tval;
  for (const auto& t : m.transfer) {
    if (t.i < 0 || t.j < 0 || t.i >= ns || t.j >= ns) continue;
    tterm.insert(tterm.end(), {t.i, t.si, t.j, t.sj});
    tval.push_back(t.t);
  }
  std::vector<int> intra_i, inter_ij, hund_ij;
  std::vector<double> intra_v, inter_v, hund_v;
  for (const auto& t : m.coulomb_intra) if (t.i >= 0 && t.i < ns) { intra_i.push_back(t.i); intra_v.push_back(t.v); }
  for (const auto& t : m.coulomb_inter) if (t.i >= 0 && t.j >= 0 && t.i < ns && t.j < ns) { inter_ij.insert(inter_ij.end(), {t.i, t.j}); inter_v.push_back(t.v); }
  for (const auto& t : m.hund) if (t.i >= 0 && t.j >= 0 && t.i < ns && t.j < ns) { hund_ij.insert(hund_ij.end(), {t.i, t.j}); hund_v.push_back(t.v); }
  dm.nterm = static_cast<int>(tval.size());
  dm.nintra = static_cast<int>(intra_v.size());
  dm.ninter = static_cast<int>(inter_v.size());
  dm.nhund = static_cast<int>(hund_v.size());
  dm.qpw = c->upload(m.qp_weight);
  dm.gutz_idx = c->upload(m.gutz_idx);
  dm.jast_idx = c->upload(m.jast_idx);
  dm.orb_idx = c->upload(m.orb_idx);
  dm.orb_sgn = c->upload(m.orb_sgn);
  dm.trans = c->upload(trans);
  dm.trans_sgn = c->upload(trans_sgn);
  dm.spgl = c->upload(spgl);
  // Slater-derivative site pairs by orbital (deterministic O_k of the packed measurement)
  {
    std::vector<std::vector<int>> by_orb(std::max(0, m.n_orb));
    for (int a = 0; a < ns; ++a)
      for (int b = 0; b < ns; ++b) {
        const int k = m.orb_idx[a * ns + b];
        if (k < 0 || k >= m.n_orb) continue;
        by_orb[k].push_back((a << 16) | (b << 1) | (m.orb_sgn[a * ns + b] < 0 ? 1 : 0));
      }
    std::vector<int> off(1, 0), ent;
    for (const auto& v : by_orb) {
      ent.insert(ent.end(), v.begin(), v.end());
      off.push_back(static_cast<int>(ent.size()));
    }
    std::vector<int> tinv(trans.size(), -1);
    bool perm = true;
    for (int mp = 0; mp < dm.nmp && perm; ++mp)
      for (int r = 0; r < ns; ++r) {
        const int t = trans[mp * ns + r];
        if (t < 0 || t >= ns || tinv[mp * ns + t] >= 0) {
          perm = false;
          break;
        }
        tinv[mp * ns + t] = r;
      }
    if (!ent.empty() && perm) {
      dm.orb_off = c->upload(off);
      dm.orb_ent = c->upload(ent);
      dm.trans_inv = c->upload(tinv);
    }
  }
  dm.tterm = c->upload(tterm);
  dm.tval = c->upload(tval);
  dm.intra_i = c->upload(intra_i);
  dm.intra_v = c->upload(intra_v);
  dm.inter_ij = c->upload(inter_ij);
  dm.inter_v = c->upload(inter_v);
  dm.hund_ij = c->upload(hund_ij);
  dm.hund_v = c->upload(hund_v);
  c->d_f = c->alloc<double>(m.n_orb);
  c->d_proj = c->alloc<double>(nproj);
  c->d_gsite = c->alloc<double>(ns);
  c->d_jpair = c->alloc<double>(static_cast<size_t>(ns) * ns);
  c->d_slater = c->alloc<double>(static_cast<size_t>(nqp) * ns2 * ns2);
  c->d_slater32 = c->alloc<float>(static_cast<size_t>(nqp) * ns2 * ns2);
  dm.slater = c->d_slater;
  dm.slater32 = c->d_slater32;
  dm.proj = c->d_proj;
  dm.gutz_site = c->d_gsite;
  dm.jast_pair = c->d_jpair;

  // walkers
  DevWalkers& dw = c->dw;
  const int W = c->W, S = c->S;
  dw.W = W;
  dw.sfmt = c->upload(sf);
  dw.sfmt_idx = c->upload(sf_idx);
  dw.draws = c->upload(draws);
  dw.ele_idx = c->alloc<int>(static_cast<size_t>(W) * n);
  dw.ele_cfg = c->alloc<int>(static_cast<size_t>(W) * ns2);
  dw.ele_num = c->alloc<int>(static_cast<size_t>(W) * ns2);
  dw.proj_cnt = c->alloc<int>(static_cast<size_t>(W) * std::max(1, nproj));
  dw.burn = c->alloc<int>(W);
  check(cudaMemset(dw.burn, 0, sizeof(int) * W), "memset burn");
  dw.pf = c->alloc<double>(static_cast<size_t>(W) * nqp);
  dw.counter = c->alloc<long long>(static_cast<size_t>(W) * 6);
  dw.s_idx = c->alloc<int>(static_cast<size_t>(W) * S * n);
  dw.s_cfg = c->alloc<int>(static_cast<size_t>(W) * S * ns2);
  dw.s_num = c->alloc<int>(static_cast<size_t>(W) * S * ns2);
  dw.s_cnt = c->alloc<int>(static_cast<size_t>(W) * S * std::max(1, nproj));
  dw.status = c->alloc<unsigned>(1);
  check(cudaMemset(dw.status, 0, sizeof(unsigned)), "memset status");
  dw.refresh_sweeps = opt.refresh_sweeps;
  dw.drift = c->alloc<double>(W);
  check(cudaMemset(dw.drift, 0, sizeof(double) * W), "memset drift");
  dw.nrefresh = c->alloc<long long>(2 * static_cast<size_t>(W));
  check(cudaMemset(dw.nrefresh, 0, sizeof(long long) * 2 * W), "memset refresh counts");
  dw.refresh_guard = opt.refresh_guard;
  dw.timers = nullptr;
  if (const char* t = std::getenv("MVMC_B200_TIMERS")) {
    if (std::strcmp(t, "1") == 0) {
      dw.timers = c->alloc<unsigned long long>(static_cast<size_t>(W) * kPhCount);
      check(cudaMemset(dw.timers, 0, sizeof(unsigned long long) * W * kPhCount), "memset timers");
    }
  }
  int dev = 0, limit = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&limit, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t nn = static_cast<size_t>(n) * n;
  const bool smem = sample_planes_in_smem(dm, opt.precision, limit);
  dw.inv = nullptr;
  dw.ws64 = nullptr;
  if (!smem) {
    if (opt.precision == 64) dw.inv = c->alloc<double>(static_cast<size_t>(W) * nqp * nn);
    else dw.inv = c->alloc<float>(static_cast<size_t>(W) * nqp * nn);
  }
  // FP64 sweep buffers of walkers whose buffers are not in shared memory (two per walker)
  dw.ws64 = c->alloc<double>(static_cast<size_t>(W) * 2 * nn);
  // resident measurement (FP64 path): the sampler's Pf and X⁻¹ at every save point
  if (opt.measure_resident && opt.precision == 64 && !opt.c_order) {
    dw.s_inv = c->alloc<double>(static_cast<size_t>(W) * S * nqp * nn);
    dw.s_pf = c->alloc<double>(static_cast<size_t>(W) * S * nqp);
    dm.rinv = dw.s_inv;
    dm.rpf = dw.s_pf;
  }
  // measurement
  const size_t rows = static_cast<size_t>(W) * S;
  c->d_ostore = c->alloc<double>(rows * dm.sr_size);
  c->d_eloc = c->alloc<double>(rows);
  c->d_lpsi = c->alloc<double>(rows);
  c->d_valid = c->alloc<int>(rows);
  c->d_wsum = c->alloc<double>(static_cast<size_t>(W) * (5 + 3 * dm.sr_size));
  c->d_tot = c->alloc<double>(5 + 3 * dm.sr_size);
  c->gws_blocks = std::min<int>(static_cast<int>(rows), sms * 8);
  c->d_gws = c->alloc<double>(static_cast<size_t>(c->gws_blocks) * 2 * nn);
  c->d_red = c->alloc<double>(4096);
  c->d_scal = c->alloc<double>(8);
  build_green_tables(c);
  upload_parameters(c);
}

template <typename F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const std::invalid_argument& e) {
    mvmcb::set_last_error(e.what());
    return MVMC_B200_EARG;
  } catch (const std::exception& e) {
    mvmcb::set_last_error(e.what());
    const std::string what = e.what();
    if (what.find("cuda") != std::string::npos || what.find("CUDA") != std::string::npos) return MVMC_B200_ECUDA;
    return MVMC_B200_EMODEL;
  }
}

int do_measure(mvmc_b200_ctx* c) {
  const int rows = c->W * c->S;
  int rc;
  if (c->opt.c_order) {
    // parity mode: one thread per walker in the CPU path's operation order (csrc/corder.cu)
    if (!c->d_cscr) {
      long long ds = 0, is = 0;
      corder_scratch_sizes(c->dm, &ds, &is);
      c->d_cscr = c->alloc<double>(static_cast<size_t>(c->W) * ds);
      c->d_cscr_i = c->alloc<int>(static_cast<size_t>(c->W) * is);
    }
    rc = launch_measure_corder(c->dm, c->W, c->S, c->dw.s_idx, c->dw.s_cfg, c->dw.s_num, c->dw.s_cnt, c->d_ostore,
                               c->d_eloc, c->d_lpsi, c->d_valid, c->d_wsum, c->d_cscr, c->d_cscr_i, c->stream);
    if (rc != kOk) return rc;
    rc = launch_reduce_totals(c->dm, c->W, c->d_wsum, c->d_tot, c->stream);
  } else {
    rc = launch_measure(c->dm, c->dw.s_idx, c->dw.s_cfg, c->dw.s_num, c->dw.s_cnt, rows, c->d_gws, c->gws_blocks,
                        c->d_ostore, c->d_eloc, c->d_lpsi, c->d_valid, nullptr, c->dw.status, c->stream);
    if (rc != kOk) return rc;
    rc = launch_reduce(c->dm, c->W, c->S, c->d_ostore, c->d_eloc, c->d_valid, c->dw.s_num, c->d_wsum, c->d_tot,
                       c->stream);
  }
  if (rc != kOk) return rc;
  c->tot.assign(5 + 3 * c->dm.sr_size, 0.0);
  check(cudaMemcpyAsync(c->tot.data(), c->d_tot, sizeof(double) * c->tot.size(), cudaMemcpyDeviceToHost, c->stream),
        "download reduction");
  c->d2h += static_cast<long long>(sizeof(double) * c->tot.size());
  check(cudaStreamSynchronize(c->stream), "measure");
  c->measured = true;
  return kOk;
}

// PhysCal measurement of the saved samples (accumulate_observables with NVMCCalMode 1,
// run.rs:3300-3420): energies and Green functions, no O rows. tot[0..4] receives
// Wc, <E>, <E^2>, <Sz>, <Sz^2>; gout the Green functions (one-body, TwoBodyGEx, TwoBodyG).
int do_measure_green(mvmc_b200_ctx* c, std::vector<double>& gout) {
  const size_t rows = static_cast<size_t>(c->W) * c->S;
  const size_t need = rows * std::max(1, c->dm.gw);
  if (need > c->gval_cap) {
    if (c->d_gval) {
      check(cudaFree(c->d_gval), "cudaFree");
      c->allocs.erase(std::find(c->allocs.begin(), c->allocs.end(), static_cast<void*>(c->d_gval)));
    }
    c->d_gval = c->alloc<double>(need);
    c->gval_cap = need;
  }
  int rc = launch_measure(c->dm, c->dw.s_idx, c->dw.s_cfg, c->dw.s_num, c->dw.s_cnt, static_cast<int>(rows), c->d_gws,
                          c->gws_blocks, nullptr, c->d_eloc, c->d_lpsi, c->d_valid, c->d_gval, c->dw.status,
                          c->stream);
  if (rc != kOk) return rc;
  DevModel energy_only = c->dm;
  energy_only.sr_size = 0;
  rc = launch_reduce(energy_only, c->W, c->S, nullptr, c->d_eloc, c->d_valid, c->dw.s_num, c->d_wsum, c->d_tot,
                     c->stream);
  if (rc != kOk) return rc;
  rc = launch_green_reduce(c->dm, c->W, c->S, c->n_one, c->n_ex, c->d_gex, c->d_gval, c->d_valid, c->d_gpart,
                           c->d_gout, c->stream);
  if (rc != kOk) return rc;
  c->tot.assign(5, 0.0);
  check(cudaMemcpyAsync(c->tot.data(), c->d_tot, sizeof(double) * 5, cudaMemcpyDeviceToHost, c->stream),
        "download reduction");
  gout.assign(static_cast<size_t>(c->n_one) + c->n_ex + c->dm.ngtwo, 0.0);
  if (!gout.empty())
    check(cudaMemcpyAsync(gout.data(), c->d_gout, sizeof(double) * gout.size(), cudaMemcpyDeviceToHost, c->stream),
          "download Green functions");
  c->d2h += static_cast<long long>(sizeof(double) * (5 + gout.size()));
  check(cudaStreamSynchronize(c->stream), "measure Green functions");
  c->measured = false;  // the O rows were not written
  return kOk;
}

// Direct SR (NSRCG = 0): stochastic_opt_real_with_sr_info_timed (sr.rs:77-160) with the
// Gram, the S assembly and the Cholesky solve on the device.
int do_sr_direct(mvmc_b200_ctx* c, double* info_out) {
  mvmc::Model& m = c->m;
  const int size = m.sr_size(), npara = m.npara();
  const double wc = c->tot[0];
  const double* ho = c->tot.data() + 5;
  const long long ns = static_cast<long long>(c->W) * c->S;
  if (!c->d_info) c->d_info = c->alloc<int>(1);
  // sr_precision 16 / 32: the active S block from the tensor-core Gram of the centred,
  // column-scaled samples (BF16 / TF32 inputs, FP32 accumulation), ⟨O⟩ and ⟨O²⟩ from the
  // measurement sums; otherwise the FP64 Gram of every O column (the C order)
  const bool tc = !c->opt.c_order && (c->opt.sr_precision == 16 || c->opt.sr_precision == 32);
  int rc = kOk;
  std::vector<double> row0(size), diag(size);
  if (tc) {
    std::copy(c->tot.begin() + 5 + size, c->tot.begin() + 5 + 2 * size, row0.begin());
    std::copy(c->tot.begin() + 5 + 2 * size, c->tot.begin() + 5 + 3 * size, diag.begin());
  } else {
    const size_t nn = static_cast<size_t>(size) * size;
    if (nn > c->oo_cap) {
      c->d_oo = c->alloc<double>(nn);
      c->oo_cap = nn;
    }
    rc = launch_gram(c->d_ostore, size, ns, 1.0 / wc, c->d_oo, c->stream);
    if (rc != kOk) return rc;
    // row 0 (⟨O⟩) and the diagonal (⟨O²⟩) of OO for the redundancy cut and g
    check(cudaMemcpyAsync(row0.data(), c->d_oo, sizeof(double) * size, cudaMemcpyDeviceToHost, c->stream), "OO row 0");
    check(cudaMemcpy2DAsync(diag.data(), sizeof(double), c->d_oo, sizeof(double) * (size + 1), sizeof(double), size,
                            cudaMemcpyDeviceToHost, c->stream),
          "OO diagonal");
    check(cudaStreamSynchronize(c->stream), "gram");
    c->d2h += static_cast<long long>(sizeof(double) * 2 * size);
  }
  std::vector<double> s_diag(npara);
  for (int pi = 0; pi < npara; ++pi) s_diag[pi] = diag[pi + 1] - row0[pi + 1] * row0[pi + 1];
  bool any_nan = false;
  double vmax = 0.0;
  for (double v : s_diag) {
    if (std::isnan(v)) any_nan = true;
    vmax = std::fmax(vmax, v);
  }
  if (any_nan) vmax = NAN;
  const double cut = vmax * m.red_cut;
  auto optimised = [&](int comp) {
    return static_cast<size_t>(comp) < m.opt_flags.size() && m.opt_flags[comp] == 1;
  };
  std::vector<int> map;
  for (int pi = 0; pi < npara; ++pi)
    if (optimised(2 * pi) && !(s_diag[pi] < cut)) map.push_back(pi);
  if (info_out) std::fill(info_out, info_out + 9, 0.0);
  if (map.empty()) return 0;
  const int na = static_cast<int>(map.size());
  if (static_cast<size_t>(na) > c->map_cap) {
    c->d_map = c->alloc<int>(na);
    c->map_cap = na;
  }
  const size_t smat_need = static_cast<size_t>(na) * na + na;
  if (smat_need > c->smat_cap) {
    c->d_smat = c->alloc<double>(smat_need);
    c->smat_cap = smat_need;
  }
  std::vector<double> g(na);
  for (int si = 0; si < na; ++si) {
    const int pi = map[si] + 1;
    g[si] = -2.0 * m.step_dt * (ho[pi] - ho[0] * row0[pi]);
  }
  double* d_s = c->d_smat;
  double* d_g = c->d_smat + static_cast<size_t>(na) * na;
  check(cudaMemcpyAsync(c->d_map, map.data(), sizeof(int) * na, cudaMemcpyHostToDevice, c->stream), "upload map");
  check(cudaMemcpyAsync(d_g, g.data(), sizeof(double) * na, cudaMemcpyHostToDevice, c->stream), "upload g");
  c->h2d += static_cast<long long>(sizeof(int) * na + sizeof(double) * na);
  if (tc) {
    // active ⟨O⟩, variance and column scales (the standard deviations) for the staging
    const int prec = c->opt.sr_precision;
    if (static_cast<size_t>(8) * na > c->cgvec_cap) {
      c->d_cgvec = c->alloc<double>(static_cast<size_t>(8) * na);
      c->cgvec_cap = static_cast<size_t>(8) * na;
    }
    std::vector<double> v3(static_cast<size_t>(3) * na);
    for (int si = 0; si < na; ++si) {
      const double var = s_diag[map[si]];
      v3[si] = row0[map[si] + 1];
      v3[na + si] = var;
      v3[2 * na + si] = (std::isfinite(var) && var > 0.0) ? std::sqrt(var) : 1.0;
    }
    double* d_mean = c->d_cgvec;
    double* d_var = c->d_cgvec + na;
    double* d_cs = c->d_cgvec + 7 * static_cast<size_t>(na);
    check(cudaMemcpyAsync(d_mean, v3.data(), sizeof(double) * 2 * na, cudaMemcpyHostToDevice, c->stream),
          "upload mean, var");
    check(cudaMemcpyAsync(d_cs, v3.data() + 2 * na, sizeof(double) * na, cudaMemcpyHostToDevice, c->stream),
          "upload column scales");
    c->h2d += static_cast<long long>(sizeof(double) * 3 * na);
    int na_pad = 0;
    long long ld = 0;
    gram_tc_dims(na, ns, prec, &na_pad, &ld);
    const size_t staged = static_cast<size_t>(na_pad) * ld * (prec == 16 ? 2 : 4);
    if (staged > c->staged_cap) {
      c->d_staged = c->alloc<unsigned char>(staged);
      c->staged_cap = staged;
    }
    if (static_cast<size_t>(na) * na > c->gram_cap) {
      c->d_gram = c->alloc<float>(static_cast<size_t>(na) * na);
      c->gram_cap = static_cast<size_t>(na) * na;
    }
    rc = launch_gram_stage(c->d_ostore, size, ns, c->d_map, na, d_mean, d_cs, prec, c->d_staged, c->stream);
    if (rc != kOk) return rc;
    rc = launch_gram_tc(c->d_staged, na, ns, prec, c->d_gram, na, c->dw.status, c->stream);
    if (rc != kOk) return rc;
    rc = launch_assemble_s_gram(c->d_gram, na, d_cs, d_var, na, 1.0 / wc, m.sta_del, d_s, c->stream);
  } else {
    rc = launch_assemble_s(c->d_oo, size, c->d_map, na, 1.0 + m.sta_del, d_s, c->stream);
  }
  if (rc != kOk) return rc;
  rc = launch_cholesky_solve(d_s, na, d_g, c->d_info, c->stream);
  if (rc != kOk) return rc;
  int info = 0;
  check(cudaMemcpyAsync(&info, c->d_info, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "cholesky info");
  check(cudaMemcpyAsync(g.data(), d_g, sizeof(double) * na, cudaMemcpyDeviceToHost, c->stream), "download x");
  check(cudaStreamSynchronize(c->stream), "sr-direct");
  c->d2h += static_cast<long long>(sizeof(double) * na + sizeof(int));
  if (tc) {
    unsigned dst = 0;
    check(cudaMemcpy(&dst, c->dw.status, sizeof(unsigned), cudaMemcpyDeviceToHost), "status");
    if (dst & kDevTimeout) throw std::runtime_error("sr-direct: the tensor-core Gram timed out (cuda device wait)");
  }
  if (info != 0) return 1;
  for (double v : g)
    if (!std::isfinite(v)) return 1;
  // SRinfo in C's complex index space (real value, zero imaginary variance; sr.rs:309-360)
  double smax = s_diag[0], smin = s_diag[0];
  int opt_num = 0, cut_num = 0;
  for (int comp = 0; comp < 2 * npara; ++comp) {
    const double d = (comp & 1) ? 0.0 : s_diag[comp / 2];
    if (d > smax) smax = d;
    if (d < smin) smin = d;
  }
  for (int comp = 0; comp < 2 * npara; ++comp) {
    const double d = (comp & 1) ? 0.0 : s_diag[comp / 2];
    if (!optimised(comp)) ++opt_num;
    else if (d < smax * m.red_cut) ++cut_num;
  }
  int imax = 0;
  for (int i = 1; i < na; ++i)
    if (std::fabs(g[imax]) < std::fabs(g[i])) imax = i;
  if (info_out) {
    const double row[9] = {static_cast<double>(npara), static_cast<double>(na), static_cast<double>(opt_num),
                           static_cast<double>(cut_num), smax, smin, g[imax], static_cast<double>(2 * map[imax]), 0.0};
    std::copy(row, row + 9, info_out);
  }
  std::vector<double> p = mvmc::all_parameters(m);
  for (int si = 0; si < na; ++si) p[map[si]] += g[si];
  mvmc::set_all_parameters(m, p);
  mvmc::sync_modified_parameter(m, true);
  upload_parameters(c);
  return 0;
}

// stochastic_opt_cg_with_reducer (sr_cg.rs:201-490) around the device solve.
int do_sr_cg(mvmc_b200_ctx* c, double* info_out) {
  mvmc::Model& m = c->m;
  const int size = m.sr_size(), npara = m.npara();
  if (!c->measured) return MVMC_B200_ESTATE;
  if (m.nsrcg == 0) return do_sr_direct(c, info_out);
  if (m.rescale_smat) throw std::runtime_error("RescaleSmat is not supported by the device SR path");
  const double wc = c->tot[0];
  const double* ho = c->tot.data() + 5;
  const double* mean_all = c->tot.data() + 5 + size;
  const double* diag_all = c->tot.data() + 5 + 2 * size;
  std::vector<double> var(npara);
  for (int pi = 0; pi < npara; ++pi) var[pi] = diag_all[pi + 1] - mean_all[pi + 1] * mean_all[pi + 1];
  double vmax = -INFINITY, vmin = INFINITY;
  bool any_nan = false;
  for (double v : var) {
    if (std::isnan(v)) any_nan = true;
    vmax = std::fmax(vmax, v);
    vmin = std::fmin(vmin, v);
  }
  if (any_nan) vmax = vmin = NAN;
  const double threshold = vmax * m.red_cut;
  std::vector<int> map;
  int opt_cut = 0, diag_cut = 0;
  for (int pi = 0; pi < npara; ++pi) {
    const bool optimised = static_cast<size_t>(2 * pi) < m.opt_flags.size() && m.opt_flags[2 * pi] == 1;
    if (!optimised) ++opt_cut;
    else if (var[pi] < threshold) ++diag_cut;
    else map.push_back(pi);
  }
  if (info_out) std::fill(info_out, info_out + 9, 0.0);
  if (map.empty()) return 0;
  const int na = static_cast<int>(map.size());
  std::vector<double> vecs(static_cast<size_t>(3) * na);
  const double dt = 2.0 * m.step_dt;
  for (int si = 0; si < na; ++si) {
    const int idx = map[si] + 1;
    vecs[si] = mean_all[idx];
    vecs[na + si] = var[map[si]];
    vecs[2 * na + si] = -dt * (ho[idx] - ho[0] * mean_all[idx]);
  }
  const long long ns = static_cast<long long>(c->W) * c->S;
  // operator storage: 0 FP64 (C order), 1 FP32, 2 BF16 (centred, column-scaled)
  const int kind = c->opt.c_order ? 0 : (c->opt.sr_precision == 32 ? 1 : (c->opt.sr_precision == 16 ? 2 : 0));
  const size_t oa_need = kind == 0 ? static_cast<size_t>(ns) * na
                                   : (static_cast<size_t>(ns) * low_lda(na, kind) * (kind == 1 ? 4 : 2) + 7) / 8;
  if (oa_need > c->oa_cap) {
    c->d_oa = c->alloc<double>(oa_need);
    c->oa_cap = oa_need;
  }
  if (static_cast<size_t>(ns) > c->y_cap) {
    c->d_y = c->alloc<double>(ns);
    c->y_cap = static_cast<size_t>(ns);
  }
  if (static_cast<size_t>(8) * na > c->cgvec_cap) {
    c->d_cgvec = c->alloc<double>(static_cast<size_t>(8) * na);
    c->cgvec_cap = static_cast<size_t>(8) * na;
  }
  if (static_cast<size_t>(na) > c->map_cap) {
    c->d_map = c->alloc<int>(na);
    c->map_cap = na;
  }
  const int blocks = cg_grid_blocks_kind(ns, na, kind);
  const int nchunk = cg_nchunk(ns, na, kind, blocks);
  if (static_cast<size_t>(nchunk) * na > c->part_cap) {
    c->d_part = c->alloc<double>(static_cast<size_t>(nchunk) * na);
    c->part_cap = static_cast<size_t>(nchunk) * na;
  }
  check(cudaMemcpyAsync(c->d_map, map.data(), sizeof(int) * na, cudaMemcpyHostToDevice, c->stream), "upload map");
  if (kind != 0) {
    // column scales: the standard deviation of each active column (1 where it vanishes)
    vecs.resize(static_cast<size_t>(8) * na);
    for (int si = 0; si < na; ++si) {
      const double v = vecs[na + si];
      vecs[7 * static_cast<size_t>(na) + si] = (std::isfinite(v) && v > 0.0) ? std::sqrt(v) : 1.0;
    }
    check(cudaMemcpyAsync(c->d_cgvec + 7 * static_cast<size_t>(na), vecs.data() + 7 * static_cast<size_t>(na),
                          sizeof(double) * na, cudaMemcpyHostToDevice, c->stream), "upload column scales");
    c->h2d += static_cast<long long>(sizeof(double) * na);
  }
  check(cudaMemcpyAsync(c->d_cgvec, vecs.data(), sizeof(double) * 3 * na, cudaMemcpyHostToDevice, c->stream),
        "upload cg vectors");
  // Gram form: G = OlᵀOl on the tensor cores (BF16 for sr_precision 16, TF32 for 32)
  const bool gram = kind != 0 && c->opt.sr_gram != 0;
  int rc;
  if (gram) {
    const int prec = kind == 2 ? 16 : 32;
    int na_pad = 0;
    long long ld = 0;
    gram_tc_dims(na, ns, prec, &na_pad, &ld);
    const size_t staged = static_cast<size_t>(na_pad) * ld * (prec == 16 ? 2 : 4);
    if (staged > c->staged_cap) {
      c->d_staged = c->alloc<unsigned char>(staged);
      c->staged_cap = staged;
    }
    if (static_cast<size_t>(na) * na > c->gram_cap) {
      c->d_gram = c->alloc<float>(static_cast<size_t>(na) * na);
      c->gram_cap = static_cast<size_t>(na) * na;
    }
    rc = launch_gram_stage(c->d_ostore, size, ns, c->d_map, na, c->d_cgvec, c->d_cgvec + 7 * static_cast<size_t>(na),
                           prec, c->d_staged, c->stream);
    if (rc != kOk) return rc;
    rc = launch_gram_tc(c->d_staged, na, ns, prec, c->d_gram, na, c->dw.status, c->stream);
  } else {
    rc = kind == 0 ? launch_gather_active(c->d_ostore, size, ns, c->d_map, na, c->d_oa, c->stream)
                   : launch_gather_active_low(c->d_ostore, size, ns, c->d_map, na, c->d_cgvec,
                                              c->d_cgvec + 7 * static_cast<size_t>(na), kind, c->d_oa, c->stream);
  }
  if (rc != kOk) return rc;
  CgArgs a;
  a.O = c->d_oa;
  a.mean = c->d_cgvec;
  a.diag = c->d_cgvec + na;
  a.g = c->d_cgvec + 2 * na;
  a.x = c->d_cgvec + 3 * na;
  a.r = c->d_cgvec + 4 * na;
  a.d = c->d_cgvec + 5 * na;
  a.q = c->d_cgvec + 6 * na;
  a.y = c->d_y;
  a.part = c->d_part;
  a.red = c->d_red;
  a.scal = c->d_scal;
  a.ns = ns;
  a.na = na;
  a.nchunk = nchunk;
  a.max_iter = m.cg_max_iter > 0 ? m.cg_max_iter : na;
  a.diag_scale = m.diag_scale ? 1 : 0;
  a.inv_w = 1.0 / wc;
  a.shift = m.sta_del;
  a.tol = m.cg_tol;
  if (kind != 0) {
    a.Ol = gram ? static_cast<const void*>(c->d_gram) : static_cast<const void*>(c->d_oa);
    a.cs = c->d_cgvec + 7 * static_cast<size_t>(na);
    a.lda = gram ? na : low_lda(na, kind);
    a.o_kind = gram ? 3 : kind;
  }
  auto solve = [&]() { return c->opt.c_order ? launch_cg_corder(a, c->W, c->S, c->stream) : launch_sr_cg(a, c->stream); };
  rc = solve();
  if (rc != kOk) return rc;
  std::vector<double> x(na), scal(8);
  check(cudaMemcpyAsync(x.data(), a.x, sizeof(double) * na, cudaMemcpyDeviceToHost, c->stream), "download x");
  check(cudaMemcpyAsync(scal.data(), c->d_scal, sizeof(double) * 8, cudaMemcpyDeviceToHost, c->stream), "download scal");
  check(cudaStreamSynchronize(c->stream), "sr-cg");
  c->h2d += static_cast<long long>(sizeof(int) * na + sizeof(double) * 3 * na);
  c->d2h += static_cast<long long>(sizeof(double) * (na + 8));
  if (gram) {
    unsigned dst = 0;
    check(cudaMemcpy(&dst, c->dw.status, sizeof(unsigned), cudaMemcpyDeviceToHost), "status");
    if (dst & kDevTimeout) throw std::runtime_error("sr-cg: the tensor-core Gram timed out (cuda device wait)");
  }
  long long status = static_cast<long long>(scal[1]);
  long long info = status;
  if (status < 0) {
    const long long fallback_iter = std::max(-status - 1, 0LL);
    if (m.cg_fallback) {
      a.diag_scale = !a.diag_scale;
      rc = solve();
      if (rc != kOk) return rc;
      check(cudaMemcpyAsync(x.data(), a.x, sizeof(double) * na, cudaMemcpyDeviceToHost, c->stream), "download x");
      check(cudaMemcpyAsync(scal.data(), c->d_scal, sizeof(double) * 8, cudaMemcpyDeviceToHost, c->stream), "download");
      check(cudaStreamSynchronize(c->stream), "sr-cg fallback");
      info = -(fallback_iter + 1);
      if (static_cast<long long>(scal[1]) < 0 && m.cg_abort) throw std::runtime_error("fallback SR-CG failed");
    } else {
      if (m.cg_abort) throw std::runtime_error("SR-CG failed and fallback is disabled");
      info = -(fallback_iter + 1);
    }
  }
  int imax = 0;
  for (int i = 1; i < na; ++i)
    if (std::fabs(x[imax]) < std::fabs(x[i])) imax = i;
  if (info_out) {
    const double row[9] = {static_cast<double>(npara), static_cast<double>(na), static_cast<double>(opt_cut),
                           static_cast<double>(diag_cut), vmax, vmin, x[imax], static_cast<double>(map[imax]),
                           static_cast<double>(info)};
    std::copy(row, row + 9, info_out);
  }
  for (double v : x)
    if (!std::isfinite(v)) {
      if (m.cg_abort) throw std::runtime_error("SR-CG produced non-finite updates");
      return 1;
    }
  std::vector<double> p = mvmc::all_parameters(m);
  for (int si = 0; si < na; ++si) p[map[si]] += x[si];
  mvmc::set_all_parameters(m, p);
  mvmc::sync_modified_parameter(m, true);
  upload_parameters(c);
  return 0;
}

}  // namespace

extern "C" int mvmc_b200_create(const char* namelist, const char* initial_def, const mvmc_b200_options* opt,
                                mvmc_b200_ctx** out) {
  if (!namelist || !out) return MVMC_B200_EARG;
  *out = nullptr;
  mvmc_b200_options o;
  mvmc_b200_default_options(&o);
  if (opt) o = *opt;
  return guarded([&]() {
    auto* c = new mvmc_b200_ctx();
    try {
      build_context(c, namelist, initial_def, o);
    } catch (...) {
      delete c;
      throw;
    }
    *out = c;
    return MVMC_B200_OK;
  });
}

extern "C" void mvmc_b200_destroy(mvmc_b200_ctx* ctx) { delete ctx; }

extern "C" int mvmc_b200_dims(const mvmc_b200_ctx* c, int* dims) {
  if (!c || !dims) return MVMC_B200_EARG;
  const int v[8] = {c->m.nsite, c->m.ne, c->m.nqp, c->m.nproj(), c->m.npara(), c->S, c->W, c->m.n_orb};
  std::copy(v, v + 8, dims);
  return MVMC_B200_OK;
}

extern "C" int mvmc_b200_get_parameters(const mvmc_b200_ctx* c, double* params, int npara) {
  if (!c || !params || npara != c->m.npara()) return MVMC_B200_EARG;
  const std::vector<double> p = mvmc::all_parameters(c->m);
  std::copy(p.begin(), p.end(), params);
  return MVMC_B200_OK;
}

extern "C" int mvmc_b200_set_parameters(mvmc_b200_ctx* c, const double* params, int npara) {
  if (!c || !params || npara != c->m.npara()) return MVMC_B200_EARG;
  return guarded([&]() {
    mvmc::set_all_parameters(c->m, std::vector<double>(params, params + npara));
    upload_parameters(c);
    return MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_sample(mvmc_b200_ctx* c) {
  if (!c) return MVMC_B200_EARG;
  return guarded([&]() {
    int rc = launch_sample(c->dm, c->dw, c->opt.precision, c->stream);
    if (rc != kOk) return rc;
    check(cudaStreamSynchronize(c->stream), "sample");
    c->sampled = true;
    c->measured = false;
    return MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_get_samples(const mvmc_b200_ctx* c, int64_t* ele_idx, int64_t* ele_cfg, int64_t* ele_num,
                                     int64_t* proj_cnt, int64_t* counters, int64_t* draws) {
  if (!c) return MVMC_B200_EARG;
  return guarded([&]() {
    const size_t rows = static_cast<size_t>(c->W) * c->S;
    auto fetch = [&](const int* src, size_t count, int64_t* dst) {
      if (!dst) return;
      std::vector<int> tmp(count);
      check(cudaMemcpy(tmp.data(), src, sizeof(int) * count, cudaMemcpyDeviceToHost), "download samples");
      for (size_t k = 0; k < count; ++k) dst[k] = tmp[k];
    };
    fetch(c->dw.s_idx, rows * c->dm.n, ele_idx);
    fetch(c->dw.s_cfg, rows * c->dm.ns2, ele_cfg);
    fetch(c->dw.s_num, rows * c->dm.ns2, ele_num);
    fetch(c->dw.s_cnt, rows * c->dm.nproj, proj_cnt);
    if (counters) {
      std::vector<long long> tmp(static_cast<size_t>(c->W) * 6);
      check(cudaMemcpy(tmp.data(), c->dw.counter, sizeof(long long) * tmp.size(), cudaMemcpyDeviceToHost), "counters");
      std::copy(tmp.begin(), tmp.end(), counters);
    }
    if (draws) {
      std::vector<unsigned long long> tmp(c->W);
      check(cudaMemcpy(tmp.data(), c->dw.draws, sizeof(unsigned long long) * c->W, cudaMemcpyDeviceToHost), "draws");
      for (int w = 0; w < c->W; ++w) draws[w] = static_cast<int64_t>(tmp[w]);
    }
    return MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_measure(mvmc_b200_ctx* c, double* energy, double* ho, double* oo) {
  if (!c) return MVMC_B200_EARG;
  if (!c->sampled) return MVMC_B200_ESTATE;
  return guarded([&]() {
    int rc = do_measure(c);
    if (rc != kOk) return rc;
    const int size = c->dm.sr_size;
    if (energy) std::copy(c->tot.begin(), c->tot.begin() + 5, energy);
    if (ho) std::copy(c->tot.begin() + 5, c->tot.begin() + 5 + size, ho);
    if (oo) std::copy(c->tot.begin() + 5 + size, c->tot.begin() + 5 + 3 * size, oo);
    return MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_get_o_store(const mvmc_b200_ctx* c, double* o_store, long long count) {
  if (!c || !o_store) return MVMC_B200_EARG;
  const long long need = static_cast<long long>(c->W) * c->S * c->dm.sr_size;
  if (count < need) return MVMC_B200_EARG;
  return guarded([&]() {
    check(cudaMemcpy(o_store, c->d_ostore, sizeof(double) * need, cudaMemcpyDeviceToHost), "download O store");
    return MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_get_log_amplitudes(const mvmc_b200_ctx* c, double* log_psi, long long count) {
  if (!c || !log_psi) return MVMC_B200_EARG;
  const long long need = static_cast<long long>(c->W) * c->S;
  if (count < need) return MVMC_B200_EARG;
  if (!c->measured) return MVMC_B200_ESTATE;
  return guarded([&]() {
    check(cudaMemcpy(log_psi, c->d_lpsi, sizeof(double) * need, cudaMemcpyDeviceToHost), "download ln|psi|");
    return MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_get_local_energies(const mvmc_b200_ctx* c, double* e_loc, long long count) {
  if (!c || !e_loc) return MVMC_B200_EARG;
  const long long need = static_cast<long long>(c->W) * c->S;
  if (count < need) return MVMC_B200_EARG;
  return guarded([&]() {
    check(cudaMemcpy(e_loc, c->d_eloc, sizeof(double) * need, cudaMemcpyDeviceToHost), "download energies");
    return MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_sr_cg(mvmc_b200_ctx* c, double* sr_info) {
  if (!c) return MVMC_B200_EARG;
  return guarded([&]() { return do_sr_cg(c, sr_info); });
}

extern "C" int mvmc_b200_sampler_timers(const mvmc_b200_ctx* c, double* cycles) {
  if (!c || !cycles) return MVMC_B200_EARG;
  std::fill(cycles, cycles + kPhCount, 0.0);
  if (!c->dw.timers) return MVMC_B200_OK;
  return guarded([&]() {
    std::vector<unsigned long long> t(static_cast<size_t>(c->W) * kPhCount);
    check(cudaMemcpy(t.data(), c->dw.timers, sizeof(unsigned long long) * t.size(), cudaMemcpyDeviceToHost), "timers");
    for (int w = 0; w < c->W; ++w)
      for (int k = 0; k < kPhCount; ++k) cycles[k] += static_cast<double>(t[static_cast<size_t>(w) * kPhCount + k]);
    return MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_refresh_stats(const mvmc_b200_ctx* c, double* stats) {
  if (!c || !stats) return MVMC_B200_EARG;
  return guarded([&]() {
    std::vector<double> d(c->W);
    std::vector<long long> r(2 * static_cast<size_t>(c->W));
    check(cudaMemcpy(d.data(), c->dw.drift, sizeof(double) * c->W, cudaMemcpyDeviceToHost), "drift");
    check(cudaMemcpy(r.data(), c->dw.nrefresh, sizeof(long long) * r.size(), cudaMemcpyDeviceToHost), "refreshes");
    double mx = 0.0, sum = 0.0, sched = 0.0, guard = 0.0;
    for (int w = 0; w < c->W; ++w) {
      mx = std::max(mx, d[w]);
      sum += d[w];
      sched += static_cast<double>(r[2 * static_cast<size_t>(w)]);
      guard += static_cast<double>(r[2 * static_cast<size_t>(w) + 1]);
    }
    stats[0] = mx;
    stats[1] = sum / c->W;
    stats[2] = sched / c->W;
    stats[3] = guard / c->W;
    return MVMC_B200_OK;
  });
}

extern "C" void* mvmc_b200_stream(mvmc_b200_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

extern "C" int mvmc_b200_transfer_bytes(const mvmc_b200_ctx* c, long long* h2d, long long* d2h) {
  if (!c || !h2d || !d2h) return MVMC_B200_EARG;
  *h2d = c->h2d;
  *d2h = c->d2h;
  return MVMC_B200_OK;
}

extern "C" int mvmc_b200_status(mvmc_b200_ctx* c, unsigned* device_status) {
  if (!c || !device_status) return MVMC_B200_EARG;
  return guarded([&]() {
    check(cudaMemcpy(device_status, c->dw.status, sizeof(unsigned), cudaMemcpyDeviceToHost), "status");
    return MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_run_opt(const char* namelist, const char* initial_def, const char* out_dir,
                                 const mvmc_b200_options* opt, int nsteps) {
  if (!namelist || !out_dir) return MVMC_B200_EARG;
  mvmc_b200_ctx* c = nullptr;
  int rc = mvmc_b200_create(namelist, initial_def, opt, &c);
  if (rc != MVMC_B200_OK) return rc;
  rc = guarded([&]() {
    mvmc::Model& m = c->m;
    if (nsteps > 0) {
      m.nsr_opt_itr_step = nsteps;
      m.nsr_opt_itr_smp = std::min(m.nsr_opt_itr_smp, nsteps);
    }
    const int window_start = m.nsr_opt_itr_step - m.nsr_opt_itr_smp;
    std::vector<mvmc::OptPoint> window;
    bool first_info = true;
    for (int step = 0; step < m.nsr_opt_itr_step; ++step) {
      int r = launch_sample(c->dm, c->dw, c->opt.precision, c->stream);
      if (r != kOk) return r;
      c->sampled = true;
      r = do_measure(c);
      if (r != kOk) return r;
      const double* t = c->tot.data();
      mvmc::write_out_row(m, out_dir, step, mvmc::StepEnergy{t[1], t[2], t[3], t[4]});
      double info[9];
      const int sr = do_sr_cg(c, info);
      if (info[1] > 0) {
        mvmc::SrInfoRow row{static_cast<int>(info[0]), static_cast<int>(info[1]), static_cast<int>(info[2]),
                            static_cast<int>(info[3]), info[4], info[5], info[6], static_cast<int>(info[7]),
                            static_cast<int>(info[8])};
        mvmc::write_srinfo_row(out_dir, m, first_info, row);
        first_info = false;
      }
      if (sr != 0) throw std::runtime_error("SR failed at step " + std::to_string(step));
      if (step >= window_start) window.push_back({t[1], t[2], mvmc::all_parameters(m)});
    }
    mvmc::write_opt_files(m, out_dir, window);
    return MVMC_B200_OK;
  });
  mvmc_b200_destroy(c);
  return rc;
}

// ---------------------------------------------------------------------------------------
// PhysCal (NVMCCalMode 1): fixed parameters, energies and Green functions per data block
// (vmc_phys_cal_in_place_with_options_timed, crates/mvmc-core/src/run.rs:980-1156).
// ---------------------------------------------------------------------------------------
extern "C" int mvmc_b200_physcal_create(const char* namelist, const char* zqp_opt, const mvmc_b200_options* opt,
                                        mvmc_b200_ctx** out) {
  if (!namelist || !zqp_opt || !out) return MVMC_B200_EARG;
  *out = nullptr;
  mvmc_b200_options o;
  mvmc_b200_default_options(&o);
  if (opt) o = *opt;
  return guarded([&]() {
    auto* c = new mvmc_b200_ctx();
    try {
      build_context(c, namelist, nullptr, o, zqp_opt);
    } catch (...) {
      delete c;
      throw;
    }
    *out = c;
    return MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_green_dims(const mvmc_b200_ctx* c, int* dims) {
  if (!c || !dims) return MVMC_B200_EARG;
  const int v[5] = {c->n_one, c->n_ex, c->dm.ngtwo, c->m.data_qty_smp, c->m.data_idx_start};
  std::copy(v, v + 5, dims);
  return MVMC_B200_OK;
}

extern "C" int mvmc_b200_measure_green(mvmc_b200_ctx* c, double* energy, double* one, double* two_ex, double* two) {
  if (!c) return MVMC_B200_EARG;
  if (!c->sampled) return MVMC_B200_ESTATE;
  return guarded([&]() {
    std::vector<double> g;
    const int rc = do_measure_green(c, g);
    if (rc != kOk) return rc;
    if (energy) std::copy(c->tot.begin(), c->tot.begin() + 5, energy);
    if (one) std::copy(g.begin(), g.begin() + c->n_one, one);
    if (two_ex) std::copy(g.begin() + c->n_one, g.begin() + c->n_one + c->n_ex, two_ex);
    if (two) std::copy(g.begin() + c->n_one + c->n_ex, g.end(), two);
    return MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_run_physcal(const char* namelist, const char* zqp_opt, const char* out_dir,
                                     const mvmc_b200_options* opt) {
  if (!namelist || !zqp_opt || !out_dir) return MVMC_B200_EARG;
  mvmc_b200_ctx* c = nullptr;
  int rc = mvmc_b200_physcal_create(namelist, zqp_opt, opt, &c);
  if (rc != MVMC_B200_OK) return rc;
  rc = guarded([&]() {
    const mvmc::Model& m = c->m;
    for (int b = 0; b < std::max(0, m.data_qty_smp); ++b) {
      int r = launch_sample(c->dm, c->dw, c->opt.precision, c->stream);
      if (r != kOk) return r;
      c->sampled = true;
      std::vector<double> g;
      r = do_measure_green(c, g);
      if (r != kOk) return r;
      const double* t = c->tot.data();
      mvmc::write_physcal_block(m, out_dir, m.data_idx_start + b, mvmc::StepEnergy{t[1], t[2], t[3], t[4]}, g.data(),
                                g.data() + c->n_one, g.data() + c->n_one + c->n_ex);
    }
    return MVMC_B200_OK;
  });
  mvmc_b200_destroy(c);
  return rc;
}

// ---------------------------------------------------------------------------------------
// One walker's Pfaffian stage (RealPfStage, crates/mvmc-core/src/sampling/stage.rs:56-129).
// ---------------------------------------------------------------------------------------
struct mvmc_b200_stage {
  mvmc_b200_ctx* ctx = nullptr;
  StageBufs b{};
  int* d_idx = nullptr;
  std::vector<void*> allocs;
  ~mvmc_b200_stage() {
    for (void* p : allocs) cudaFree(p);
  }
  template <typename T>
  T* alloc(size_t count) {
    void* p = nullptr;
    check(cudaMalloc(&p, std::max<size_t>(1, count) * sizeof(T)), "stage cudaMalloc");
    allocs.push_back(p);
    return static_cast<T*>(p);
  }
};

namespace {

// Candidate configuration of the call: validated on the host, copied to the device.
void stage_upload_idx(mvmc_b200_stage* st, const int64_t* ele_idx) {
  const mvmc_b200_ctx* c = st->ctx;
  const int n = c->dm.n;
  std::vector<int> idx(n);
  for (int k = 0; k < n; ++k) {
    if (ele_idx[k] < 0 || ele_idx[k] >= c->dm.ns) throw std::invalid_argument("stage: ele_idx entry out of range");
    idx[k] = static_cast<int>(ele_idx[k]);
  }
  check(cudaMemcpyAsync(st->d_idx, idx.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c->stream), "stage idx");
}

int stage_run(mvmc_b200_stage* st, int op, int msa, int msb, int rsa_old, int rsb_old) {
  mvmc_b200_ctx* c = st->ctx;
  const int rc = launch_stage(c->dm, st->b, op, msa, msb, rsa_old, rsb_old, c->dw.status, c->stream);
  if (rc != kOk) return rc;
  return kOk;
}

void stage_download(mvmc_b200_stage* st, const double* dev, double* host) {
  mvmc_b200_ctx* c = st->ctx;
  if (host)
    check(cudaMemcpyAsync(host, dev, sizeof(double) * c->dm.nqp, cudaMemcpyDeviceToHost, c->stream), "stage pf");
  check(cudaStreamSynchronize(c->stream), "stage");
}

int stage_guard(mvmc_b200_stage* st, const int64_t* ele_idx, int ma, int sa, int mb, int sb, bool two) {
  if (!st || !ele_idx) return MVMC_B200_EARG;
  const int ne = st->ctx->dm.ne;
  if (ma < 0 || ma >= ne || sa < 0 || sa > 1) return MVMC_B200_EARG;
  if (two && (mb < 0 || mb >= ne || sb < 0 || sb > 1 || (ma + sa * ne) == (mb + sb * ne))) return MVMC_B200_EARG;
  return MVMC_B200_OK;
}

}  // namespace

extern "C" int mvmc_b200_stage_create(mvmc_b200_ctx* c, mvmc_b200_stage** out) {
  if (!c || !out) return MVMC_B200_EARG;
  *out = nullptr;
  auto* st = new mvmc_b200_stage();
  st->ctx = c;
  const int rc = guarded([&]() {
    const size_t nn = static_cast<size_t>(c->dm.n) * c->dm.n;
    st->b.planes = st->alloc<double>(nn * c->dm.nqp);
    st->b.ws = st->alloc<double>(2 * nn);
    st->b.pf = st->alloc<double>(c->dm.nqp);
    st->b.pfn = st->alloc<double>(c->dm.nqp);
    st->d_idx = st->alloc<int>(c->dm.n);
    st->b.idx = st->d_idx;
    st->b.info = st->alloc<int>(1);
    check(cudaMemsetAsync(st->b.pf, 0, sizeof(double) * c->dm.nqp, c->stream), "stage memset");
    check(cudaMemsetAsync(st->b.pfn, 0, sizeof(double) * c->dm.nqp, c->stream), "stage memset");
    check(cudaStreamSynchronize(c->stream), "stage create");
    return MVMC_B200_OK;
  });
  if (rc != MVMC_B200_OK) {
    delete st;
    return rc;
  }
  *out = st;
  return MVMC_B200_OK;
}

extern "C" void mvmc_b200_stage_destroy(mvmc_b200_stage* st) { delete st; }

extern "C" int mvmc_b200_stage_recompute(mvmc_b200_stage* st, const int64_t* ele_idx, double* pf) {
  if (!st || !ele_idx) return MVMC_B200_EARG;
  return guarded([&]() {
    stage_upload_idx(st, ele_idx);
    const int rc = stage_run(st, kStageRecompute, 0, 0, 0, 0);
    if (rc != kOk) return rc;
    int info = 0;
    check(cudaMemcpyAsync(&info, st->b.info, sizeof(int), cudaMemcpyDeviceToHost, st->ctx->stream), "stage info");
    stage_download(st, st->b.pf, pf);
    return info != 0 ? 1 : MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_stage_begin(mvmc_b200_stage* st, const int64_t* ele_idx, double* pf) {
  return mvmc_b200_stage_recompute(st, ele_idx, pf);
}

extern "C" int mvmc_b200_stage_propose_hop(mvmc_b200_stage* st, const int64_t* ele_idx, int ma, int spin,
                                           double* pf_new) {
  const int g = stage_guard(st, ele_idx, ma, spin, 0, 0, false);
  if (g != MVMC_B200_OK) return g;
  return guarded([&]() {
    stage_upload_idx(st, ele_idx);
    const int rc = stage_run(st, kStageProposeHop, ma + spin * st->ctx->dm.ne, 0, 0, 0);
    if (rc != kOk) return rc;
    stage_download(st, st->b.pfn, pf_new);
    return MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_stage_accept_hop(mvmc_b200_stage* st, const int64_t* ele_idx, int ma, int spin,
                                          const double* pf_new) {
  const int g = stage_guard(st, ele_idx, ma, spin, 0, 0, false);
  if (g != MVMC_B200_OK) return g;
  return guarded([&]() {
    stage_upload_idx(st, ele_idx);
    const int rc = stage_run(st, kStageAcceptHop, ma + spin * st->ctx->dm.ne, 0, 0, 0);
    if (rc != kOk) return rc;
    // afterwards the current Pfaffians equal the proposal's (stage.rs:83-92)
    if (pf_new)
      check(cudaMemcpyAsync(st->b.pf, pf_new, sizeof(double) * st->ctx->dm.nqp, cudaMemcpyHostToDevice,
                            st->ctx->stream), "stage pf_new");
    stage_download(st, st->b.pf, nullptr);
    return MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_stage_propose_exchange(mvmc_b200_stage* st, const int64_t* ele_idx, int ma, int sa,
                                                int mb, int sb, double* pf_new) {
  const int g = stage_guard(st, ele_idx, ma, sa, mb, sb, true);
  if (g != MVMC_B200_OK) return g;
  return guarded([&]() {
    stage_upload_idx(st, ele_idx);
    const int ne = st->ctx->dm.ne;
    const int rc = stage_run(st, kStageProposeExchange, ma + sa * ne, mb + sb * ne, 0, 0);
    if (rc != kOk) return rc;
    stage_download(st, st->b.pfn, pf_new);
    return MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_stage_accept_exchange(mvmc_b200_stage* st, const int64_t* ele_idx, int ma, int sa,
                                               int mb, int sb, int ra_old, int rb_old) {
  const int g = stage_guard(st, ele_idx, ma, sa, mb, sb, true);
  if (g != MVMC_B200_OK) return g;
  const int ns = st->ctx->dm.ns;
  if (ra_old < 0 || ra_old >= ns || rb_old < 0 || rb_old >= ns) return MVMC_B200_EARG;
  return guarded([&]() {
    stage_upload_idx(st, ele_idx);
    const int ne = st->ctx->dm.ne;
    const int rc = stage_run(st, kStageAcceptExchange, ma + sa * ne, mb + sb * ne, ra_old + sa * ns, rb_old + sb * ns);
    if (rc != kOk) return rc;
    stage_download(st, st->b.pf, nullptr);
    return MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_stage_state(const mvmc_b200_stage* st, double* pf, double* inv_m) {
  if (!st) return MVMC_B200_EARG;
  return guarded([&]() {
    const mvmc_b200_ctx* c = st->ctx;
    const size_t nn = static_cast<size_t>(c->dm.n) * c->dm.n;
    if (pf) check(cudaMemcpy(pf, st->b.pf, sizeof(double) * c->dm.nqp, cudaMemcpyDeviceToHost), "stage pf");
    if (inv_m)
      check(cudaMemcpy(inv_m, st->b.planes, sizeof(double) * nn * c->dm.nqp, cudaMemcpyDeviceToHost), "stage inv");
    return MVMC_B200_OK;
  });
}

// ---------------------------------------------------------------------------------------
// Walker-sharded SR (the reference's Reducer seam, crates/mvmc-core/src/reducer.rs:20-168):
// each rank measures its own walkers; the caller adds the sums and the CG products across
// ranks and runs the recurrence; every rank applies the same update.
// ---------------------------------------------------------------------------------------
extern "C" int mvmc_b200_measure_sums(const mvmc_b200_ctx* c, double* sums) {
  if (!c || !sums) return MVMC_B200_EARG;
  if (!c->measured) return MVMC_B200_ESTATE;
  const double wc = c->tot[0];
  sums[0] = wc;
  for (size_t k = 1; k < c->tot.size(); ++k) sums[k] = c->tot[k] * wc;
  return MVMC_B200_OK;
}

extern "C" int mvmc_b200_sr_gather(mvmc_b200_ctx* c, const int* map, int na) {
  if (!c || !map || na <= 0) return MVMC_B200_EARG;
  if (!c->measured) return MVMC_B200_ESTATE;
  const int npara = c->m.npara();
  for (int i = 0; i < na; ++i)
    if (map[i] < 0 || map[i] >= npara) return MVMC_B200_EARG;
  return guarded([&]() {
    const long long ns = static_cast<long long>(c->W) * c->S;
    if (static_cast<size_t>(ns) * na > c->oa_cap) {
      c->d_oa = c->alloc<double>(static_cast<size_t>(ns) * na);
      c->oa_cap = static_cast<size_t>(ns) * na;
    }
    if (static_cast<size_t>(ns) > c->y_cap) {
      c->d_y = c->alloc<double>(ns);
      c->y_cap = static_cast<size_t>(ns);
    }
    if (static_cast<size_t>(na) > c->map_cap) {
      c->d_map = c->alloc<int>(na);
      c->map_cap = na;
    }
    if (static_cast<size_t>(2) * na > c->shard_vec_cap) {
      c->d_shard_vec = c->alloc<double>(static_cast<size_t>(2) * na);
      c->shard_vec_cap = static_cast<size_t>(2) * na;
    }
    const size_t part = static_cast<size_t>(local_product_chunks(ns, na)) * na;
    if (part > c->shard_part_cap) {
      c->d_shard_part = c->alloc<double>(part);
      c->shard_part_cap = part;
    }
    check(cudaMemcpyAsync(c->d_map, map, sizeof(int) * na, cudaMemcpyHostToDevice, c->stream), "upload map");
    c->h2d += static_cast<long long>(sizeof(int) * na);
    const int rc = launch_gather_active(c->d_ostore, c->dm.sr_size, ns, c->d_map, na, c->d_oa, c->stream);
    if (rc != kOk) return rc;
    check(cudaStreamSynchronize(c->stream), "gather");
    c->shard_na = na;
    return MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_sr_local_product(mvmc_b200_ctx* c, const double* v, double* z) {
  if (!c || !v || !z) return MVMC_B200_EARG;
  if (c->shard_na <= 0) return MVMC_B200_ESTATE;
  return guarded([&]() {
    const int na = c->shard_na;
    const long long ns = static_cast<long long>(c->W) * c->S;
    double* dv = c->d_shard_vec;
    double* dz = dv + na;
    check(cudaMemcpyAsync(dv, v, sizeof(double) * na, cudaMemcpyHostToDevice, c->stream), "upload v");
    const int rc = launch_local_product(c->d_oa, ns, na, dv, dz, c->d_y, c->d_shard_part, c->stream);
    if (rc != kOk) return rc;
    check(cudaMemcpyAsync(z, dz, sizeof(double) * na, cudaMemcpyDeviceToHost, c->stream), "download z");
    check(cudaStreamSynchronize(c->stream), "local product");
    c->h2d += static_cast<long long>(sizeof(double) * na);
    c->d2h += static_cast<long long>(sizeof(double) * na);
    return MVMC_B200_OK;
  });
}

// Device-buffer form: v, z are device pointers ordered on the caller's `stream`; the
// product runs on the engine's stream between two event joins, so no host copy is made.
extern "C" int mvmc_b200_sr_local_product_device(mvmc_b200_ctx* c, const double* v, double* z, void* stream) {
  if (!c || !v || !z) return MVMC_B200_EARG;
  if (c->shard_na <= 0) return MVMC_B200_ESTATE;
  return guarded([&]() {
    const long long ns = static_cast<long long>(c->W) * c->S;
    cudaStream_t caller = static_cast<cudaStream_t>(stream);
    if (!c->join_event) check(cudaEventCreateWithFlags(&c->join_event, cudaEventDisableTiming), "event");
    check(cudaEventRecord(c->join_event, caller), "record");
    check(cudaStreamWaitEvent(c->stream, c->join_event, 0), "join engine stream");
    const int rc = launch_local_product(c->d_oa, ns, c->shard_na, v, z, c->d_y, c->d_shard_part, c->stream);
    if (rc != kOk) return rc;
    check(cudaEventRecord(c->join_event, c->stream), "record");
    check(cudaStreamWaitEvent(caller, c->join_event, 0), "join caller stream");
    return MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_sr_apply(mvmc_b200_ctx* c, const int* map, int na, const double* x) {
  if (!c || (na > 0 && (!map || !x)) || na < 0) return MVMC_B200_EARG;
  const int npara = c->m.npara();
  for (int i = 0; i < na; ++i)
    if (map[i] < 0 || map[i] >= npara) return MVMC_B200_EARG;
  return guarded([&]() {
    std::vector<double> p = mvmc::all_parameters(c->m);
    for (int si = 0; si < na; ++si) p[map[si]] += x[si];
    mvmc::set_all_parameters(c->m, p);
    mvmc::sync_modified_parameter(c->m, true);
    upload_parameters(c);
    check(cudaStreamSynchronize(c->stream), "apply");
    return MVMC_B200_OK;
  });
}

extern "C" int mvmc_b200_sr_config(const mvmc_b200_ctx* c, double* cfg, int* flags) {
  if (!c || !cfg) return MVMC_B200_EARG;
  const mvmc::Model& m = c->m;
  const double v[10] = {static_cast<double>(m.nsrcg), m.red_cut, m.step_dt, m.sta_del, m.cg_tol,
                        static_cast<double>(m.cg_max_iter), m.diag_scale ? 1.0 : 0.0, m.cg_fallback ? 1.0 : 0.0,
                        m.cg_abort ? 1.0 : 0.0, static_cast<double>(m.npara())};
  std::copy(v, v + 10, cfg);
  if (flags) {
    const int width = 2 * m.npara();
    for (int k = 0; k < width; ++k) flags[k] = static_cast<size_t>(k) < m.opt_flags.size() ? m.opt_flags[k] : 0;
  }
  return MVMC_B200_OK;
}
