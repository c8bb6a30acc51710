// Expert-mode reader, parameter initialisation and output writers.
// File formats follow crates/mvmc-expert-parsers/src/parsers/*.rs of AtelierArith/mvmc-rs
// (five header lines per definition file, the count on line 2, flags after the
// index block); arithmetic follows the files cited in expert.h.
#include "expert.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>

namespace mvmc {
namespace {

std::string dir_of(const std::string& path) {
  auto pos = path.find_last_of('/');
  return pos == std::string::npos ? std::string(".") : path.substr(0, pos);
}

std::vector<std::string> read_lines(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::vector<std::string> lines;
  std::string line;
  while (std::getline(f, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    lines.push_back(line);
  }
  return lines;
}

std::vector<std::string> tokens(const std::string& s) {
  std::istringstream is(s);
  std::vector<std::string> out;
  std::string t;
  while (is >> t) out.push_back(t);
  return out;
}

// Count on line 2 of a definition file ("NXxx  count").
int header_count(const std::vector<std::string>& lines, const std::string& path) {
  if (lines.size() < 5) throw std::runtime_error(path + ": fewer than five header lines");
  auto t = tokens(lines[1]);
  if (t.size() < 2) throw std::runtime_error(path + ": missing count on line 2");
  return std::stoi(t[1]);
}

int header_complex(const std::vector<std::string>& lines) {
  auto t = tokens(lines[2]);
  if (t.size() >= 2 && t[0] == "ComplexType") return std::stoi(t[1]);
  return 0;
}

// All whitespace-separated tokens of the body (lines 6..).
std::vector<std::string> body_tokens(const std::vector<std::string>& lines) {
  std::vector<std::string> out;
  for (size_t k = 5; k < lines.size(); ++k) {
    auto t = tokens(lines[k]);
    out.insert(out.end(), t.begin(), t.end());
  }
  return out;
}

// Flags "idx flag" pairs; row order assigns the flag (the printed index is ignored).
std::vector<int> read_flags(const std::vector<std::string>& tok, size_t start, int count,
                            const std::string& path) {
  if (tok.size() < start + 2 * static_cast<size_t>(count))
    throw std::runtime_error(path + ": incomplete optimisation-flag section");
  std::vector<int> f(count);
  for (int k = 0; k < count; ++k) f[k] = std::stoi(tok[start + 2 * k + 1]);
  return f;
}

bool key_is(const std::string& a, const char* b) {
  if (a.size() != std::char_traits<char>::length(b)) return false;
  for (size_t i = 0; i < a.size(); ++i)
    if (std::tolower(a[i]) != std::tolower(b[i])) return false;
  return true;
}

void parse_modpara(Model& m, const std::string& path) {
  auto lines = read_lines(path);
  int ncond = -1;
  for (const auto& line : lines) {
    auto t = tokens(line);
    if (t.size() < 2) continue;
    const std::string& k = t[0];
    const std::string& v = t[1];
    if (key_is(k, "NVMCCalMode")) m.calc_mode = std::stoi(v);
    else if (key_is(k, "Nsite")) m.nsite = std::stoi(v);
    else if (key_is(k, "Ncond")) ncond = std::stoi(v);
    else if (key_is(k, "2Sz")) m.two_sz = std::stoi(v);
    else if (key_is(k, "NSPGaussLeg")) m.nsp_gauss_leg = std::stoi(v);
    else if (key_is(k, "NSPStot")) m.nsp_stot = std::stoi(v);
    else if (key_is(k, "NMPTrans")) m.nmp_trans = std::stoi(v);
    else if (key_is(k, "NSROptItrStep")) m.nsr_opt_itr_step = std::stoi(v);
    else if (key_is(k, "NSROptItrSmp")) m.nsr_opt_itr_smp = std::stoi(v);
    else if (key_is(k, "DSROptRedCut")) m.red_cut = std::stod(v);
    else if (key_is(k, "DSROptStaDel")) m.sta_del = std::stod(v);
    else if (key_is(k, "DSROptStepDt")) m.step_dt = std::stod(v);
    else if (key_is(k, "NVMCWarmUp")) m.nvmc_warmup = std::stoi(v);
    else if (key_is(k, "NVMCInterval")) m.nvmc_interval = std::stoi(v);
    else if (key_is(k, "NVMCSample")) m.nvmc_sample = std::stoi(v);
    else if (key_is(k, "NExUpdatePath")) m.nex_update_path = std::stoi(v);
    else if (key_is(k, "RndSeed")) m.rnd_seed = std::stoll(v);
    else if (key_is(k, "NSplitSize")) m.nsplit_size = std::stoi(v);
    else if (key_is(k, "NStore")) m.nstore = std::stoi(v);
    else if (key_is(k, "NSRCG")) m.nsrcg = std::stoi(v);
    else if (key_is(k, "NSROptCGMaxIter")) m.cg_max_iter = std::stoi(v);
    else if (key_is(k, "DSROptCGTol")) m.cg_tol = std::stod(v);
    else if (key_is(k, "NSRCGFallback")) m.cg_fallback = std::stoi(v) != 0;
    else if (key_is(k, "NSRCGAbortOnFail")) m.cg_abort = std::stoi(v) != 0;
    else if (key_is(k, "RescaleSmat")) m.rescale_smat = std::stoi(v) != 0;
    else if (key_is(k, "NDataIdxStart")) m.data_idx_start = std::stoi(v);
    else if (key_is(k, "NDataQtySmp")) m.data_qty_smp = std::stoi(v);
    else if (key_is(k, "CDataFileHead")) m.data_head = v;
    else if (key_is(k, "CParaFileHead")) m.para_head = v;
    else if (key_is(k, "ComplexType") || key_is(k, "NLanczosMode") || key_is(k, "NSROptFixSmp") ||
             key_is(k, "NLocalSpin") || key_is(k, "Model_Parameters") ||
             key_is(k, "NSplitSize"))
      continue;
  }
  // readdef.c: NSRCG 2 selects DiagScale CG and becomes NSRCG 1.
  if (m.nsrcg == 2) {
    m.nsrcg = 1;
    m.diag_scale = true;
  }
  if (ncond < 0) throw std::runtime_error(path + ": Ncond is required");
  m.ne = ncond / 2;
}

}  // namespace

Model read_expert(const std::string& namelist_path) {
  Model m;
  const std::string dir = dir_of(namelist_path);
  std::map<std::string, std::string> files;
  for (const auto& line : read_lines(namelist_path)) {
    auto t = tokens(line);
    if (t.size() >= 2) files[t[0]] = dir + "/" + t[1];
  }
  auto need = [&](const char* key) -> std::string {
    auto it = files.find(key);
    if (it == files.end()) throw std::runtime_error(std::string("namelist lacks ") + key);
    return it->second;
  };
  for (const char* unsupported : {"PairHop", "Exchange", "InterAll", "DH2", "DH4",
                                  "OrbitalGeneral", "OrbitalParallel", "OrbitalAntiParallel",
                                  "GeneralRBM_PhysLayer", "ChargeRBM_PhysLayer", "SpinRBM_PhysLayer",
                                  "TransOpt"}) {
    if (files.count(unsupported))
      throw std::runtime_error(std::string("namelist names ") + unsupported +
                               ", which the real sz-conserved hot path does not cover");
  }
  parse_modpara(m, need("ModPara"));
  const int ns = m.nsite;

  // LocSpin
  m.loc_spn.assign(ns, 0);
  if (files.count("LocSpin")) {
    auto lines = read_lines(files["LocSpin"]);
    auto tok = body_tokens(lines);
    for (int k = 0; k + 1 < static_cast<int>(tok.size()) && k / 2 < ns; k += 2) {
      int site = std::stoi(tok[k]);
      if (site >= 0 && site < ns) m.loc_spn[site] = std::stoi(tok[k + 1]);
    }
    for (int v : m.loc_spn)
      if (v == 1) throw std::runtime_error("local spins are outside the Hubbard hot path");
  }

  // Trans
  if (files.count("Trans")) {
    auto lines = read_lines(files["Trans"]);
    int n = header_count(lines, files["Trans"]);
    for (int k = 0; k < n; ++k) {
      auto t = tokens(lines.at(5 + k));
      if (t.size() < 5) throw std::runtime_error("trans.def: short line");
      TransferTerm term{std::stoi(t[0]), std::stoi(t[1]), std::stoi(t[2]), std::stoi(t[3]),
                        std::stod(t[4])};
      double im = t.size() >= 6 ? std::stod(t[5]) : 0.0;
      if (im != 0.0) throw std::runtime_error("complex transfer amplitudes are not supported");
      m.transfer.push_back(term);
    }
  }
  // CoulombIntra / CoulombInter / Hund
  auto read_site_terms = [&](const char* key) {
    std::vector<SiteTerm> out;
    if (!files.count(key)) return out;
    auto lines = read_lines(files[key]);
    int n = header_count(lines, files[key]);
    for (int k = 0; k < n; ++k) {
      auto t = tokens(lines.at(5 + k));
      out.push_back({std::stoi(t[0]), std::stod(t[1])});
    }
    return out;
  };
  auto read_pair_terms = [&](const char* key) {
    std::vector<PairTerm> out;
    if (!files.count(key)) return out;
    auto lines = read_lines(files[key]);
    int n = header_count(lines, files[key]);
    for (int k = 0; k < n; ++k) {
      auto t = tokens(lines.at(5 + k));
      out.push_back({std::stoi(t[0]), std::stoi(t[1]), std::stod(t[2])});
    }
    return out;
  };
  m.coulomb_intra = read_site_terms("CoulombIntra");
  m.coulomb_inter = read_pair_terms("CoulombInter");
  m.hund = read_pair_terms("Hund");

  std::vector<int> flags_g, flags_j, flags_o;
  // Gutzwiller
  m.gutz_idx.assign(ns, -1);
  if (files.count("Gutzwiller")) {
    auto lines = read_lines(files["Gutzwiller"]);
    m.n_gutz = header_count(lines, files["Gutzwiller"]);
    if (header_complex(lines) != 0) throw std::runtime_error("complex Gutzwiller not supported");
    auto tok = body_tokens(lines);
    for (int k = 0; k < ns; ++k) m.gutz_idx[std::stoi(tok.at(2 * k))] = std::stoi(tok.at(2 * k + 1));
    flags_g = read_flags(tok, 2 * ns, m.n_gutz, files["Gutzwiller"]);
  }
  // Jastrow
  m.jast_idx.assign(ns * ns, -1);
  if (files.count("Jastrow")) {
    auto lines = read_lines(files["Jastrow"]);
    m.n_jast = header_count(lines, files["Jastrow"]);
    if (header_complex(lines) != 0) throw std::runtime_error("complex Jastrow not supported");
    auto tok = body_tokens(lines);
    const int nmap = ns * (ns - 1);
    for (int k = 0; k < nmap; ++k) {
      int i = std::stoi(tok.at(3 * k)), j = std::stoi(tok.at(3 * k + 1));
      m.jast_idx[i * ns + j] = std::stoi(tok.at(3 * k + 2));
    }
    flags_j = read_flags(tok, 3 * nmap, m.n_jast, files["Jastrow"]);
  }
  // Orbital (anti-parallel, ns*ns lines "i j idx [sgn]"; the sign carries over)
  m.orb_idx.assign(ns * ns, -1);
  m.orb_sgn.assign(ns * ns, 1);
  {
    const std::string path = need("Orbital");
    auto lines = read_lines(path);
    m.n_orb = header_count(lines, path);
    if (header_complex(lines) != 0) throw std::runtime_error("complex orbitals not supported");
    const int nmap = ns * ns;
    int sign = 1;
    for (int k = 0; k < nmap; ++k) {
      auto t = tokens(lines.at(5 + k));
      int i = std::stoi(t.at(0)), j = std::stoi(t.at(1)), idx = std::stoi(t.at(2));
      if (t.size() >= 4) sign = std::stoi(t[3]);
      m.orb_idx[i * ns + j] = idx;
      m.orb_sgn[i * ns + j] = sign;
    }
    std::vector<std::string> tok;
    for (size_t k = 5 + nmap; k < lines.size(); ++k) {
      auto t = tokens(lines[k]);
      tok.insert(tok.end(), t.begin(), t.end());
    }
    flags_o = read_flags(tok, 0, m.n_orb, path);
  }
  // TransSym (qptransidx.def)
  {
    const std::string path = need("TransSym");
    auto lines = read_lines(path);
    m.n_qp_trans = header_count(lines, path);
    m.qp_trans_weight.assign(m.n_qp_trans, 0.0);
    m.qp_trans.assign(m.n_qp_trans * ns, -1);
    m.qp_trans_sgn.assign(m.n_qp_trans * ns, 1);
    size_t k = 5;
    for (int q = 0; q < m.n_qp_trans; ++q, ++k) {
      auto t = tokens(lines.at(k));
      m.qp_trans_weight.at(std::stoi(t.at(0))) = std::stod(t.at(1));
    }
    for (; k < lines.size(); ++k) {
      auto t = tokens(lines[k]);
      if (t.size() < 3) continue;
      int q = std::stoi(t[0]), i = std::stoi(t[1]), j = std::stoi(t[2]);
      int s = t.size() >= 4 ? std::stoi(t[3]) : 1;
      m.qp_trans[q * ns + i] = j;
      m.qp_trans_sgn[q * ns + i] = s;
    }
  }
  if (m.mp_trans() == 0) m.nmp_trans = 1;  // C treats NMPTrans 0 as a single identity sector
  if (m.mp_trans() > m.n_qp_trans) throw std::runtime_error("NMPTrans exceeds NQPTrans");

  m.opt_flags.clear();
  auto push_flags = [&](const std::vector<int>& f) {
    for (int v : f) {
      m.opt_flags.push_back(v);
      m.opt_flags.push_back(0);  // imaginary slot: real mode never optimises it
    }
  };
  push_flags(flags_g);
  push_flags(flags_j);
  push_flags(flags_o);
  m.gutz.assign(m.n_gutz, 0.0);
  m.jast.assign(m.n_jast, 0.0);
  m.slater.assign(m.n_orb, 0.0);

  // PhysCal Green-function lists (green.rs:16-270): the count on line 2, five header
  // lines, one term per non-empty body line; sites in [0, Nsite), spins 0 or 1, and the
  // number of rows equal to the count.
  auto green_rows = [&](const char* key, size_t fields, bool exact) {
    std::vector<std::vector<int>> rows;
    if (!files.count(key)) return rows;
    const std::string path = files[key];
    auto lines = read_lines(path);
    if (lines.size() < 2) throw std::runtime_error(path + ": missing count on line 2");
    auto head = tokens(lines[1]);
    if (head.size() < 2) throw std::runtime_error(path + ": missing count on line 2");
    const int count = std::stoi(head[1]);
    if (count == 0) return rows;
    if (lines.size() < 5) throw std::runtime_error(path + ": fewer than five header lines");
    for (size_t k = 5; k < lines.size(); ++k) {
      auto t = tokens(lines[k]);
      if (t.empty()) continue;
      if (t.size() < fields || (exact && t.size() != fields))
        throw std::runtime_error(path + ": expected " + std::to_string(fields) + " integer fields");
      std::vector<int> row(fields);
      for (size_t f = 0; f < fields; ++f) {
        size_t used = 0;
        row[f] = std::stoi(t[f], &used);
        if (used != t[f].size()) throw std::runtime_error(path + ": malformed integer " + t[f]);
        const bool spin = f % 2 == 1;
        if (spin ? (row[f] != 0 && row[f] != 1) : (row[f] < 0 || row[f] >= ns))
          throw std::runtime_error(path + ": site or spin out of range");
      }
      rows.push_back(row);
    }
    if (static_cast<int>(rows.size()) != count)
      throw std::runtime_error(path + ": declared row count does not match the rows");
    return rows;
  };
  for (const auto& r : green_rows("OneBodyG", 4, false)) m.green_one.push_back({r[0], r[1], r[2], r[3]});
  for (const auto& r : green_rows("TwoBodyG", 8, false))
    m.green_two.push_back({r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7]});
  // TwoBodyGEx "i s j t k u l v" is the product <c†_is c_jt>·<c†_lv c_ku>*: its factors are
  // the one-body terms (i s j t) and (l v k u) (green.rs:252-261; types.rs:1169-1215).
  const auto ex_rows = green_rows("TwoBodyGEx", 8, true);
  if (!ex_rows.empty()) {
    std::vector<GreenOneTerm> canonical;
    for (const auto& t : m.green_one)
      if (std::find(canonical.begin(), canonical.end(), t) == canonical.end()) canonical.push_back(t);
    m.green_one = canonical;
  }
  auto one_index = [&](const GreenOneTerm& t) {
    auto it = std::find(m.green_one.begin(), m.green_one.end(), t);
    if (it != m.green_one.end()) return static_cast<int>(it - m.green_one.begin());
    m.green_one.push_back(t);
    return static_cast<int>(m.green_one.size()) - 1;
  };
  for (const auto& r : ex_rows) {
    const int first = one_index({r[0], r[1], r[2], r[3]});
    const int second = one_index({r[6], r[7], r[4], r[5]});
    m.green_two_ex.emplace_back(first, second);
  }
  return m;
}

// ---- QP weights (qp_weight.rs:24-170) --------------------------------------------
namespace {
void gauss_legendre(double x1, double x2, int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  const int mm = (n + 1) / 2;
  const double xm = 0.5 * (x2 + x1), xl = 0.5 * (x2 - x1);
  for (int i = 0; i < mm; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5));
    double pp;
    while (true) {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= n; ++j) {
        double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      double z1 = z;
      z = z1 - p1 / pp;
      if (std::fabs(z - z1) <= 5.0e-14) break;
    }
    x[i] = xm - xl * z;
    x[n - 1 - i] = xm + xl * z;
    w[i] = 2.0 * xl / ((1.0 - z * z) * pp * pp);
    w[n - 1 - i] = w[i];
  }
}
double legendre_poly(double x, int n) {
  if (n <= 0) return 1.0;
  if (n == 1) return x;
  double p01 = 1.0, p02 = x, p03 = x;
  for (int i = 2; i <= n; ++i) {
    double fi = i;
    p03 = (1.0 / fi) * ((2.0 * fi - 1.0) * x * p02 - (fi - 1.0) * p01);
    p01 = p02;
    p02 = p03;
  }
  return p03;
}
}  // namespace

void init_qp_weight(Model& m) {
  const int nleg = std::max(1, m.nsp_gauss_leg);
  const int nmp = m.mp_trans();
  m.nqp = nleg * nmp;
  std::vector<double> fix(m.nqp, 0.0);
  m.spgl_cs.assign(nleg, 0.0);
  m.spgl_cc.assign(nleg, 0.0);
  m.spgl_ss.assign(nleg, 0.0);
  if (nleg == 1) {
    m.spgl_cc[0] = 1.0;
    for (int j = 0; j < nmp; ++j) fix[j] = m.qp_trans_weight[j];
  } else {
    std::vector<double> beta, wgl;
    gauss_legendre(0.0, M_PI, nleg, beta, wgl);
    for (int i = 0; i < nleg; ++i) {
      double ch = std::cos(0.5 * beta[i]), sh = std::sin(0.5 * beta[i]);
      m.spgl_cs[i] = ch * sh;
      m.spgl_cc[i] = ch * ch;
      m.spgl_ss[i] = sh * sh;
      double w = 0.5 * std::sin(beta[i]) * wgl[i] * legendre_poly(std::cos(beta[i]), m.nsp_stot);
      for (int j = 0; j < nmp; ++j) fix[i + j * nleg] = m.qp_trans_weight[j] * w;
    }
  }
  m.qp_weight = fix;
}

void translated_site(const Model& m, int site, int mpidx, int* out_site, int* out_sign) {
  const int ns = m.nsite;
  int mapped = m.qp_trans[mpidx * ns + site];
  if (mapped < 0) mapped = site;
  *out_site = mapped;
  *out_sign = m.antiperiodic() ? m.qp_trans_sgn[mpidx * ns + site] : 1;
}

void build_slater_table(const Model& m, std::vector<double>& s) {
  const int ns = m.nsite, ns2 = 2 * ns, nleg = std::max(1, m.nsp_gauss_leg), nmp = m.mp_trans();
  const size_t plane = static_cast<size_t>(ns2) * ns2;
  s.assign(static_cast<size_t>(m.nqp) * plane, 0.0);
  for (int qp = 0; qp < m.nqp; ++qp) {
    const int mpidx = (qp % (nleg * nmp)) / nleg;
    const int spidx = qp % nleg;
    const double cs = m.spgl_cs[spidx], cc = m.spgl_cc[spidx], ss = m.spgl_ss[spidx];
    double* p = s.data() + qp * plane;
    for (int ri = 0; ri < ns; ++ri) {
      int tri, sgni;
      translated_site(m, ri, mpidx, &tri, &sgni);
      for (int rj = 0; rj < ns; ++rj) {
        int trj, sgnj;
        translated_site(m, rj, mpidx, &trj, &sgnj);
        const int qpsgn = sgni * sgnj;
        const int idx_ij = m.orb_idx[tri * ns + trj], idx_ji = m.orb_idx[trj * ns + tri];
        if (idx_ij < 0 || idx_ji < 0) continue;
        const double slt_ij = m.slater[idx_ij] * static_cast<double>(m.orb_sgn[tri * ns + trj] * qpsgn);
        const double slt_ji = m.slater[idx_ji] * static_cast<double>(m.orb_sgn[trj * ns + tri] * qpsgn);
        p[ri * ns2 + rj] = -(slt_ij - slt_ji) * cs;
        p[ri * ns2 + rj + ns] = slt_ij * cc + slt_ji * ss;
        p[(ri + ns) * ns2 + rj] = -slt_ij * ss - slt_ji * cc;
        p[(ri + ns) * ns2 + rj + ns] = (slt_ij - slt_ji) * cs;
      }
    }
  }
}

// ---- parameters -------------------------------------------------------------------
void init_parameter(Model& m, const std::function<double()>& real2) {
  std::fill(m.gutz.begin(), m.gutz.end(), 0.0);
  std::fill(m.jast.begin(), m.jast.end(), 0.0);
  const int np = m.nproj();
  for (int i = 0; i < m.n_orb; ++i) {
    const size_t flag = 2 * static_cast<size_t>(i + np);
    const bool opt = flag < m.opt_flags.size() ? m.opt_flags[flag] > 0 : true;
    m.slater[i] = opt ? 2.0 * (real2() - 0.5) : 0.0;
  }
}

void sync_modified_parameter(Model& m, bool shift_correlations) {
  if (shift_correlations && m.n_gutz > 0 && m.n_jast > 0) {
    // Active only when every Gutzwiller and Jastrow parameter is optimised.
    bool all_active = true;
    if (!m.opt_flags.empty())
      for (int i = 0; i < m.n_gutz + m.n_jast; ++i)
        if (m.opt_flags[2 * i] != 1) all_active = false;
    if (all_active) {
      double shift = 0.0;
      for (double g : m.gutz) shift += g;
      for (double j : m.jast) shift += j;
      shift /= static_cast<double>(m.n_gutz + m.n_jast);
      for (double& g : m.gutz) g -= shift;
      for (double& j : m.jast) j -= shift;
    }
  }
  double xmax = 0.0;
  for (double v : m.slater) {
    const double a = std::fabs(v);
    if (a > xmax) xmax = a;
  }
  if (xmax > 0.0) {
    const double ratio = 4.0 / xmax;
    for (double& v : m.slater) v *= ratio;
  }
}

std::vector<double> all_parameters(const Model& m) {
  std::vector<double> p;
  p.insert(p.end(), m.gutz.begin(), m.gutz.end());
  p.insert(p.end(), m.jast.begin(), m.jast.end());
  p.insert(p.end(), m.slater.begin(), m.slater.end());
  return p;
}

void set_all_parameters(Model& m, const std::vector<double>& p) {
  size_t k = 0;
  for (double& g : m.gutz) g = p[k++];
  for (double& j : m.jast) j = p[k++];
  for (double& s : m.slater) s = p[k++];
}

bool read_para_triples(Model& m, const std::string& path, std::string* why) {
  std::ifstream f(path);
  if (!f) {
    if (why) *why = "not found";
    return false;
  }
  std::vector<double> values;
  std::string t;
  while (f >> t) {
    try {
      values.push_back(std::stod(t));
    } catch (...) {
      if (why) *why = "non-numeric token";
      return false;
    }
  }
  const size_t expected = 6 + 3 * static_cast<size_t>(m.npara());
  if (values.size() != expected) {
    if (why) *why = "parameter count does not match the model";
    return false;
  }
  const double* v = values.data() + (values.size() - expected);
  std::vector<double> p(m.npara());
  for (int i = 0; i < m.npara(); ++i) p[i] = v[6 + 3 * i] + 0.0 * v[7 + 3 * i];
  set_all_parameters(m, p);
  return true;
}

// ---- writers -----------------------------------------------------------------------
std::string c_double(double v) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "% .18e", v);
  return buf;
}

namespace {
std::string c_double_nospace(double v) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.18e", v);
  return buf;
}
FILE* open_step(const std::string& path, bool first) {
  FILE* f = std::fopen(path.c_str(), first ? "w" : "a");
  if (!f) throw std::runtime_error("cannot write " + path);
  return f;
}
std::string c_exp5(double x) {
  if (std::isnan(x)) return std::signbit(x) ? "-nan" : " nan";
  if (std::isinf(x)) return x < 0 ? "-inf" : " inf";
  char buf[64];
  std::snprintf(buf, sizeof buf, "% .5e", x);
  return buf;
}
}  // namespace

void write_out_row(const Model& m, const std::string& dir, int step, const StepEnergy& e) {
  const double variance =
      std::fabs(e.etot) > 1.0e-14 ? (e.etot2 - e.etot * e.etot) / (e.etot * e.etot) : 0.0;
  FILE* f = open_step(dir + "/" + m.data_head + "_out.dat", step == 0);
  std::fprintf(f, "%s %s  %s %s %s %s\n", c_double(e.etot).c_str(), c_double(0.0).c_str(),
               c_double(e.etot2).c_str(), c_double(variance).c_str(),
               c_double_nospace(e.sztot).c_str(), c_double_nospace(e.sztot2).c_str());
  std::fclose(f);
  FILE* v = open_step(dir + "/" + m.data_head + "_var.dat", step == 0);
  std::fprintf(v, "%s %s 0.0 %s %s 0.0 ", c_double(e.etot).c_str(), c_double(0.0).c_str(),
               c_double(e.etot2).c_str(), c_double(0.0).c_str());
  for (double p : all_parameters(m))
    std::fprintf(v, "%s %s 0.0 ", c_double(p).c_str(), c_double(0.0).c_str());
  std::fprintf(v, "\n");
  std::fclose(v);
}

void write_physcal_block(const Model& m, const std::string& dir, int index, const StepEnergy& e,
                         const double* one, const double* two_ex, const double* two) {
  char tag[32];
  std::snprintf(tag, sizeof tag, "_%03d.dat", index);
  auto open = [&](const char* kind) {
    const std::string path = dir + "/" + m.data_head + "_" + kind + tag;
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) throw std::runtime_error("cannot write " + path);
    return f;
  };
  // C complex quotient (etot2 − etot²)/etot² with zero imaginary parts: a plain division.
  const double variance = (e.etot2 - e.etot * e.etot) / (e.etot * e.etot);
  FILE* f = open("out");
  std::fprintf(f, "%s %s  %s %s %s %s\n", c_double(e.etot).c_str(), c_double(0.0).c_str(),
               c_double(e.etot2).c_str(), c_double(variance).c_str(), c_double_nospace(e.sztot).c_str(),
               c_double_nospace(e.sztot2).c_str());
  std::fclose(f);
  f = open("var");
  std::fprintf(f, "%s %s 0.0 %s %s 0.0 ", c_double(e.etot).c_str(), c_double(0.0).c_str(),
               c_double(e.etot2).c_str(), c_double(0.0).c_str());
  for (double p : all_parameters(m)) std::fprintf(f, "%s %s 0.0 ", c_double(p).c_str(), c_double(0.0).c_str());
  std::fprintf(f, "\n");
  std::fclose(f);
  if (!m.green_one.empty()) {
    f = open("cisajs");
    for (size_t k = 0; k < m.green_one.size(); ++k) {
      const auto& t = m.green_one[k];
      std::fprintf(f, "%d %d %d %d %s  %s \n", t.i, t.si, t.j, t.sj, c_double(one[k]).c_str(),
                   c_double(0.0).c_str());
    }
    std::fprintf(f, "\n");
    std::fclose(f);
  }
  if (!m.green_two_ex.empty()) {
    f = open("cisajscktaltex");
    for (size_t k = 0; k < m.green_two_ex.size(); ++k)
      std::fprintf(f, "%s  %s ", c_double(two_ex[k]).c_str(), c_double(0.0).c_str());
    std::fprintf(f, "\n");
    std::fclose(f);
  }
  if (!m.green_two.empty()) {
    f = open("cisajscktalt");
    for (size_t k = 0; k < m.green_two.size(); ++k) {
      const auto& t = m.green_two[k];
      std::fprintf(f, "%d %d %d %d %d %d %d %d %s %s\n", t.i, t.si, t.j, t.sj, t.k, t.sk, t.l, t.sl,
                   c_double(two[k]).c_str(), c_double(0.0).c_str());
    }
    std::fprintf(f, "\n");
    std::fclose(f);
  }
}

void write_srinfo_row(const std::string& dir, const Model& m, bool first, const SrInfoRow& r) {
  // output_files.rs:55-100: the " info" column exists in SR-CG mode only
  const bool cg = m.nsrcg != 0;
  FILE* f = open_step(dir + "/" + m.data_head + "_SRinfo.dat", first);
  if (first)
    std::fprintf(f, cg ? "#Npara Msize optCut diagCut sDiagMax  sDiagMin    absRmax       imax info\n"
                       : "#Npara Msize optCut diagCut sDiagMax  sDiagMin    absRmax       imax\n");
  std::fprintf(f, "%5d %5d %5d %5d %s %s %s %5d", r.npara, r.nsmat, r.opt_cut, r.diag_cut,
               c_exp5(r.sdiag_max).c_str(), c_exp5(r.sdiag_min).c_str(), c_exp5(r.rmax).c_str(), r.imax);
  if (cg) std::fprintf(f, " %d", r.info);
  std::fprintf(f, "\n");
  std::fclose(f);
}

void write_opt_files(const Model& m, const std::string& dir, const std::vector<OptPoint>& window) {
  if (window.empty()) return;
  const int width = m.npara();
  auto value = [&](const OptPoint& p, int index) {
    return index == 0 ? p.etot : index == 1 ? p.etot2 : p.params[index - 2];
  };
  FILE* f = std::fopen((dir + "/" + m.para_head + "_opt.dat").c_str(), "w");
  if (!f) throw std::runtime_error("cannot write zqp_opt.dat");
  std::vector<double> means(width + 2);
  if (window.size() == 1) {
    for (int i = 0; i < width + 2; ++i) {
      means[i] = value(window[0], i);
      std::fprintf(f, "%s %s ", c_double(means[i]).c_str(), c_double(0.0).c_str());
    }
  } else {
    for (int i = 0; i < width + 2; ++i) {
      double mean = 0.0;
      for (const auto& p : window) mean += value(p, i);
      mean /= static_cast<double>(window.size());
      double var = 0.0;
      for (const auto& p : window) {
        const double d = value(p, i) - mean;
        var += d * d;
      }
      means[i] = mean;
      std::fprintf(f, "%s %s %s ", c_double(mean).c_str(), c_double(0.0).c_str(),
                   c_double(std::sqrt(var / (static_cast<double>(window.size()) - 1.0))).c_str());
    }
  }
  std::fprintf(f, "\n");
  std::fclose(f);
  struct Block {
    const char* suffix;
    const char* label;
    int count;
  };
  const Block blocks[] = {{"gutzwiller", "NGutzwillerIdx", m.n_gutz},
                          {"jastrow", "NJastrowIdx", m.n_jast},
                          {"orbital", "NOrbitalIdx", m.n_orb}};
  int offset = 2;
  for (const auto& b : blocks) {
    if (b.count > 0) {
      FILE* g = std::fopen((dir + "/" + m.para_head + "_" + b.suffix + "_opt.dat").c_str(), "w");
      if (!g) throw std::runtime_error("cannot write parameter block");
      std::fprintf(g, "======================\n%s  %d\n======================\n"
                      "======================\n======================\n",
                   b.label, b.count);
      for (int i = 0; i < b.count; ++i)
        std::fprintf(g, "%d %s %s \n", i, c_double(means[offset + i]).c_str(),
                     c_double(0.0).c_str());
      std::fclose(g);
    }
    offset += b.count;
  }
}

}  // namespace mvmc
