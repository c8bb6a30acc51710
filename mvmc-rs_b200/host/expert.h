// Expert-mode model description for the real, sz-conserved VMC optimizer.
//
// This is the input/output boundary of the sampling + SR hot path: the subset of
// mVMC's Expert-mode definition files that the real normal-orbital optimizer reads
// (namelist.def, modpara.def, locspn.def, trans.def, coulombintra.def,
// coulombinter.def, hund.def, gutzwilleridx.def, jastrowidx.def, orbitalidx.def,
// qptransidx.def) plus the Green-function lists of the PhysCal mode (greenone.def,
// greentwo.def, greentwoex.def), the derived quantum-projection weights, the parameter
// files (initial.def / zqp_opt.dat triples) and the writers of zvo_out.dat, zvo_var.dat,
// zvo_SRinfo.dat, zqp_*opt.dat and the indexed PhysCal files (zvo_out_NNN.dat,
// zvo_var_NNN.dat, zvo_cisajs_NNN.dat, zvo_cisajscktalt_NNN.dat,
// zvo_cisajscktaltex_NNN.dat).
//
// Reference behaviour followed (paths inside AtelierArith/mvmc-rs):
//   crates/mvmc-expert-parsers/src/parsers/{modpara,trans,coulomb,gutzwiller,
//     jastrow,orbital,qptrans,locspin}.rs   file formats (5 header lines, flags)
//   crates/mvmc-expert-parsers/src/parsers/green.rs:83-270     Green-function lists
//   crates/mvmc-expert-parsers/src/types.rs:1169-1215          TwoBodyGEx canonical map
//   crates/mvmc-expert-parsers/src/utils/qp_weight.rs:24-170   QP weights
//   crates/mvmc-expert-parsers/src/utils/parameter_init.rs:63-260 init + sync
//   crates/mvmc-core/src/slater_update.rs:17-120               Slater table
//   crates/mvmc-core/src/qp.rs:33-70                          translated_site
//   crates/mvmc-core/src/io.rs:142-220,561-730                output files
//   crates/mvmc-core/src/output_files.rs:55-100               SRinfo rows
//   crates/mvmc-core/src/io.rs:259-403                        PhysCal output files
#pragma once

#include <cstdint>
#include <functional>
#include <string>
#include <utility>
#include <vector>

namespace mvmc {

// c†_{i,si} c_{j,sj} with amplitude t; the Hamiltonian term is -t c†c.
struct TransferTerm {
  int i, si, j, sj;
  double t;
};
struct SiteTerm {  // CoulombIntra: U n_i↑ n_i↓
  int i;
  double v;
};
struct PairTerm {  // CoulombInter: V n_i n_j ; Hund: -J (n_i↑n_j↑ + n_i↓n_j↓)
  int i, j;
  double v;
};

// Green-function terms of the PhysCal measurement: c†_{i si} c_{j sj} (OneBodyG) and
// c†_{i si} c_{j sj} c†_{k sk} c_{l sl} (TwoBodyG, the direct "DC" form).
struct GreenOneTerm {
  int i, si, j, sj;
  bool operator==(const GreenOneTerm& o) const { return i == o.i && si == o.si && j == o.j && sj == o.sj; }
};
struct GreenTwoTerm {
  int i, si, j, sj, k, sk, l, sl;
};

struct Model {
  // ---- modpara.def (C defaults of SetDefaultValuesModPara) ----
  int calc_mode = 0;
  int nsite = 16, ne = 8, two_sz = -1;
  int nsp_gauss_leg = 1, nsp_stot = 0, nmp_trans = 0;
  int nsr_opt_itr_step = 1000, nsr_opt_itr_smp = 100;
  double red_cut = 1e-3, sta_del = 0.02, step_dt = 0.02;
  int nvmc_warmup = 10, nvmc_interval = 1, nvmc_sample = 10, nex_update_path = 0;
  long long rnd_seed = 11272;
  int nsplit_size = 1, nstore = 1, nsrcg = 0, cg_max_iter = 0;
  double cg_tol = 1e-10;
  bool diag_scale = false, cg_fallback = false, cg_abort = true, rescale_smat = false;
  int data_idx_start = 0, data_qty_smp = 1;
  std::string data_head = "zvo", para_head = "zqp";

  // ---- lattice / Hamiltonian ----
  std::vector<int> loc_spn;  // [nsite], 1 = local spin
  std::vector<TransferTerm> transfer;
  std::vector<SiteTerm> coulomb_intra;
  std::vector<PairTerm> coulomb_inter, hund;

  // ---- PhysCal Green-function lists ----
  // One-body terms: OneBodyG, de-duplicated in order when TwoBodyGEx is present, then the
  // TwoBodyGEx factors that OneBodyG lacks, appended in TwoBodyGEx order (all are output).
  std::vector<GreenOneTerm> green_one;
  std::vector<GreenTwoTerm> green_two;            // TwoBodyG in file order
  std::vector<std::pair<int, int>> green_two_ex;  // TwoBodyGEx: indices of its two factors

  // ---- projection and orbital index tables ----
  int n_gutz = 0, n_jast = 0, n_orb = 0;
  std::vector<int> gutz_idx;  // [nsite]
  std::vector<int> jast_idx;  // [nsite*nsite], -1 where undefined
  std::vector<int> orb_idx;   // [nsite*nsite]
  std::vector<int> orb_sgn;   // [nsite*nsite]
  int n_qp_trans = 0;
  std::vector<double> qp_trans_weight;  // [n_qp_trans]
  std::vector<int> qp_trans;            // [n_qp_trans*nsite]
  std::vector<int> qp_trans_sgn;        // [n_qp_trans*nsite]
  std::vector<int> opt_flags;           // [2*npara]: (real, imag) flag per parameter

  // ---- variational parameters (real mode) ----
  std::vector<double> gutz, jast, slater;

  // ---- derived by init_qp_weight ----
  int nqp = 0;                              // NQPFull
  std::vector<double> qp_weight;            // [nqp]
  std::vector<double> spgl_cs, spgl_cc, spgl_ss;  // [nsp_gauss_leg]

  int nsize() const { return 2 * ne; }
  int nsite2() const { return 2 * nsite; }
  int nproj() const { return n_gutz + n_jast; }
  int npara() const { return n_gutz + n_jast + n_orb; }
  int sr_size() const { return 1 + npara(); }
  int mp_trans() const { return nmp_trans < 0 ? -nmp_trans : nmp_trans; }
  bool antiperiodic() const { return nmp_trans < 0; }
};

// Parse namelist.def and the files it names. Throws std::runtime_error on input the
// real sz-conserved optimizer does not support (complex types, RBM, doublon-holon,
// general orbitals, pair-hop / exchange / InterAll terms).
Model read_expert(const std::string& namelist_path);

// QP weights: Gauss–Legendre spin projection × momentum projection weights.
void init_qp_weight(Model& m);

// init_parameter (parameter_init.rs:63): projection parameters zero, Slater
// parameters 2·(real2 − 0.5) for each optimized slot; `real2` draws SFMT genrand_real2.
void init_parameter(Model& m, const std::function<double()>& real2);

// sync_modified_parameter (parameter_init.rs:167): optional G/J shift, then Slater
// amplitudes rescaled to max |f| = 4.
void sync_modified_parameter(Model& m, bool shift_correlations);

// Load the last 6 + 3·NPara floats of an initial.def / zqp_opt.dat file.
// Returns false (and leaves the model untouched) when the file is absent or malformed.
bool read_para_triples(Model& m, const std::string& path, std::string* why = nullptr);

// Build SlaterElm[q][2Ns][2Ns] (row-major) for the current Slater parameters.
void build_slater_table(const Model& m, std::vector<double>& slater_elm);

// Translated site of `site` under momentum projection `mpidx` (opt-trans absent).
void translated_site(const Model& m, int site, int mpidx, int* out_site, int* out_sign);

// Flattened parameter vector in the reference order: G, J, Slater.
std::vector<double> all_parameters(const Model& m);
void set_all_parameters(Model& m, const std::vector<double>& p);

// ---- output files (C "% .18e" formatting) ----
std::string c_double(double v);  // "% .18e"
struct StepEnergy {
  double etot = 0, etot2 = 0, sztot = 0, sztot2 = 0;
};
void write_out_row(const Model& m, const std::string& dir, int step, const StepEnergy& e);
struct SrInfoRow {
  int npara, nsmat, opt_cut, diag_cut;
  double sdiag_max, sdiag_min, rmax;
  int imax, info;
};
void write_srinfo_row(const std::string& dir, const Model& m, bool first, const SrInfoRow& r);
struct OptPoint {
  double etot, etot2;
  std::vector<double> params;
};
void write_opt_files(const Model& m, const std::string& dir, const std::vector<OptPoint>& window);

// One PhysCal data block (io.rs:259-403): <head>_out_<index>.dat, <head>_var_<index>.dat
// and, for non-empty lists, <head>_cisajs_, <head>_cisajscktaltex_ and
// <head>_cisajscktalt_<index>.dat ("%03d" index). `one`, `two_ex` and `two` are the
// weight-averaged real Green functions in term order; imaginary parts are written as 0.
void write_physcal_block(const Model& m, const std::string& dir, int index, const StepEnergy& e,
                         const double* one, const double* two_ex, const double* two);

}  // namespace mvmc
