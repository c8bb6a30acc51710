// Oracle: CPU restatement of the VMC sampling + SR hot path of AtelierArith/mvmc-rs.
//
// TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA path: tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline leg (and `bench.py --impl
// reference`) are the only callers. The product (mvmc-rs_b200/) never links it.
//
// Parity is pinned against the reference's own C-1.4.0 fixtures, read as text:
//   * SFMT19937 first words per seed (crates/sfmt19937/tests/golden_vs_c.rs)
//   * every saved configuration, counter, draw count and the next 624 SFMT words of a
//     native C sampler run (tests/fixtures/native_c_physcal_181/hubbard_chain_real)
//   * the PhysCal Green functions zvo_cisajs / zvo_cisajscktalt / zvo_cisajscktaltex of
//     that run on 1, 2 and 4 chains (native_c_physcal_181/hubbard_chain_real{,_mpi2,_mpi4})
//   * step-1 SR operands E, HO, <O>, <O^2>, last O (tests/fixtures/c_order_sr_operands)
//   * pfapack identities on tests/fixtures/pfapack/real_n*.orig.txt
#pragma once
#include <cstdint>

#ifdef __cplusplus
extern "C" {
#endif

// SFMT19937: first `count` gen_rand32 words after init_gen_rand(seed).
void oracle_sfmt_words(uint32_t seed, int count, uint32_t* out);

// Batched Pfaffian + inverse of skew-symmetric planes (column-major, back to back).
// Mirrors PfaffianStages::pfaffian_inverse_batch: `inv` receives the true X^-1,
// `status[p]` = 0 ok, k > 0 the 1-based zero-pivot row, -1 non-finite Pfaffian.
void oracle_pfinv_batch(const double* x, int n, int planes, double* pf, double* inv, int* status);

// Full optimisation run (vmc_para_opt) with W independent chains seeded RndSeed + w.
// Writes zvo_out.dat / zvo_var.dat / zvo_SRinfo.dat / zqp_*opt.dat into out_dir.
// nsteps <= 0 keeps NSROptItrStep. Returns 0 on success, nonzero on failure; the
// message is copied to `err` (size err_len).
int oracle_run_opt(const char* namelist, const char* initial_def, const char* out_dir,
                   int walkers, int nsteps, long long seed_override, char* err, int err_len);

// One optimisation step's SR operands before the solve (C NSROptItrStep = 1), for the
// step-1 fixtures. Overrides: NSRCG=cg, NStore=store, RndSeed=seed. Outputs (sizes
// sr_size = 1 + NPara): energy[1], ho[sr_size], oo[2*sr_size] (mean then diagonal),
// o_last[sr_size].
int oracle_step1_operands(const char* namelist, int cg, int store, long long seed,
                          double* energy, double* ho, double* oo, double* o_last, int sr_size,
                          char* err, int err_len);

// PhysCal sampling with fixed parameters from zqp_opt.dat (vmc_phys_cal): records every
// saved configuration of NDataQtySmp sample blocks. Output arrays are sized by the
// caller: ele_idx[blocks*NS*nsize], ele_cfg[blocks*NS*2Ns], ele_num[same],
// proj_cnt[blocks*NS*NProj], counters[blocks*6], draws[blocks], next624[blocks*624],
// energies[blocks*2] (<E>, <E^2> of each block's measurement).
int oracle_physcal_samples(const char* namelist, const char* zqp_opt, long long seed,
                           int64_t* ele_idx, int64_t* ele_cfg, int64_t* ele_num,
                           int64_t* proj_cnt, int64_t* counters, int64_t* draws,
                           uint32_t* next624, double* energies, char* err, int err_len);

// Green-function list sizes of a namelist: dims[0] one-body terms (canonical, as output),
// dims[1] TwoBodyGEx terms, dims[2] TwoBodyG terms, dims[3] NDataQtySmp, dims[4] NDataIdxStart.
int oracle_green_dims(const char* namelist, int* dims, char* err, int err_len);

// PhysCal run (vmc_phys_cal_in_place_with_options_timed, run.rs:980-1156) with fixed
// parameters from zqp_opt.dat over `walkers` chains seeded seed + w, each consuming its
// initial-parameter draws first. For every data block b: energy[4b..] = weight-averaged
// Etot, Etot2, Sztot, Sztot2; one[b*dims[0]..], ex[b*dims[1]..], two[b*dims[2]..] = the
// Green functions, each chain's sums scaled by its 1/Wc, summed over chains in order and
// scaled by 1/walkers (normalize_physcal_green run.rs:287, average_physcal_rank_
// contributions run.rs:1158). With out_dir non-empty it also writes the block files.
int oracle_physcal_green(const char* namelist, const char* zqp_opt, long long seed, int walkers,
                         double* energy, double* one, double* ex, double* two, const char* out_dir,
                         char* err, int err_len);

// Identity check of the Green-function ratios: one PhysCal block on one chain; for every
// valid sample and every one-body hop and general (two-hop) TwoBodyG term whose moves are
// allowed, the update-formula ratio against exp(Σ α Δc)·IP(x')/IP(x) with IP(x') from a
// fresh CalculateMAll of the moved configuration. out[0] = largest relative difference,
// out[1] = number of one-body hops checked, out[2] = number of two-hop terms checked.
int oracle_green_identity(const char* namelist, const char* zqp_opt, long long seed, double* out, char* err,
                          int err_len);

// Step 1 of an optimisation with W chains (seed + w): every walker's saved samples,
// counters, draw counts, the O store [W][S][sr_size] and the reduced operands
// (energy[5] = Wc, <E>, <E^2>, <Sz>, <Sz^2>; ho[sr_size]; oo[2*sr_size]).
int oracle_opt_step1_walkers(const char* namelist, const char* initial_def, int walkers,
                             long long seed, int64_t* ele_idx, int64_t* proj_cnt, int64_t* counters,
                             int64_t* draws, double* energy, double* ho, double* oo, double* ostore,
                             char* err, int err_len);

// SR-CG on fixed operands (SampledSrOperator::solve_with_product): samples are
// [samples][n]; returns the C status (iterations, or -(iter+1)). z_apply (optional)
// receives S·g.
int oracle_cg_fixed(int n, int samples, const double* mean, const double* diag, const double* smp,
                    const double* g, double inv_w, double shift, double tol, int max_iter,
                    int diag_scale, double* x_out, double* z_apply);

// Teacher-forced replay of the RealPfStage operations (sampling/stage.rs:56-129) on one
// walker: Slater table of `params`, inverses of idx0, then nops calls with rows
// ops[7k..] = {code, ma, sa, mb, sb, ra_old, rb_old} (0 propose hop, 1 accept hop, 2 propose
// exchange, 3 accept exchange, 4 recompute) and the call's ele_idx in idx_seq[k*n..].
// out[k*nqp..]: pf_new of a proposal, else the current Pf; inv_out: the final InvM planes.
int oracle_stage_replay(const char* namelist, const double* params, int npara, const int64_t* idx0, int nops,
                        const int* ops, const int64_t* idx_seq, double* out, double* inv_out, char* err,
                        int err_len);

// One FP64 chain (walker `walker` of the first SR step: RndSeed + walker, parameters as in
// oracle_opt_step1_walkers) run for min(blocks, warm-up + samples) blocks with a long-double
// shadow of its Pfaffians and inverses, teacher-forced on the FP64 decisions. Returns the
// start configuration idx0[n] and the chain's stage operations in the format of
// oracle_stage_replay (ops[7k..], candidate configurations cands[k*n..]), at most max_ops,
// with rec[8k..]: for a proposal {dproj, u, log-weight FP64, log-weight long double,
// accepted, ln|IP| tracked FP64, ln|IP| tracked long double, min_q |pf'_q/pf_q|}; for a
// recompute {ln|IP| tracked FP64 before, recomputed FP64, recomputed long double, tracked
// long double before}; zeros for accepts.
int oracle_trace_chain(const char* namelist, const char* initial_def, long long seed, int walker, int blocks,
                       int max_ops, int64_t* idx0, int32_t* ops, int64_t* cands, double* rec, int* nops,
                       char* err, int err_len);

// The QP weights of the model (init_qp_weight): out[nqp].
int oracle_qp_weights(const char* namelist, double* out, char* err, int err_len);

// Largest |ln|IP|_recomputed − ln|IP|_tracked| at a sampler refresh since the last reset
// (the FP64 rank-2 updates' drift on the C refresh schedule); reset != 0 clears it.
double oracle_refresh_drift(int reset);

// The refresh guard of the device's mixed path, restated for the FP64 chain: recompute right
// after an accepted move whose Pfaffian ratio on any QP plane lies outside [g, 1/g]
// (0 = off, the reference's schedule). Counts: scheduled and guard refreshes since reset.
void oracle_set_refresh_guard(double g);
void oracle_refresh_counts(long long* sched, long long* guard, int reset);
/* 1: the local energy's projection ratios use fixed_exp (a fixed IEEE operation sequence the
 * device's C-order mode reproduces bit for bit); 0 (default): the platform libm's exp. */
void oracle_set_fixed_exp(int on);
double oracle_fixed_exp(double x);

// The direct SR solve (LAPACK dpotrf('U') + dpotrs order): a is n×n row-major symmetric,
// overwritten by U (a = UᵀU) in its upper triangle; b becomes x. Returns 0, the 1-based
// failing pivot, or -1 for a non-finite solution.
int oracle_cholesky_solve(double* a, double* b, int n);

// Model dimensions for buffer sizing: [nsite, ne, nqp, nproj, npara, nvmc_sample,
// data_qty_smp, n_orb].
int oracle_model_dims(const char* namelist, int* dims, char* err, int err_len);

#ifdef __cplusplus
}
#endif
