/* mvmc_b200.h — C ABI of the B200-native VMC sampling + SR hot path.
 *
 * The entry points replace the in-process stage seams of AtelierArith/mvmc-rs that the
 * `mvmc` optimizer loop (crates/mvmc-core/src/run.rs:1226-1502, vmc_para_opt_timed)
 * calls; each declaration names the reference interface it stands in for.
 *
 * Conventions: plain pointers and sizes; `int` status 0 = ok, > 0 = numeric status
 * (1-based zero-pivot row), < 0 = error class (MVMC_B200_E*). No exceptions cross the
 * ABI. A context owns one CUDA stream and its device buffers; it is thread-compatible,
 * not thread-safe (stages are Send, not Sync: crates/mvmc-core/src/stage_backend.rs:1004).
 * There is no CPU fallback: without a CUDA device every compute entry point returns
 * MVMC_B200_ECUDA.
 */
#ifndef MVMC_B200_H
#define MVMC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MVMC_B200_OK 0
#define MVMC_B200_EARG (-1)
#define MVMC_B200_ECUDA (-2)
#define MVMC_B200_EMODEL (-3)
#define MVMC_B200_ENUMERIC (-4)
#define MVMC_B200_ETIMEOUT (-5)
#define MVMC_B200_ESTATE (-6)

/* ---------------------------------------------------------------------------------
 * Batched Pfaffian + inverse.
 * Replaces PfaffianStages::pfaffian_inverse_batch(x, n, planes) -> PfInvBatch
 * (crates/mvmc-core/src/stage_backend.rs:121-165): planes are column-major n×n back to
 * back; `inv` receives the true X⁻¹ (the caller negates for InvM); `status[p]` is 0,
 * the 1-based row of a zero pivot (PlaneOutcome::ZeroPivot), or -1 (NonFinite).
 * Host buffers; the call allocates device memory.
 * ------------------------------------------------------------------------------- */
int mvmc_b200_pfinv_batch(const double* x, int n, int planes, double* pf, double* inv,
                          int* status);

/* Mixed sizes in one launch: plane p has side sizes[p] and starts where plane p-1 ends.
 * precision 64 (FP64 sweep) or 32 (FP32 sweep, FP64 in/out). Host buffers. */
int mvmc_b200_pfinv_batch_mixed(const double* x, const int* sizes, int planes, int precision,
                                double* pf, double* inv, int* status);

/* Device-buffer form (no allocation): sizes/offsets may be NULL for a uniform batch of
 * side n_uniform; n_max bounds every side. stream is a cudaStream_t (NULL = default). */
int mvmc_b200_pfinv_batch_device(const double* x, const int* sizes, const long long* offsets,
                                 int n_uniform, int planes, int n_max, double* pf, double* inv,
                                 int* status, int precision, void* stream);

/* Complex skew planes (the Pfaffian + inverse of the complex mode's CalculateMAll,
 * calc_m_all_complex, crates/mvmc-core/src/pfaffian.rs:340-360): x holds `planes`
 * column-major n×n planes of (re, im) pairs; pf receives (re, im) per plane, inv the true
 * X⁻¹ in the same layout, status as mvmc_b200_pfinv_batch. FP64. */
int mvmc_b200_pfinv_batch_complex(const double* x, int n, int planes, double* pf, double* inv,
                                  int* status);

/* Device-buffer form of mvmc_b200_pfinv_batch_complex (PfaffianStages' complex batch on
 * device-resident planes; stage_backend.rs:121-165): same layouts, no allocation, launched
 * on `stream` (a cudaStream_t; NULL = default) and not synchronised. */
int mvmc_b200_pfinv_batch_complex_device(const double* x, int n, int planes, double* pf, double* inv,
                                         int* status, void* stream);

/* Gram matrix on the tensor cores (the Oᵀ·O of the SR matrix, SrStages::gram_real,
 * crates/mvmc-core/src/sr_backend.rs:464; the reference GPU path's cuBLAS dgemm,
 * gpu/mvmc-gpu-cuda/src/opt.rs:1133-1147): gram[na][na] (host, FP32) = Σ_s x_s x_sᵀ of
 * samples[ns][na] (host, row-major), the samples rounded to BF16 (precision 16) or read as
 * TF32 (precision 32), FP32 accumulation (tcgen05.mma). Returns 1 when a bounded device
 * wait expired (no result), < 0 on errors. Allocates device memory. */
int mvmc_b200_gram_tc(const double* samples, long long ns, int na, int precision, float* gram);

/* ---------------------------------------------------------------------------------
 * Walker ensemble engine.
 * ------------------------------------------------------------------------------- */
typedef struct mvmc_b200_ctx mvmc_b200_ctx;

typedef struct mvmc_b200_options {
  int walkers;          /* W independent chains, walker w seeded RndSeed + w (multichain.rs:88) */
  int precision;        /* 64: plain FP64 path; 32: FP32 rank-2 updates + FP64 refresh */
  int refresh_sweeps;   /* FP32 path: FP64 refresh every this many sweeps (0 = C rule only) */
  int saved_per_walker; /* samples saved per walker and SR step; 0 = NVMCSample (C semantics) */
  long long seed;       /* < 0: RndSeed of modpara.def */
  int device;           /* CUDA device ordinal */
  int sr_precision;     /* SR-CG sample matrix: 64 (or 0) FP64 in the C order; 32 FP32 or 16 BF16,
                         * centred and column-scaled, FP32 products (the mixed path's operator).
                         * Direct SR (NSRCG 0) with 32 / 16 assembles S from the tensor-core Gram
                         * of those samples (TF32 / BF16 inputs) and solves it in FP64. */
  double refresh_guard; /* g in [0, 1): FP64 refresh right after an accepted move whose Pfaffian
                         * ratio on any QP plane lies outside [g, 1/g]; 0 = off (C behaviour) */
  int c_order;          /* 1: measurement, its sums and SR-CG in the reference CPU path's operation
                         * order without FMA (pfapack LTLᵀ inverse, serial sums; results equal the
                         * CPU path's bit for bit up to libm's exp): the parity mode of the 10-step
                         * zvo_out.dat gate (phase5_zvo_gate_hubbard.rs:19-80). 0: throughput kernels. */
  int sr_gram;          /* 1 with sr_precision 16 / 32: SR-CG applies S through the Gram G = OᵀO of the
                         * centred, column-scaled samples, formed once per SR step on the tensor cores
                         * (BF16 / TF32 inputs, FP32 accumulation); 0: one pass over the samples per
                         * CG product */
  int measure_resident; /* 1 with precision 64: the sampler stores each saved sample's Pf and X⁻¹ as it
                         * holds them (after its rank-2 / rank-4 updates since the last refresh) and the
                         * measurement reads them instead of recomputing (the reference recomputes
                         * them, CalculateMAll per sample); W·saved·NQP·n² doubles of device memory.
                         * 0: recompute. */
} mvmc_b200_options;

void mvmc_b200_default_options(mvmc_b200_options* opt);

/* Parse the Expert-mode namelist (crates/mvmc-expert-parsers, parse_expert_mode_files) and
 * upload the model: Slater index tables, QP weights, projection index tables and the
 * Transfer / CoulombIntra / CoulombInter / Hund term lists. Parameters are initialised as
 * run_para_opt_timed does (run.rs:1696-1737: init_parameter per walker stream, optional
 * initial.def, sync_modified). */
int mvmc_b200_create(const char* namelist, const char* initial_def, const mvmc_b200_options* opt,
                     mvmc_b200_ctx** out);
void mvmc_b200_destroy(mvmc_b200_ctx* ctx);

/* Dimensions: [nsite, ne, nqp, nproj, npara, saved_per_walker, walkers, n_orb]. */
int mvmc_b200_dims(const mvmc_b200_ctx* ctx, int* dims);

/* Current parameters (G, J, Slater order) as pack_variational_parameters (sync.rs:20). */
int mvmc_b200_get_parameters(const mvmc_b200_ctx* ctx, double* params, int npara);
int mvmc_b200_set_parameters(mvmc_b200_ctx* ctx, const double* params, int npara);

/* One SR step's sampling for every walker: update_slater_elm (slater_update.rs:17) on the
 * device, then vmc_make_sample_real_engine (sampling/driver.rs:175-438) with
 * HostEngine::run_block's proposal loop (sampling/engine.rs:188-476) run resident on the
 * device: SFMT19937 per walker, hop/exchange proposals, rank-2 updates, refresh when the
 * accept window exceeds Nsite. Saved configurations stay on the device. */
int mvmc_b200_sample(mvmc_b200_ctx* ctx);

/* Download the saved configurations of the last mvmc_b200_sample (parity checks):
 * ele_idx[W*S*nsize], ele_cfg[W*S*2Ns], ele_num[W*S*2Ns], proj_cnt[W*S*nproj],
 * counters[W*6] (C Counter[0..6]), draws[W] (SFMT words consumed). Any pointer may be NULL. */
int mvmc_b200_get_samples(const mvmc_b200_ctx* ctx, int64_t* ele_idx, int64_t* ele_cfg,
                          int64_t* ele_num, int64_t* proj_cnt, int64_t* counters, int64_t* draws);

/* Local measurement of every saved sample (MeasurementStages::measure_sample,
 * stage_backend.rs:387-440; accumulate_observables_local, run.rs:2937-3614): Pfaffian and
 * inverse, IP, local energy, O = [1, projection counts, ∂lnΨ/∂f] written as rows of the SR
 * sample matrix (calculate_oo_store_real, observables.rs:297), then the rank-ordered
 * reduction and weight average (average.rs:18-80). energy[5] = {Wc, <E>, <E²>, <Sz>, <Sz²>};
 * ho[sr_size], oo[2*sr_size] (mean then diagonal) may be NULL. */
int mvmc_b200_measure(mvmc_b200_ctx* ctx, double* energy, double* ho, double* oo);

/* Rows of the SR sample matrix (W*S rows × sr_size, row-major) for parity checks. */
int mvmc_b200_get_o_store(const mvmc_b200_ctx* ctx, double* o_store, long long count);
/* Per-sample local energies (W*S). */
int mvmc_b200_get_local_energies(const mvmc_b200_ctx* ctx, double* e_loc, long long count);
/* Per-sample ln|Psi(x)| (W*S) of the last measurement: the Gutzwiller-Jastrow exponent
 * sum_k alpha_k c_k plus ln|IP| (calculate_ip_real, observables.rs:128; log_proj_ratio,
 * projection.rs:403). With set_parameters + measure on the same saved samples this gives
 * ln|Psi| at shifted parameters, the finite-difference check of the O rows. */
int mvmc_b200_get_log_amplitudes(const mvmc_b200_ctx* ctx, double* log_psi, long long count);

/* SR step of the model's mode. NSRCG 0 (direct): stochastic_opt_real_with_sr_info_timed
 * (sr.rs:77-160) — Gram, redundancy cut, S/g assembly and Cholesky solve on the device.
 * Otherwise SR-CG: stochastic_opt_cg_with_reducer (sr_cg.rs:201-490) with
 * SampledSrOperator::solve_with_product (sr_cg.rs:700-880) run on the device; S·v is
 * Oᵀ(O·v)/W − ⟨O⟩(⟨O⟩·v) + δ·diag(S)·v. Updates the parameters (update_parameter_value,
 * sr.rs:439) and applies sync_modified_parameter_local (sync.rs:87). sr_info receives
 * {npara, nsmat, opt_cut, diag_cut, sdiag_max, sdiag_min, rmax, imax, info}; returns 0, or
 * 1 when the update was non-finite and skipped, or < 0 on error. */
int mvmc_b200_sr_cg(mvmc_b200_ctx* ctx, double* sr_info);

/* SR-CG on fixed operands (SrStages::cg_step, crates/mvmc-core/src/sr_backend.rs:193-297;
 * the recurrence of SampledSrOperator::solve_with_product, sr_cg.rs:700-880). samples is
 * [ns][na] row-major; status receives the C status (iterations, or -(iter+1)). Host buffers. */
int mvmc_b200_cg_solve(const double* samples, long long ns, int na, const double* mean,
                       const double* diag, const double* g, double inv_w, double shift, double tol,
                       int max_iter, int diag_scale, double* x, long long* status);

/* SR-CG on device buffers without any device allocation. This entry point has no
 * counterpart in the reference: it serves callers whose device memory is owned by their
 * own allocator (a pooling framework allocator, a fixed memory budget), where a library
 * cudaMalloc would fragment the pool or overrun the budget and cudaMalloc/cudaFree would
 * synchronise the device. All pointers are device pointers: samples [ns][na] row-major,
 * mean/diag/g [na] inputs; x [na] and result [3] = {delta, status, iterations} outputs.
 * The working vectors live in an 8 MiB array compiled into the library (held on every
 * GPU that loads it until exit); problems needing more than 1048576 doubles of it
 * (3·na + ns + column and block partials) return MVMC_B200_EARG with a message. The first call on
 * a device looks up that array's device address; make it before any stream capture.
 * Calls share the array: calls that overlap on the GPU race and must be serialised.
 * stream is a cudaStream_t (NULL = default); the call returns once the solve is queued. */
int mvmc_b200_cg_solve_noalloc(const double* samples, long long ns, int na, const double* mean,
                               const double* diag, const double* g, double inv_w, double shift,
                               double tol, int max_iter, int diag_scale, double* x, double* result,
                               void* stream);

/* Sticky device status word (first failing stage wins): MVMC_B200_DEV_* bits. */
#define MVMC_B200_DEV_SINGULAR 1u
#define MVMC_B200_DEV_NONFINITE 2u
#define MVMC_B200_DEV_INITLOOPS 4u
#define MVMC_B200_DEV_BOUNDS 8u
#define MVMC_B200_DEV_CANDIDATE 16u
int mvmc_b200_status(mvmc_b200_ctx* ctx, unsigned* device_status);

/* The whole optimisation (run_para_opt_from_namelist, run.rs:1558; the `mvmc namelist.def`
 * CLI path): NSROptItrStep steps of sample → measure → SR-CG → sync, writing zvo_out.dat,
 * zvo_var.dat, zvo_SRinfo.dat and zqp_*opt.dat into out_dir. nsteps <= 0 keeps the
 * modpara value. */
int mvmc_b200_run_opt(const char* namelist, const char* initial_def, const char* out_dir,
                      const mvmc_b200_options* opt, int nsteps);

/* PhysCal (NVMCCalMode 1) with fixed parameters: replaces prepare_phys_cal_from_namelist
 * (crates/mvmc-core/src/run.rs:555) and vmc_phys_cal_to_dir (run.rs:751-780). Each walker
 * consumes its initial-parameter draws (seed + w), then the parameters are read from
 * zqp_opt (the last 6 + 3·NPara numbers) without the G/J shift and |NMPTrans| is used.
 * The OneBodyG / TwoBodyG / TwoBodyGEx lists of the namelist are measured. */
int mvmc_b200_physcal_create(const char* namelist, const char* zqp_opt, const mvmc_b200_options* opt,
                             mvmc_b200_ctx** out);
/* dims[5]: one-body terms (OneBodyG after the TwoBodyGEx canonical map, as written to
 * zvo_cisajs), TwoBodyGEx terms, TwoBodyG terms, NDataQtySmp, NDataIdxStart. */
int mvmc_b200_green_dims(const mvmc_b200_ctx* ctx, int* dims);
/* Measurement of the saved samples in the PhysCal form (accumulate_observables with
 * NVMCCalMode 1, run.rs:3300-3420; ordinary_green_values, observables/
 * green_measurements.rs:264): energy[5] = Wc, <E>, <E^2>, <Sz>, <Sz^2> (weight-averaged
 * over all walkers) and the Green functions one[dims[0]], two_ex[dims[1]], two[dims[2]]
 * (each walker's sums scaled by its 1/Wc, summed over walkers and scaled by 1/W, as
 * normalize_physcal_green run.rs:287 and average_physcal_rank_contributions run.rs:1158).
 * No O rows are written. Any output pointer may be null. */
int mvmc_b200_measure_green(mvmc_b200_ctx* ctx, double* energy, double* one, double* two_ex, double* two);
/* The PhysCal run: NDataQtySmp blocks of sample → measure, writing zvo_out_NNN.dat,
 * zvo_var_NNN.dat, zvo_cisajs_NNN.dat, zvo_cisajscktaltex_NNN.dat and
 * zvo_cisajscktalt_NNN.dat (NNN = NDataIdxStart + block, io.rs:259-403) into out_dir. */
int mvmc_b200_run_physcal(const char* namelist, const char* zqp_opt, const char* out_dir,
                          const mvmc_b200_options* opt);

/* Sampler phase timers (the device analogue of the C timers of the sampler substeps):
 * cycles[8] = {candidate, ratio, metropolis, update, refresh, total, -, -} summed over walkers
 * for the last mvmc_b200_sample, measured by each walker's control thread. Zero unless the
 * environment variable MVMC_B200_TIMERS=1 was set when the context was created. */
int mvmc_b200_sampler_timers(const mvmc_b200_ctx* ctx, double* cycles);

/* Accuracy of the incrementally updated amplitudes in the last mvmc_b200_sample. At every
 * FP64 refresh the drift |ln|IP|_refreshed − ln|IP|_tracked| is recorded; stats[4] =
 * {max over walkers of each walker's largest drift, mean of those, scheduled refreshes
 * per walker (C rule or refresh_sweeps), guard-triggered refreshes per walker}. */
int mvmc_b200_refresh_stats(const mvmc_b200_ctx* ctx, double* stats);

/* ---------------------------------------------------------------------------------
 * One walker's Pfaffian stage: the five operations of RealPfStage
 * (crates/mvmc-core/src/sampling/stage.rs:56-129) on device-resident FP64 inverses, for a
 * host-driven (teacher-forced) chain. The host keeps the configuration and the RNG and
 * passes the candidate configuration ele_idx[2*Ne] (sites, the move already applied) with
 * every call; the stage reads the context's Slater table (set_parameters rebuilds it).
 * Slots: electron ma of spin sa is slot ma + sa*Ne. Pfaffian vectors have NQP entries.
 * ------------------------------------------------------------------------------- */
typedef struct mvmc_b200_stage mvmc_b200_stage;

int mvmc_b200_stage_create(mvmc_b200_ctx* ctx, mvmc_b200_stage** out);
void mvmc_b200_stage_destroy(mvmc_b200_stage* stage);
/* begin (stage.rs:60): build the resident inverses of ele_idx; pf may be NULL. */
int mvmc_b200_stage_begin(mvmc_b200_stage* stage, const int64_t* ele_idx, double* pf);
/* propose_hop (stage.rs:71-81): pf_new[q] of the one-electron move of slot (ma, spin). */
int mvmc_b200_stage_propose_hop(mvmc_b200_stage* stage, const int64_t* ele_idx, int ma, int spin,
                                double* pf_new);
/* accept_hop (stage.rs:83-92): rank-2 inverse update; the current Pf become pf_new
 * (NULL keeps the update's own product). */
int mvmc_b200_stage_accept_hop(mvmc_b200_stage* stage, const int64_t* ele_idx, int ma, int spin,
                               const double* pf_new);
/* propose_exchange (stage.rs:94-102): pf_new of the two-electron exchange of slots
 * (ma, sa) and (mb, sb). */
int mvmc_b200_stage_propose_exchange(mvmc_b200_stage* stage, const int64_t* ele_idx, int ma, int sa,
                                     int mb, int sb, double* pf_new);
/* accept_exchange (stage.rs:104-114): rank-4 update; ra_old, rb_old are the sites before
 * the move. */
int mvmc_b200_stage_accept_exchange(mvmc_b200_stage* stage, const int64_t* ele_idx, int ma, int sa,
                                    int mb, int sb, int ra_old, int rb_old);
/* recompute (stage.rs:116-123): returns 1 on a numeric failure (zero pivot), 0 ok. */
int mvmc_b200_stage_recompute(mvmc_b200_stage* stage, const int64_t* ele_idx, double* pf);
/* Current Pf[NQP] and inverses inv_m[NQP][n*n] in mVMC's InvM layout (column-major -X^-1,
 * state.rs:208, without the pad slot); either may be NULL. */
int mvmc_b200_stage_state(const mvmc_b200_stage* stage, double* pf, double* inv_m);

/* SrStages::gram_real (crates/mvmc-core/src/sr_backend.rs:464): out[n][n] = Σ_s row_s row_sᵀ
 * of `samples` stored rows of n values (host buffers). */
int mvmc_b200_gram(const double* store, int n, long long samples, double* out);

/* SrStages::cholesky_solve (sr_backend.rs:243-247, sr.rs:535 dpotrf('U') + dpotrs): solve
 * S x = rhs for the symmetric positive-definite row-major n×n S (host buffers); rhs becomes
 * x. Returns 1 on a non-positive pivot or a non-finite solution (the reference's Err(())),
 * 0 on success. The engine's direct SR (NSRCG 0) runs the same kernels on device buffers. */
int mvmc_b200_cholesky_solve(const double* s, double* rhs, int n);

/* ---------------------------------------------------------------------------------
 * Walker-sharded SR across ranks (the reference's Reducer seam, reducer.rs:20-168, and
 * stochastic_opt_cg_with_reducer, sr_cg.rs:201-490): each rank samples and measures its
 * own walkers; the caller adds the measurement sums and every CG product across ranks,
 * runs the recurrence, and every rank applies the same update (mvmc-rs_b200/sharded.py).
 * ------------------------------------------------------------------------------- */
/* Sums of the last measurement over this context's walkers, before the weight average:
 * sums[5 + 3*sr_size] = {Wc, Σ E, Σ E², Σ Sz, Σ Sz², Σ HO[sr_size], Σ O[sr_size],
 * Σ O²[sr_size]}. */
int mvmc_b200_measure_sums(const mvmc_b200_ctx* ctx, double* sums);
/* Compact the active columns map[0..na) (parameter indices) of the stored O rows. */
int mvmc_b200_sr_gather(mvmc_b200_ctx* ctx, const int* map, int na);
/* SrStages::cg_local_product (sr_backend.rs:249-255): z = Σ_s O_s (O_s·v) over this
 * context's samples and the gathered columns; no mean, diagonal or cross-rank terms.
 * v, z: na host doubles. */
int mvmc_b200_sr_local_product(mvmc_b200_ctx* ctx, const double* v, double* z);

/* Device-buffer form of mvmc_b200_sr_local_product (SrStages::cg_local_product on
 * device-resident vectors, sr_backend.rs:249-255): v and z are device pointers (n_active
 * doubles) ordered on `stream` (a cudaStream_t); the product is joined to that stream with
 * events, no host copy is made and nothing is synchronised. A walker-sharded CG then reduces
 * z across ranks on the device (an NCCL all-reduce of z) without leaving the GPU. */
int mvmc_b200_sr_local_product_device(mvmc_b200_ctx* ctx, const double* v, double* z, void* stream);
/* Apply an SR solution: parameter map[i] += x[i], then sync_modified_parameter and the
 * upload (update_parameter_value, sr.rs:439; sync.rs:87). */
int mvmc_b200_sr_apply(mvmc_b200_ctx* ctx, const int* map, int na, const double* x);
/* SR settings: cfg[10] = {NSRCG, DSROptRedCut, DSROptStepDt, DSROptStaDel, DSROptCGTol,
 * NSROptCGMaxIter, DiagScale, CG fallback, CG abort-on-fail, NPara}; flags[2*NPara] the
 * optimisation flags (real, imaginary) per parameter (may be NULL). */
int mvmc_b200_sr_config(const mvmc_b200_ctx* ctx, double* cfg, int* flags);

/* The context's CUDA stream (a cudaStream_t), for timing and ordering with caller work. */
void* mvmc_b200_stream(mvmc_b200_ctx* ctx);

/* Bytes the context copied host→device and device→host since creation (counters). */
int mvmc_b200_transfer_bytes(const mvmc_b200_ctx* ctx, long long* h2d, long long* d2h);

/* Last error message of the calling thread (empty when none). */
const char* mvmc_b200_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* MVMC_B200_H */
