// Device-side model and walker-ensemble state shared by the sampler, measurement and
// SR kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace mvmcb {

// Read-only model tables (device pointers) and dimensions.
struct DevModel {
  int ns, ne, n, ns2, nqp, nproj, n_gutz, n_jast, norb, nleg, nmp, nex_path;
  int nterm, nintra, ninter, nhund;
  int warmup, interval, saved;  // NVMCWarmUp, NVMCInterval, samples saved per walker
  int sr_size;
  const double* slater;    // [nqp][ns2][ns2] row-major
  const float* slater32;   // FP32 copy (mixed path)
  const double* qpw;       // [nqp] QPFullWeight (real)
  const double* proj;      // [nproj] G then J parameter values
  const int* gutz_idx;     // [ns]
  const int* jast_idx;     // [ns*ns] (-1 undefined)
  const double* gutz_site; // [ns] direct projection tables (observables.rs:1553)
  const double* jast_pair; // [ns*ns]
  const int* orb_idx;      // [ns*ns]
  const int* orb_sgn;      // [ns*ns]
  const int* trans;        // [nmp*ns] translated site
  const int* trans_sgn;    // [nmp*ns] boundary sign (already 1 when periodic)
  const double* spgl;      // [3*nleg]: cs, cc, ss
  const int* tterm;        // [nterm*4]: i, si, j, sj
  const double* tval;      // [nterm]
  const int* intra_i;      // [nintra]
  const double* intra_v;
  const int* inter_ij;     // [ninter*2]
  const double* inter_v;
  const int* hund_ij;      // [nhund*2]
  const double* hund_v;
  // PhysCal Green functions. One-body terms: the output list first, then the one-body
  // values that coincident-index TwoBodyG terms reduce to. TwoBodyG terms carry the index
  // of that one-body value (ref, or -1) and of their two-hop slot (gen, or -1). A measured
  // sample's row holds [ngone one-body | ngtwo two-body | nggen two-hop] values (width gw).
  int ngone = 0, ngtwo = 0, nggen = 0, gw = 0;
  int gacc_smem = 0;          // set by the launcher: one-body plane sums in shared memory
  // Dense one-body lists: all (empty destination, electron) pairs of a spin are evaluated
  // as one product per plane; gterm_of[(s·ns + i)·ns + j] = first one-body term
  // (i s j s) with i != j (or -1), gfirst[k] = first term equal to term k.
  int gdense = 0;
  const int* gterm_of = nullptr;
  const int* gfirst = nullptr;
  // Slater-derivative site pairs by orbital: the translated site pairs (a', b') with
  // orb_idx[a'·ns + b'] = k are orb_ent[orb_off[k] .. orb_off[k+1]), packed as
  // (a' << 16) | (b' << 1) | (orb_sgn < 0); trans_inv[mp·ns + a'] is the site a with
  // translation mp mapping a to a' (null when a translation is not a permutation).
  const int* orb_off = nullptr;
  const int* orb_ent = nullptr;
  const int* trans_inv = nullptr;
  const int* gone = nullptr;  // [ngone*4]: i, s, j, t of c†_{i s} c_{j t}
  const int* gtwo = nullptr;  // [ngtwo*8]: ri, rj, rk, rl, s, u, ref, gen
  const int* ggen = nullptr;  // [nggen*6]: ri, rj, rk, rl, s, u of the two-hop terms
  // Resident measurement: each saved sample's Pf [nqp] and X⁻¹ [nqp][n][n] (FP64) as the
  // sampler held them at the save point; null = recompute them from the configuration.
  const double* rinv = nullptr;
  const double* rpf = nullptr;
};

// Per-walker persistent state, arrays of W entries each.
struct DevWalkers {
  int W;
  uint32_t* sfmt;             // [W*624]
  int* sfmt_idx;              // [W]
  unsigned long long* draws;  // [W]
  int* ele_idx;               // [W*n]
  int* ele_cfg;               // [W*ns2]
  int* ele_num;               // [W*ns2]
  int* proj_cnt;              // [W*nproj]
  int* burn;                  // [W]
  void* inv;                  // [W*nqp*n*n] planes when not shared-memory resident
  double* ws64;               // [W*n*n] FP64 refresh workspace (mixed path)
  double* pf;                 // [W*nqp]
  long long* counter;         // [W*6]
  int* s_idx;                 // [W*saved*n]
  int* s_cfg;                 // [W*saved*ns2]
  int* s_num;                 // [W*saved*ns2]
  int* s_cnt;                 // [W*saved*nproj]
  unsigned* status;           // [1] sticky
  int refresh_sweeps;         // mixed path: extra FP64 refresh cadence in sweeps (0 = off)
  unsigned long long* timers; // [W*8] clock cycles per sampler phase, or null (off)
  double* drift;              // [W] max |Δ ln|IP|| between the tracked and the refreshed amplitude
  long long* nrefresh;        // [W*2] scheduled (C rule / NRefresh) and guard-triggered refreshes
  double refresh_guard;       // refresh after an accepted move with a plane ratio outside [g, 1/g] (0 off)
  double* s_inv = nullptr;    // [W*saved*nqp*n*n] FP64 X⁻¹ at each save point (resident measurement), or null
  double* s_pf = nullptr;     // [W*saved*nqp] Pf at each save point
};

// One walker's Pfaffian stage buffers (device): FP64 planes and sweep scratch, Pf, the
// proposal Pf, the candidate configuration and the recomputation status.
struct StageBufs {
  double* planes;  // [nqp][n][n] row-major InvM (= X^-1)
  double* ws;      // [2][n][n]
  double* pf;      // [nqp]
  double* pfn;     // [nqp]
  const int* idx;  // [n]
  int* info;       // [1]
};
enum StageOp { kStageRecompute = 0, kStageProposeHop, kStageAcceptHop, kStageProposeExchange, kStageAcceptExchange };
constexpr int kStageThreads = 256;

// Sampler phases timed by thread 0 of each walker (cycles, barrier waits included):
// candidate, ratio, metropolis, update, refresh, total.
enum SamplerPhase { kPhCandidate = 0, kPhRatio, kPhMetropolis, kPhUpdate, kPhRefresh, kPhTotal, kPhCount = 8 };

// Arguments of the cooperative SR-CG solve.
struct CgArgs {
  const double* O;     // [ns][na] active sample matrix (rows = samples)
  const double* mean;  // [na]
  const double* diag;  // [na]
  const double* g;     // [na]
  double* x;           // [na] solution
  double* r;           // [na] residual
  double* d;           // [na] direction
  double* q;           // [na] product / preconditioned residual
  double* y;           // [ns]
  double* part;        // [nchunk][na] column partial sums
  double* red;         // [gridDim] block partials
  double* scal;        // [8]: delta, status, iterations
  long long ns;
  int na, nchunk, max_iter, diag_scale;
  double inv_w, shift, tol;
  // Reduced-precision operator (o_kind 1: FP32, 2: BF16): the centred, column-scaled
  // active matrix Ol[s][i] = (O[s][i] − ⟨O⟩_i)/cs[i] (zero rows for skipped samples), row
  // stride lda, so that S·v = Wc⁻¹·cs ⊙ Olᵀ(Ol·(cs ⊙ v)) + shift·diag ⊙ v. o_kind 0 uses O.
  // o_kind 3: Ol is the FP32 Gram G = OlᵀOl (na × na, row stride lda) formed on the tensor
  // cores, so that S·v = Wc⁻¹·cs ⊙ G·(cs ⊙ v) + shift·diag ⊙ v.
  const void* Ol = nullptr;
  const double* cs = nullptr;  // [na]
  int lda = 0;
  int o_kind = 0;
};

}  // namespace mvmcb
