// K10: Gram matrix of the SR sample matrix on the 5th-generation tensor cores.
//
// G = Õᵀ·Õ over the centred, column-scaled active sample matrix
// Õ[s][i] = (O[s][i] − ⟨O⟩_i)/cs_i (zero rows for skipped samples), so that the SR matrix
// is S = Wc⁻¹·diag(cs)·G·diag(cs) (+ the diagonal shift): the Oᵀ(O·v) − (⟨O⟩·v)⟨O⟩ product
// of SampledSrOperator::apply_with_product (crates/mvmc-core/src/sr_cg.rs:952-1009) formed
// once per SR step instead of once per CG iteration, and the Gram of the direct solve
// (gram_real, sr_backend.rs:464; the reference GPU path runs it as a cuBLAS dgemm,
// gpu/mvmc-gpu-cuda/src/opt.rs:1133-1147).
//
// Õ is staged transposed, Õᵀ[na_pad][ld] with samples contiguous (K-major for both MMA
// operands), in BF16 or FP32 (TF32 MMA). One CTA of four warps computes one 128×128 tile
// of G: warp 0 (one thread) streams 128-row × 128-byte K slabs of the two operand tiles
// with TMA (128-byte swizzle) into a 4-stage shared-memory ring guarded by mbarriers; warp 1
// (one thread) issues tcgen05.mma (M = N = 128, K = 16 BF16 / 8 TF32 per instruction) into
// a 128-column FP32 accumulator in tensor memory and commits each stage back to the ring;
// all four warps read the accumulator with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31)
// and store the tile. Every wait is bounded: on expiry the CTA records kGramTimeout in the
// status word, still frees its tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <vector>

#include "../host/abi_common.h"
#include "common.cuh"

namespace mvmcb {

constexpr int kGramTile = 128;            // M = N = 128 per CTA
constexpr int kGramStages = 4;            // TMA ring depth
constexpr int kGramSlabBytes = 128 * 128;  // one operand slab: 128 rows × 128 bytes
constexpr unsigned kGramTimeout = kDevTimeout;  // status bit: a bounded wait expired
constexpr long long kGramSpin = 1LL << 26;  // polls before a wait gives up

struct GramSmem {
  uint8_t a[kGramStages][kGramSlabBytes];  // 1024-byte aligned slabs (swizzle atoms)
  uint8_t b[kGramStages][kGramSlabBytes];
  uint64_t full[kGramStages];
  uint64_t empty[kGramStages];
  uint64_t done;
  uint32_t tmem_base;
  int bad;
  int issued;    // K slabs whose TMA loads were issued
  int consumed;  // K slabs whose loads the MMA thread saw land
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, unsigned phase) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

// Bounded wait for the barrier phase; false when it expired.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned phase) {
  for (long long k = 0; k < kGramSpin; ++k)
    if (mbar_test(bar, phase)) return true;
  return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Shared-memory matrix descriptor of a K-major slab with 128-byte swizzle: start address,
// leading byte offset 16 B (unused by the swizzled K-major form), stride byte offset
// 1024 B between 8-row groups, descriptor version 1, layout type 2 (128-byte swizzle).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  return static_cast<uint64_t>((addr >> 4) & 0x3fff) | (static_cast<uint64_t>(1) << 16) |
         (static_cast<uint64_t>(1024 >> 4) << 32) | (static_cast<uint64_t>(1) << 46) |
         (static_cast<uint64_t>(2) << 61);
}

// Instruction descriptor: FP32 accumulator, A and B of format `fmt` (1 BF16, 2 TF32), both
// K-major, N = 128, M = 128.
__host__ __device__ constexpr uint32_t gram_idesc(uint32_t fmt) {
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);
}

template <bool kTf32>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  if constexpr (kTf32)
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc));
  else
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// One 128×128 tile (blockIdx.x, blockIdx.y) of G = A·Aᵀ, A = Õᵀ[na][k] (K-major, `kblocks`
// slabs of 128 bytes). Tiles strictly above the diagonal are skipped: the lower tile is
// stored together with its transpose.
template <bool kTf32>
__global__ void __launch_bounds__(128, 1)
    k_gram_tc(const __grid_constant__ CUtensorMap map, int na, int kblocks, float* __restrict__ G, int ldg,
              unsigned* status) {
  const int bm = blockIdx.y, bn = blockIdx.x;
  if (bn > bm) return;
  extern __shared__ uint8_t smem_raw[];
  // the slabs start on 1024-byte boundaries of the shared address space (swizzle atoms)
  const uint32_t pad = (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
  GramSmem& sh = *reinterpret_cast<GramSmem*>(smem_raw + pad);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kGramStages; ++s) {
      mbar_init(&sh.full[s], 1);
      mbar_init(&sh.empty[s], 1);
    }
    mbar_init(&sh.done, 1);
    sh.bad = 0;
    sh.issued = 0;
    sh.consumed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {  // 128 accumulator columns (FP32: one per output column)
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh.tmem_base)),
                 "r"(128)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = sh.tmem_base;
  const int m0 = bm * kGramTile, n0 = bn * kGramTile;
  const int kstep = kTf32 ? 32 : 64;  // elements per 128-byte slab row
  if (warp == 0 && lane == 0) {
    // producer: slab kb of both operand tiles into stage kb % S
    for (int kb = 0; kb < kblocks; ++kb) {
      const int s = kb % kGramStages;
      if (kb >= kGramStages && !mbar_wait(&sh.empty[s], ((kb / kGramStages) - 1) & 1)) {
        atomicOr(status, kGramTimeout);
        sh.bad = 1;
        break;
      }
      mbar_expect_tx(&sh.full[s], bm == bn ? kGramSlabBytes : 2 * kGramSlabBytes);
      tma_load_2d(sh.a[s], &map, kb * kstep, m0, &sh.full[s]);
      if (bm != bn) tma_load_2d(sh.b[s], &map, kb * kstep, n0, &sh.full[s]);
      sh.issued = kb + 1;
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issue: four K steps of 32 bytes per slab (16 BF16 or 8 TF32 each)
    constexpr uint32_t idesc = gram_idesc(kTf32 ? 2u : 1u);
    for (int kb = 0; kb < kblocks; ++kb) {
      const int s = kb % kGramStages;
      if (!mbar_wait(&sh.full[s], (kb / kGramStages) & 1)) {
        atomicOr(status, kGramTimeout);
        sh.bad = 1;
        break;
      }
      sh.consumed = kb + 1;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a_addr = smem_u32(sh.a[s]);
      const uint32_t b_addr = bm == bn ? a_addr : smem_u32(sh.b[s]);
#pragma unroll
      for (int t = 0; t < 4; ++t)
        umma<kTf32>(tmem, sw128_desc(a_addr + 32 * t), sw128_desc(b_addr + 32 * t), idesc, (kb | t) != 0 ? 1u : 0u);
      umma_commit(&sh.empty[s]);  // the stage is free once these MMAs have read it
    }
    umma_commit(&sh.done);
  }
  __syncwarp();
  // epilogue: all four warps wait for the accumulator
  const bool ok = mbar_wait(&sh.done, 0);
  if (!ok && lane == 0) atomicOr(status, kGramTimeout);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < kGramTile; c0 += 32) {
      uint32_t v[32];
      tmem_ld32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + c0, v);
      if (row < na) {
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int col = n0 + c0 + j;
          if (col < na) {
            const float g = __uint_as_float(v[j]);
            G[static_cast<size_t>(row) * ldg + col] = g;
            if (bm != bn) G[static_cast<size_t>(col) * ldg + row] = g;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (sh.bad && threadIdx.x == 0) {
    // after an expired wait: let the loads still in flight (issued, not seen to land by the
    // MMA thread; at most one per stage) complete before the CTA's shared memory is released
    for (int kb = sh.consumed; kb < sh.issued; ++kb) mbar_wait(&sh.full[kb % kGramStages], (kb / kGramStages) & 1);
  }
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128) : "memory");
}

// Õᵀ[i][s] = (store[s][map[i] + 1] − mean[i]) / cs[i] for valid samples (the stored row's
// leading 1 is non-zero), 0 for skipped samples and for the padding rows i ≥ na and columns
// s ≥ ns, transposed through 32×33 shared tiles.
template <typename OT>
__global__ void k_gram_stage(const double* __restrict__ store, int sr_size, long long ns, const int* __restrict__ map,
                             int na, int na_pad, long long ld, const double* __restrict__ mean,
                             const double* __restrict__ cs, OT* __restrict__ out) {
  __shared__ float tile[32][33];
  const long long s0 = static_cast<long long>(blockIdx.x) * 32;
  const int i0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 × 8 threads
  for (int r = ty; r < 32; r += 8) {
    const long long s = s0 + r;
    const int i = i0 + tx;
    float v = 0.0f;
    if (s < ns && i < na && store[s * sr_size] != 0.0)
      v = static_cast<float>((store[s * sr_size + map[i] + 1] - mean[i]) / cs[i]);
    tile[r][tx] = v;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int i = i0 + r;
    const long long s = s0 + tx;
    if (i < na_pad && s < ld) {
      const float v = tile[tx][r];
      if constexpr (sizeof(OT) == 2)
        out[static_cast<long long>(i) * ld + s] = __float2bfloat16_rn(v);
      else
        out[static_cast<long long>(i) * ld + s] = v;
    }
  }
}

namespace {
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}
}  // namespace

// Staged operand sizes: rows padded to the tile, samples to one 128-byte slab.
void gram_tc_dims(int na, long long ns, int precision, int* na_pad, long long* ld) {
  *na_pad = (na + kGramTile - 1) / kGramTile * kGramTile;
  const long long slab = precision == 16 ? 64 : 32;
  *ld = std::max<long long>(slab, (ns + slab - 1) / slab * slab);
}

int launch_gram_stage(const double* store, int sr_size, long long ns, const int* map, int na, const double* mean,
                      const double* cs, int precision, void* staged, cudaStream_t stream) {
  int na_pad = 0;
  long long ld = 0;
  gram_tc_dims(na, ns, precision, &na_pad, &ld);
  const dim3 grid(static_cast<unsigned>((ld + 31) / 32), static_cast<unsigned>((na_pad + 31) / 32));
  if (precision == 16)
    k_gram_stage<__nv_bfloat16><<<grid, 256, 0, stream>>>(store, sr_size, ns, map, na, na_pad, ld, mean, cs,
                                                          static_cast<__nv_bfloat16*>(staged));
  else
    k_gram_stage<float><<<grid, 256, 0, stream>>>(store, sr_size, ns, map, na, na_pad, ld, mean, cs,
                                                  static_cast<float*>(staged));
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

// G[na][ldg] (FP32, full symmetric matrix) of the staged Õᵀ; precision 16 (BF16) or 32 (TF32).
int launch_gram_tc(const void* staged, int na, long long ns, int precision, float* G, int ldg, unsigned* status,
                   cudaStream_t stream) {
  if (precision != 16 && precision != 32) return kErrArgument;
  auto encode = tensor_map_encoder();
  if (!encode) {
    set_last_error("gram: cuTensorMapEncodeTiled unavailable");
    return kErrCuda;
  }
  int na_pad = 0;
  long long ld = 0;
  gram_tc_dims(na, ns, precision, &na_pad, &ld);
  const int esize = precision == 16 ? 2 : 4;
  CUtensorMap map;
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(ld), static_cast<cuuint64_t>(na_pad)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld) * esize};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(128 / esize), 128};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode(&map, precision == 16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                            2, const_cast<void*>(staged), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_last_error("gram: tensor map encoding failed");
    return kErrCuda;
  }
  const int kblocks = static_cast<int>(ld * esize / 128);
  const size_t smem = sizeof(GramSmem) + 1024;
  const dim3 grid(na_pad / kGramTile, na_pad / kGramTile);
  if (precision == 16) {
    MVMCB_CUDA(cudaFuncSetAttribute(k_gram_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    k_gram_tc<false><<<grid, 128, smem, stream>>>(map, na, kblocks, G, ldg, status);
  } else {
    MVMCB_CUDA(cudaFuncSetAttribute(k_gram_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    k_gram_tc<true><<<grid, 128, smem, stream>>>(map, na, kblocks, G, ldg, status);
  }
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

}  // namespace mvmcb

using namespace mvmcb;

namespace {
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};
}  // namespace

// Fixed-operand form for parity tests: samples[ns][na] (host, row-major) → gram[na][na]
// (host, FP32) = Σ_s x_s x_sᵀ with the samples rounded to BF16 (precision 16) or read as
// TF32 from FP32 (precision 32) on the tensor cores. Status 1 when a bounded wait expired.
extern "C" int mvmc_b200_gram_tc(const double* samples, long long ns, int na, int precision, float* gram) {
  if (!samples || !gram || ns <= 0 || na <= 0 || (precision != 16 && precision != 32)) return kErrArgument;
  const int sr = na + 1;
  std::vector<double> store(static_cast<size_t>(ns) * sr);
  for (long long s = 0; s < ns; ++s) {
    store[s * sr] = 1.0;
    for (int i = 0; i < na; ++i) store[s * sr + 1 + i] = samples[s * na + i];
  }
  std::vector<int> map(na);
  for (int i = 0; i < na; ++i) map[i] = i;
  std::vector<double> mc(2 * static_cast<size_t>(na), 0.0);
  for (int i = 0; i < na; ++i) mc[na + i] = 1.0;
  int na_pad = 0;
  long long ld = 0;
  gram_tc_dims(na, ns, precision, &na_pad, &ld);
  DevBuf dstore, dmap, dmc, dstaged, dg, dst;
  MVMCB_CUDA(cudaMalloc(&dstore.p, store.size() * sizeof(double)));
  MVMCB_CUDA(cudaMalloc(&dmap.p, map.size() * sizeof(int)));
  MVMCB_CUDA(cudaMalloc(&dmc.p, mc.size() * sizeof(double)));
  MVMCB_CUDA(cudaMalloc(&dstaged.p, static_cast<size_t>(na_pad) * ld * (precision == 16 ? 2 : 4)));
  MVMCB_CUDA(cudaMalloc(&dg.p, static_cast<size_t>(na) * na * sizeof(float)));
  MVMCB_CUDA(cudaMalloc(&dst.p, sizeof(unsigned)));
  MVMCB_CUDA(cudaMemset(dst.p, 0, sizeof(unsigned)));
  MVMCB_CUDA(cudaMemcpy(dstore.p, store.data(), store.size() * sizeof(double), cudaMemcpyHostToDevice));
  MVMCB_CUDA(cudaMemcpy(dmap.p, map.data(), map.size() * sizeof(int), cudaMemcpyHostToDevice));
  MVMCB_CUDA(cudaMemcpy(dmc.p, mc.data(), mc.size() * sizeof(double), cudaMemcpyHostToDevice));
  const double* mean = static_cast<const double*>(dmc.p);
  int rc = launch_gram_stage(static_cast<const double*>(dstore.p), sr, ns, static_cast<const int*>(dmap.p), na, mean,
                             mean + na, precision, dstaged.p, nullptr);
  if (rc != kOk) return rc;
  rc = launch_gram_tc(dstaged.p, na, ns, precision, static_cast<float*>(dg.p), na, static_cast<unsigned*>(dst.p),
                      nullptr);
  if (rc != kOk) return rc;
  unsigned st = 0;
  MVMCB_CUDA(cudaMemcpy(gram, dg.p, static_cast<size_t>(na) * na * sizeof(float), cudaMemcpyDeviceToHost));
  MVMCB_CUDA(cudaMemcpy(&st, dst.p, sizeof(unsigned), cudaMemcpyDeviceToHost));
  return (st & kGramTimeout) ? 1 : kOk;
}
