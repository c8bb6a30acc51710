// Batched Pfaffian + inverse of complex skew-symmetric planes: the computational core of
// the complex mode's CalculateMAll (calc_m_all_complex, crates/mvmc-core/src/pfaffian.rs:
// 340-360, which runs pfapack's complex LTLᵀ per QP plane).
//
// Same skew Gauss–Jordan sweep with 2×2 pivots as the real kernels (pfinv.cuh), in complex
// FP64: p = smallest unswept index, q = the first maximum of |Re A[p][j]| + |Im A[p][j]|
// over unswept j ≠ p (the 1-norm of IZAMAX that zsktf2 pivots by, crates/pfapack/src/ltl.rs:
// 38-41, which neither underflows nor overflows where |z|² would),
// A[i][j] += (A[q][i]/a)·A[p][j] − (A[p][i]/a)·A[q][j] with a = A[p][q], Pf = sgn(σ)·Πa.
// One CTA per plane sweeps it in place in the output buffer (L2-resident), rows p and q
// snapshot in shared memory. Planes are column-major (re, im) pairs as the real entry point
// takes them; the returned inverse is the true X⁻¹.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "../../include/mvmc_b200.h"
#include "common.cuh"

namespace mvmcb {

namespace {

struct cplx {
  double re, im;
};
__device__ __forceinline__ cplx cmul(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ cplx csub(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cplx cneg(cplx a) { return {-a.re, -a.im}; }
// 1/a by Smith's scaled division (no overflow of |a|² for large components)
__device__ __forceinline__ cplx cinv(cplx a) {
  if (fabs(a.re) >= fabs(a.im)) {
    const double r = a.im / a.re, d = a.re + a.im * r;
    return {1.0 / d, -r / d};
  }
  const double r = a.re / a.im, d = a.re * r + a.im;
  return {r / d, -1.0 / d};
}

constexpr int kCplxThreads = 256;

__global__ void __launch_bounds__(kCplxThreads)
    k_pfinv_complex(const cplx* __restrict__ x, int n, int planes, cplx* __restrict__ inv, cplx* __restrict__ pf,
                    int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem[];
  cplx* rowp = reinterpret_cast<cplx*>(smem);
  cplx* rowq = rowp + n;
  int* swept = reinterpret_cast<int*>(rowq + n);
  __shared__ int s_q, s_st, s_par;
  __shared__ double s_best;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  const size_t nn = static_cast<size_t>(n) * n;
  for (int plane = blockIdx.x; plane < planes; plane += gridDim.x) {
    const cplx* xp = x + plane * nn;
    cplx* A = inv + plane * nn;
    // column-major X read row-major is Xᵀ = −X: the negated buffer is X row-major
    for (size_t k = tid; k < nn; k += nt) A[k] = cneg(xp[k]);
    for (int j = tid; j < n; j += nt) swept[j] = 0;
    if (tid == 0) {
      s_st = 0;
      s_par = 0;
    }
    __syncthreads();
    int p = 0;
    cplx pfv{1.0, 0.0};
    for (int step = 0; step < n / 2; ++step) {
      for (int j = tid; j < n; j += nt) rowp[j] = A[static_cast<size_t>(p) * n + j];
      __syncthreads();
      if (warp == 0) {
        double best = -1.0;
        int bi = n;
        for (int j = lane; j < n; j += 32) {
          if (!swept[j] && j != p) {
            const double v = fabs(rowp[j].re) + fabs(rowp[j].im);
            if (v > best) {
              best = v;
              bi = j;
            }
          }
        }
        warp_argmax_first(best, bi);
        const int q = __shfl_sync(0xffffffffu, bi, 0);
        best = __shfl_sync(0xffffffffu, best, 0);
        int cnt = 0;
        for (int j = lane; j < n; j += 32) cnt += (!swept[j] && j > p && j < q) ? 1 : 0;
        for (int off = 16; off > 0; off >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
        if (lane == 0) {
          s_q = q;
          s_best = best;
          s_par += cnt;
        }
      }
      __syncthreads();
      const int q = s_q;
      if (!(s_best > 0.0)) {
        if (tid == 0) s_st = p + 1;
        break;  // every thread reads the same s_best: all leave together
      }
      const cplx a = rowp[q];
      pfv = cmul(pfv, a);
      const cplx ia = cinv(a);
      for (int j = tid; j < n; j += nt) rowq[j] = A[static_cast<size_t>(q) * n + j];
      __syncthreads();
      for (int i = warp; i < n; i += nwarp) {
        cplx* Ai = A + static_cast<size_t>(i) * n;
        if (i == p) {
          for (int j = lane; j < n; j += 32)
            Ai[j] = (j == q) ? cneg(ia) : (j == p ? cplx{0.0, 0.0} : cmul(rowq[j], ia));
        } else if (i == q) {
          for (int j = lane; j < n; j += 32)
            Ai[j] = (j == p) ? ia : (j == q ? cplx{0.0, 0.0} : cneg(cmul(rowp[j], ia)));
        } else {
          // coefficients scaled by 1/a first (as LTLᵀ forms t = α·A before its rank-2 step),
          // so that entries near the under- or overflow limits never meet in a product
          const cplx cq = cmul(rowq[i], ia), cp = cmul(rowp[i], ia);
          for (int j = lane; j < n; j += 32) {
            cplx v;
            if (j == p) v = cneg(cq);
            else if (j == q) v = cp;
            else v = cadd(Ai[j], csub(cmul(cq, rowp[j]), cmul(cp, rowq[j])));
            Ai[j] = v;
          }
        }
      }
      if (tid == 0) {
        swept[p] = 1;
        swept[q] = 1;
      }
      __syncthreads();
      int nxt = n;
      for (int j = 0; j < n; ++j)
        if (!swept[j]) {
          nxt = j;
          break;
        }
      p = nxt < n ? nxt : 0;
    }
    __syncthreads();
    int st = s_st;
    cplx v = (s_par & 1) ? cneg(pfv) : pfv;
    if (st == 0 && !(isfinite(v.re) && isfinite(v.im))) st = -1;
    if (st != 0) v = {0.0, 0.0};
    // row-major X⁻¹ negated is the column-major X⁻¹
    for (size_t k = tid; k < nn; k += nt) A[k] = cneg(A[k]);
    if (tid == 0) {
      pf[plane] = v;
      status[plane] = st;
    }
    __syncthreads();
  }
}

}  // namespace

}  // namespace mvmcb

namespace mvmcb {

// Stream-ordered launch on device buffers: x, inv hold `planes` column-major n×n complex
// planes as (re, im) doubles, pf `planes` complex values, status one int per plane.
int pfinv_complex_device(const double* x, int n, int planes, double* pf, double* inv, int* status,
                         cudaStream_t stream) {
  if (n <= 0 || (n & 1) || planes < 0) return kErrArgument;
  if (planes == 0) return kOk;
  const size_t smem = 2 * sizeof(cplx) * n + sizeof(int) * n;
  if (smem > static_cast<size_t>(current_device_attr(cudaDevAttrMaxSharedMemoryPerBlockOptin))) return kErrArgument;
  if (smem > 48 * 1024)
    MVMCB_CUDA(cudaFuncSetAttribute(k_pfinv_complex, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)));
  const int sms = current_device_attr(cudaDevAttrMultiProcessorCount);
  const int grid = std::max(1, std::min(planes, 8 * sms));
  k_pfinv_complex<<<grid, kCplxThreads, smem, stream>>>(reinterpret_cast<const cplx*>(x), n, planes,
                                                        reinterpret_cast<cplx*>(inv), reinterpret_cast<cplx*>(pf),
                                                        status);
  MVMCB_CUDA(cudaGetLastError());
  return kOk;
}

}  // namespace mvmcb

using namespace mvmcb;

extern "C" int mvmc_b200_pfinv_batch_complex_device(const double* x, int n, int planes, double* pf, double* inv,
                                                    int* status, void* stream) {
  if (planes > 0 && (!x || !pf || !inv || !status)) return kErrArgument;
  return pfinv_complex_device(x, n, planes, pf, inv, status, static_cast<cudaStream_t>(stream));
}
