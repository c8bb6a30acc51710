// Batched Pfaffian + inverse of complex skew-symmetric planes: the computational core of
// the complex mode's CalculateMAll (calc_m_all_complex, crates/mvmc-core/src/pfaffian.rs:
// 340-360, which runs pfapack's complex LTLᵀ per QP plane).
//
// Same skew Gauss–Jordan sweep with 2×2 pivots as the real kernels (pfinv.cuh), in complex
// FP64: p = smallest unswept index, q = the first maximum of |A[p][j]|² over unswept j ≠ p,
// A[i][j] += (A[q][i]·A[p][j] − A[p][i]·A[q][j]) / a with a = A[p][q], Pf = sgn(σ)·Πa.
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
            const double v = rowp[j].re * rowp[j].re + rowp[j].im * rowp[j].im;
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
          const cplx rpi = rowp[i], rqi = rowq[i];
          for (int j = lane; j < n; j += 32) {
            cplx v;
            if (j == p) v = cneg(cmul(rqi, ia));
            else if (j == q) v = cmul(rpi, ia);
            else v = cadd(Ai[j], cmul(csub(cmul(rqi, rowp[j]), cmul(rpi, rowq[j])), ia));
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

struct Buf {
  void* p = nullptr;
  ~Buf() {
    if (p) cudaFree(p);
  }
};

}  // namespace

}  // namespace mvmcb

using namespace mvmcb;

extern "C" int mvmc_b200_pfinv_batch_complex(const double* x, int n, int planes, double* pf, double* inv,
                                             int* status) {
  if (n <= 0 || (n & 1) || planes < 0) return kErrArgument;
  if (planes == 0) return kOk;
  if (!x || !pf || !inv || !status) return kErrArgument;
  const size_t elems = static_cast<size_t>(n) * n * planes;
  Buf dx, dinv, dpf, dst;
  MVMCB_CUDA(cudaMalloc(&dx.p, elems * sizeof(cplx)));
  MVMCB_CUDA(cudaMalloc(&dinv.p, elems * sizeof(cplx)));
  MVMCB_CUDA(cudaMalloc(&dpf.p, planes * sizeof(cplx)));
  MVMCB_CUDA(cudaMalloc(&dst.p, planes * sizeof(int)));
  MVMCB_CUDA(cudaMemcpy(dx.p, x, elems * sizeof(cplx), cudaMemcpyHostToDevice));
  const size_t smem = 2 * sizeof(cplx) * n + sizeof(int) * n;
  if (smem > 48 * 1024) MVMCB_CUDA(cudaFuncSetAttribute(k_pfinv_complex, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                        static_cast<int>(smem)));
  int dev = 0, sms = 0;
  MVMCB_CUDA(cudaGetDevice(&dev));
  MVMCB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int grid = std::max(1, std::min(planes, 8 * sms));
  k_pfinv_complex<<<grid, kCplxThreads, smem>>>(static_cast<const cplx*>(dx.p), n, planes,
                                                static_cast<cplx*>(dinv.p), static_cast<cplx*>(dpf.p),
                                                static_cast<int*>(dst.p));
  MVMCB_CUDA(cudaGetLastError());
  MVMCB_CUDA(cudaMemcpy(inv, dinv.p, elems * sizeof(cplx), cudaMemcpyDeviceToHost));
  MVMCB_CUDA(cudaMemcpy(pf, dpf.p, planes * sizeof(cplx), cudaMemcpyDeviceToHost));
  MVMCB_CUDA(cudaMemcpy(status, dst.p, planes * sizeof(int), cudaMemcpyDeviceToHost));
  return kOk;
}
