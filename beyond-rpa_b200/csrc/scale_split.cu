// Denominator scaling + bf16 hi/lo split of the Cholesky vectors.
//
// For a group of up to kMaxKgLaunch frequencies u_k this pass reads the FP64
// Cholesky vectors R(Q, ai) (column-major, as rpa_THC_ChiRkai reads them,
// src/rpa/rpa_THC.f90:343-371) once and writes, per frequency,
//   X_k(Q, ai) = sqrt(alpha * D(ai) / (D(ai)^2 + u_k^2)) * R(Q, ai)
// split as X = hi + lo (hi = bf16(X), lo = bf16(X - hi)), transposed to
// Q-rows with ai contiguous (the K-major operand layout of the tensor-core
// contraction).  It also accumulates the exact FP64 diagonal
//   Pi_k(Q,Q) = sum_ai X_k(Q,ai)^2
// per (ai-split, k, Q) for a deterministic second-stage reduction.
// The pass is HBM-bound: 8 B read + 4 B written per element and frequency.
#include "kernels.h"

namespace rpa {

namespace {
constexpr int kTQ = 32;        // Q rows per CTA
constexpr int kTA = 128;       // ai columns per chunk
constexpr int kThreads = 256;  // 8 warps; warp w owns the ai pairs w, w+8, ..., w+56
constexpr int kPairs = kTA / 2;
constexpr int kPairsPerThread = kPairs / 8;  // 8 pairs = 16 columns per thread
constexpr int kWordPitch = kPairs + 1;       // 65 words: conflict-free transposed staging

__device__ __forceinline__ uint32_t bf162_bits(__nv_bfloat162 v) {
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void scale_split_body(
    const double* __restrict__ R, int64_t ldR, int NQ, int64_t nov, const double* __restrict__ D,
    const FreqGroup& fg, double alpha, __nv_bfloat16* __restrict__ Xhi, __nv_bfloat16* __restrict__ Xlo,
    int64_t pitch, int64_t kstride, double* __restrict__ diag_part, int64_t ai_per_split, int qtile, int split) {
  extern __shared__ double dyn_smem[];
  auto sfac = reinterpret_cast<double(*)[kTA]>(dyn_smem);                          // [kMaxKgLaunch][kTA]
  auto sdiag = reinterpret_cast<double(*)[kMaxKgLaunch][kTQ]>(dyn_smem + kMaxKgLaunch * kTA);  // [8][k][q]
  auto ohi = reinterpret_cast<uint32_t(*)[kWordPitch]>(dyn_smem + kMaxKgLaunch * kTA + 8 * kMaxKgLaunch * kTQ);
  auto olo = ohi + kTQ;  // per-warp partial diagonal sums above need no atomics

  const int t = threadIdx.x;
  const int qi = t & 31;
  const int wa = t >> 5;
  const int q0 = qtile * kTQ;
  const int q = q0 + qi;
  const int kg = fg.n;
  const int64_t a_begin = (int64_t)split * ai_per_split;
  const int64_t a_end = min(nov, a_begin + ai_per_split);

  for (int k = 0; k < kMaxKgLaunch; ++k) sdiag[wa][k][qi] = 0.0;

  for (int64_t a0 = a_begin; a0 < a_end; a0 += kTA) {
    // scaling factors sqrt(alpha D/(D^2+u^2)) of this chunk, FP64
    for (int idx = t; idx < kg * kTA; idx += kThreads) {
      const int k = idx / kTA, aj = idx % kTA;
      const int64_t a = a0 + aj;
      double f = 0.0;
      if (a < a_end) {
        const double d = D[a];
        f = sqrt(alpha * d / (d * d + fg.u2[k]));
      }
      sfac[k][aj] = f;
    }
    // R(q, a): a warp reads 32 consecutive Q of one column (coalesced)
    double r[2 * kPairsPerThread];
#pragma unroll
    for (int p = 0; p < kPairsPerThread; ++p)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int64_t a = a0 + 2 * (wa + 8 * p) + e;
        r[2 * p + e] = (q < NQ && a < a_end) ? __ldg(R + (int64_t)q + ldR * a) : 0.0;
      }
    __syncthreads();
#pragma unroll 1
    for (int k = 0; k < kg; ++k) {
      double s = 0.0;
#pragma unroll
      for (int p = 0; p < kPairsPerThread; ++p) {
        const int pw = wa + 8 * p;
        const double x0 = r[2 * p] * sfac[k][2 * pw];
        const double x1 = r[2 * p + 1] * sfac[k][2 * pw + 1];
        s = fma(x0, x0, s);
        s = fma(x1, x1, s);
        // hi = bf16(x), lo = bf16(x - hi); x - hi is exact in FP32
        const float f0 = (float)x0, f1 = (float)x1;
        const __nv_bfloat162 h2 = __floats2bfloat162_rn(f0, f1);
        const float2 hf = __bfloat1622float2(h2);
        const __nv_bfloat162 l2 = __floats2bfloat162_rn(f0 - hf.x, f1 - hf.y);
        ohi[qi][pw] = bf162_bits(h2);
        olo[qi][pw] = bf162_bits(l2);
      }
      sdiag[wa][k][qi] += s;  // owned by this thread alone
      __syncthreads();
      // a warp stores 32 words (64 columns) of one row per instruction (128 B)
      for (int idx = t; idx < kTQ * kPairs; idx += kThreads) {
        const int row = idx / kPairs, w = idx % kPairs;
        const int64_t a = a0 + 2 * w;
        if (q0 + row < NQ && a < nov) {
          const int64_t off = (int64_t)k * kstride + (int64_t)(q0 + row) * pitch + a;
          *reinterpret_cast<uint32_t*>(Xhi + off) = ohi[row][w];
          *reinterpret_cast<uint32_t*>(Xlo + off) = olo[row][w];
        }
      }
      __syncthreads();
    }
  }
  // deterministic reduction of the 8 column owners of each row
  __syncthreads();
  for (int idx = t; idx < kg * kTQ; idx += kThreads) {
    const int k = idx / kTQ, row = idx % kTQ;
    if (q0 + row < NQ) {
      double acc = 0.0;
#pragma unroll
      for (int w = 0; w < 8; ++w) acc += sdiag[w][k][row];
      diag_part[((int64_t)split * kg + k) * NQ + q0 + row] = acc;
    }
  }
}

__global__ void __launch_bounds__(kThreads, 3) scale_split_kernel(
    const double* __restrict__ R, int64_t ldR, int NQ, int64_t nov, const double* __restrict__ D,
    FreqGroup fg, double alpha, __nv_bfloat16* __restrict__ Xhi, __nv_bfloat16* __restrict__ Xlo, int64_t pitch,
    int64_t kstride, double* __restrict__ diag_part, int64_t ai_per_split, int split0) {
  scale_split_body(R, ldR, NQ, nov, D, fg, alpha, Xhi, Xlo, pitch, kstride, diag_part, ai_per_split, blockIdx.x,
                   split0 + (int)blockIdx.y);
}

// Many instances in one launch: CTA b handles (instance, q tile, ai split) = work[b].
__global__ void __launch_bounds__(kThreads, 3) scale_split_multi_kernel(const SplitJob* __restrict__ jobs,
                                                                        const int4* __restrict__ work) {
  const int4 w = work[blockIdx.x];
  const SplitJob& j = jobs[w.x];
  scale_split_body(j.R, j.ldR, j.NQ, j.nov, j.D, j.fg, j.alpha, j.Xhi, j.Xlo, j.pitch, j.kstride, j.diag_part,
                   j.ai_per_split, w.y, w.z);
}

// diag[k*NQ+q] = sum over splits, for every instance (one thread per (instance, k, q))
__global__ void diag_reduce_multi_kernel(const SplitJob* __restrict__ jobs, const int64_t* __restrict__ offsets,
                                         int njobs, int64_t total) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (offsets[mid] <= idx) lo = mid;
    else hi = mid - 1;
  }
  const SplitJob& j = jobs[lo];
  const int64_t e = idx - offsets[lo];
  const int64_t per = (int64_t)j.fg.n * j.NQ;
  double s = 0.0;
  for (int sp = 0; sp < j.nsplit; ++sp) s += j.diag_part[(int64_t)sp * per + e];
  j.diag[e] = s;
}

__global__ void diag_reduce_kernel(const double* __restrict__ diag_part, int nsplit, int kg, int NQ,
                                   double* __restrict__ diag) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)kg * NQ) return;
  double s = 0.0;
  for (int sp = 0; sp < nsplit; ++sp) s += diag_part[(int64_t)sp * kg * NQ + idx];
  diag[idx] = s;
}
}  // namespace

SplitPlan plan_scale_split(int NQ, int64_t nov, int num_sms) {
  // Enough CTAs for ~16 waves of 2 resident CTAs per SM, so that the last
  // partial wave costs little.
  SplitPlan p;
  p.qtiles = (NQ + kTQ - 1) / kTQ;
  const int64_t chunks = (nov + kTA - 1) / kTA;
  int64_t want = (32 * (int64_t)num_sms + p.qtiles - 1) / p.qtiles;
  if (want < 1) want = 1;
  if (want > chunks) want = chunks;
  const int64_t chunks_per = (chunks + want - 1) / want;
  p.ai_per_split = chunks_per * kTA;
  p.nsplit = (int)((nov + p.ai_per_split - 1) / p.ai_per_split);
  if (p.nsplit < 1) p.nsplit = 1;
  return p;
}

constexpr size_t kSplitSmem =
    sizeof(double) * (kMaxKgLaunch * kTA + 8 * kMaxKgLaunch * kTQ) + sizeof(uint32_t) * 2 * kTQ * kWordPitch;

cudaError_t launch_scale_split_multi(const SplitJob* jobs, const int4* work, int nwork, const int64_t* offsets,
                                     int njobs, int64_t total, cudaStream_t stream) {
  cudaError_t e0 =
      cudaFuncSetAttribute(scale_split_multi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSplitSmem);
  if (e0 != cudaSuccess) return e0;
  if (nwork > 0) {
    scale_split_multi_kernel<<<nwork, kThreads, kSplitSmem, stream>>>(jobs, work);
    ++g_launches;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || total == 0) return e;
  diag_reduce_multi_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(jobs, offsets, njobs, total);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_scale_split(const double* R, int64_t ldR, int NQ, int64_t nov, const double* D,
                               const FreqGroup& fg, double alpha, __nv_bfloat16* Xhi, __nv_bfloat16* Xlo,
                               int64_t pitch, int64_t kstride, double* diag_part, double* diag,
                               const SplitPlan& plan, cudaStream_t stream) {
  dim3 grid(plan.qtiles, plan.nsplit);
  cudaError_t e0 = cudaFuncSetAttribute(scale_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSplitSmem);
  if (e0 != cudaSuccess) return e0;
  scale_split_kernel<<<grid, kThreads, kSplitSmem, stream>>>(R, ldR, NQ, nov, D, fg, alpha, Xhi, Xlo, pitch, kstride,
                                                     diag_part, plan.ai_per_split, 0);
  ++g_launches;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_diag_reduce(diag_part, plan, fg.n, NQ, diag, stream);
}

cudaError_t launch_scale_split_part(const double* R, int64_t ldR, int NQ, int64_t nov, const double* D,
                                    const FreqGroup& fg, double alpha, __nv_bfloat16* Xhi, __nv_bfloat16* Xlo,
                                    int64_t pitch, int64_t kstride, double* diag_part, const SplitPlan& plan,
                                    int split0, int split1, cudaStream_t stream) {
  if (split0 < 0 || split1 > plan.nsplit || split1 <= split0) return cudaErrorInvalidValue;
  cudaError_t e0 = cudaFuncSetAttribute(scale_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSplitSmem);
  if (e0 != cudaSuccess) return e0;
  dim3 grid(plan.qtiles, split1 - split0);
  scale_split_kernel<<<grid, kThreads, kSplitSmem, stream>>>(R, ldR, NQ, nov, D, fg, alpha, Xhi, Xlo, pitch, kstride,
                                                     diag_part, plan.ai_per_split, split0);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_diag_reduce(const double* diag_part, const SplitPlan& plan, int kg, int NQ, double* diag,
                               cudaStream_t stream) {
  const int64_t n = (int64_t)kg * NQ;
  diag_reduce_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(diag_part, plan.nsplit, kg, NQ, diag);
  ++g_launches;
  return cudaGetLastError();
}

}  // namespace rpa
