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
constexpr int kThreads = 256;  // 8 warps; warp w owns columns w, w+8, ...
constexpr int kPerThread = kTA / 8;  // 16 columns per thread
constexpr int kOutPitch = kTA + 8;   // bf16 elements per staged row (272 B)

__global__ void __launch_bounds__(kThreads) scale_split_kernel(
    const double* __restrict__ R, int64_t ldR, int NQ, int64_t nov, const double* __restrict__ D,
    FreqGroup fg, double alpha, __nv_bfloat16* __restrict__ Xhi, __nv_bfloat16* __restrict__ Xlo, int64_t pitch,
    int64_t kstride, double* __restrict__ diag_part, int64_t ai_per_split) {
  __shared__ double sfac[kMaxKgLaunch][kTA];
  __shared__ __align__(16) __nv_bfloat16 ohi[kTQ][kOutPitch];
  __shared__ __align__(16) __nv_bfloat16 olo[kTQ][kOutPitch];
  __shared__ double red[8][kTQ];

  const int t = threadIdx.x;
  const int qi = t & 31;
  const int wa = t >> 5;
  const int q0 = blockIdx.x * kTQ;
  const int q = q0 + qi;
  const int kg = fg.n;
  const int64_t a_begin = (int64_t)blockIdx.y * ai_per_split;
  const int64_t a_end = min(nov, a_begin + ai_per_split);

  double dsum[kMaxKgLaunch];
#pragma unroll
  for (int k = 0; k < kMaxKgLaunch; ++k) dsum[k] = 0.0;

  for (int64_t a0 = a_begin; a0 < a_end; a0 += kTA) {
    // scaling factors of this chunk, FP64
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
    double r[kPerThread];
#pragma unroll
    for (int i = 0; i < kPerThread; ++i) {
      const int64_t a = a0 + wa + 8 * i;
      r[i] = (q < NQ && a < a_end) ? __ldg(R + (int64_t)q + ldR * a) : 0.0;
    }
    __syncthreads();
#pragma unroll 1
    for (int k = 0; k < kg; ++k) {
      double s = 0.0;
#pragma unroll
      for (int i = 0; i < kPerThread; ++i) {
        const int aj = wa + 8 * i;
        const double x = r[i] * sfac[k][aj];
        const __nv_bfloat16 h = __double2bfloat16(x);
        const __nv_bfloat16 l = __double2bfloat16(x - (double)__bfloat162float(h));
        s = fma(x, x, s);
        ohi[qi][aj] = h;
        olo[qi][aj] = l;
      }
      // register-resident accumulator selected by a uniform branch
#pragma unroll
      for (int kk = 0; kk < kMaxKgLaunch; ++kk)
        if (kk == k) dsum[kk] += s;
      __syncthreads();
      // rows of 16-byte vectors: 32 rows x 16 vectors per array
      for (int v = t; v < kTQ * (kTA / 8); v += kThreads) {
        const int row = v / (kTA / 8);
        const int col = (v % (kTA / 8)) * 8;
        const int64_t a = a0 + col;
        if (q0 + row < NQ && a < nov) {
          const int64_t off = (int64_t)k * kstride + (int64_t)(q0 + row) * pitch + a;
          *reinterpret_cast<uint4*>(Xhi + off) = *reinterpret_cast<const uint4*>(&ohi[row][col]);
          *reinterpret_cast<uint4*>(Xlo + off) = *reinterpret_cast<const uint4*>(&olo[row][col]);
        }
      }
      __syncthreads();
    }
  }
  // deterministic reduction of the 8 column owners of each row
  for (int k = 0; k < kg; ++k) {
    double v = 0.0;
#pragma unroll
    for (int kk = 0; kk < kMaxKgLaunch; ++kk)
      if (kk == k) v = dsum[kk];
    red[wa][qi] = v;
    __syncthreads();
    if (wa == 0 && q < NQ) {
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < 8; ++w) s += red[w][qi];
      diag_part[((int64_t)blockIdx.y * kg + k) * NQ + q] = s;
    }
    __syncthreads();
  }
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
  SplitPlan p;
  p.qtiles = (NQ + kTQ - 1) / kTQ;
  const int64_t chunks = (nov + kTA - 1) / kTA;
  int64_t want = (4 * (int64_t)num_sms + p.qtiles - 1) / p.qtiles;
  if (want < 1) want = 1;
  if (want > chunks) want = chunks;
  const int64_t chunks_per = (chunks + want - 1) / want;
  p.ai_per_split = chunks_per * kTA;
  p.nsplit = (int)((nov + p.ai_per_split - 1) / p.ai_per_split);
  if (p.nsplit < 1) p.nsplit = 1;
  return p;
}

cudaError_t launch_scale_split(const double* R, int64_t ldR, int NQ, int64_t nov, const double* D,
                               const FreqGroup& fg, double alpha, __nv_bfloat16* Xhi, __nv_bfloat16* Xlo,
                               int64_t pitch, int64_t kstride, double* diag_part, double* diag,
                               const SplitPlan& plan, cudaStream_t stream) {
  dim3 grid(plan.qtiles, plan.nsplit);
  scale_split_kernel<<<grid, kThreads, 0, stream>>>(R, ldR, NQ, nov, D, fg, alpha, Xhi, Xlo, pitch, kstride,
                                                     diag_part, plan.ai_per_split);
  ++g_launches;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int64_t n = (int64_t)fg.n * NQ;
  diag_reduce_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(diag_part, plan.nsplit, fg.n, NQ, diag);
  ++g_launches;
  return cudaGetLastError();
}

}  // namespace rpa
