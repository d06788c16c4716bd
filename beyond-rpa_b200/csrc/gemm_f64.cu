// Generic batched FP64 GEMM on the FP64 tensor-core path (mma.sync m8n8k4 f64),
// used by the direct-ring T2 and exchange chains (the DGEMM calls of
// rpa_CC_IM_v5 / rpa_CC_MIM_v5 / rpa_CC_T2_v5, src/rpa/rpa_CC_Doubles.f90:369-642).
//
//   C_b(m, n) = alpha * rs(m) * sum_k A_b(m, k) ks(k) B_b(k, n) + beta * C_b(m, n)
//
// A_b(m, k) = A[b*sA + m*a_m + k*a_k], B_b(k, n) = B[b*sB + k*b_k + n*b_n],
// C column-major (ld), optional per-k scale ks (ks_stride per batch) and
// per-row scale rs.  Either stride of each operand may be 1; the loader maps
// consecutive threads along the unit-stride index.
// CTA tile 64 x 64, 4 warps (2 x 2) of 32 x 32, K chunks of 16 double-buffered
// through shared memory.
#include "kernels.h"

namespace rpa {

namespace {
constexpr int BM = 64;
constexpr int BK = 16;
constexpr int LDS = BM + 8;
constexpr int kThreads = 128;

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(kThreads) gemm_f64_kernel(const GemmF64Args g) {
  __shared__ double As[2][BK][LDS];
  __shared__ double Bs[2][BK][LDS];
  const int b = blockIdx.z;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BM;
  const double* A = g.A + (int64_t)b * g.sA;
  const double* B = g.B + (int64_t)b * g.sB;
  double* C = g.C + (int64_t)b * g.sC;
  const double* ks = g.kscale ? g.kscale + (int64_t)b * g.ks_stride : nullptr;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const bool a_mcontig = (g.a_m == 1);
  const bool b_ncontig = (g.b_n == 1);

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  double ra[8], rb[8];
  auto idx_of = [&](int i, bool contig_first, int& r, int& c) {
    // 1024 elements of a 64 x 16 tile: r in [0,64) (m or n), c in [0,16) (k)
    const int idx = t + kThreads * i;
    if (contig_first) {
      r = idx % BM;
      c = idx / BM;
    } else {
      r = idx / BK;
      c = idx % BK;
    }
  };
  auto gload = [&](int64_t k0) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      int r, c;
      idx_of(i, a_mcontig, r, c);
      const int64_t k = k0 + c;
      const int m = m0 + r;
      ra[i] = (m < g.M && k < g.K) ? A[(int64_t)m * g.a_m + k * g.a_k] : 0.0;
      idx_of(i, b_ncontig, r, c);
      const int64_t k2 = k0 + c;
      const int n = n0 + r;
      double v = (n < g.N && k2 < g.K) ? B[k2 * g.b_k + (int64_t)n * g.b_n] : 0.0;
      if (ks && k2 < g.K) v *= ks[k2];
      rb[i] = v;
    }
  };
  auto sstore = [&](int buf) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      int r, c;
      idx_of(i, a_mcontig, r, c);
      As[buf][c][r] = ra[i];
      idx_of(i, b_ncontig, r, c);
      Bs[buf][c][r] = rb[i];
    }
  };

  const int64_t nch = (g.K + BK - 1) / BK;
  gload(0);
  sstore(0);
  __syncthreads();
  for (int64_t c = 0; c < nch; ++c) {
    const int buf = (int)(c & 1);
    if (c + 1 < nch) gload((c + 1) * BK);
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      const int kr = kk + (lane & 3);
      double af[4], bf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) af[i] = As[buf][kr][wm * 32 + i * 8 + (lane >> 2)];
#pragma unroll
      for (int j = 0; j < 4; ++j) bf[j] = Bs[buf][kr][wn * 32 + j * 8 + (lane >> 2)];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
    if (c + 1 < nch) sstore(buf ^ 1);
    __syncthreads();
  }

#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + wm * 32 + i * 8 + (lane >> 2);
    if (m >= g.M) continue;
    const double rsm = g.rowscale ? g.rowscale[m] : 1.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int v = 0; v < 2; ++v) {
        const int n = n0 + wn * 32 + j * 8 + 2 * (lane & 3) + v;
        if (n >= g.N) continue;
        double* p = C + (int64_t)m + g.ldc * (int64_t)n;
        const double val = g.alpha * rsm * acc[i][j][v];
        *p = (g.beta == 0.0) ? val : val + g.beta * *p;
      }
    }
  }
}
}  // namespace

cudaError_t launch_gemm_f64(const GemmF64Args& g, cudaStream_t stream) {
  if (g.M <= 0 || g.N <= 0 || g.batch <= 0) return cudaSuccess;
  dim3 grid((unsigned)((g.N + BM - 1) / BM), (unsigned)((g.M + BM - 1) / BM), (unsigned)g.batch);
  gemm_f64_kernel<<<grid, kThreads, 0, stream>>>(g);
  ++g_launches;
  return cudaGetLastError();
}

}  // namespace rpa
