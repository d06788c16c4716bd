// FP64 lower-triangle SYRK on the FP64 tensor-core path (mma.sync m8n8k4 f64).
//
// Two uses:
//  * plain-FP64 Pi(u):  C = sum_k A(:,k) alpha c_u(k) A(:,k)^T  with
//    c_u(k) = D(k)/(D(k)^2 + u^2) -- the FP64 form of rpa_THC_PiU_BlockAlgo
//    (src/rpa/rpa_THC.f90:313-339), lower triangle only (the reference's
//    full DGEMM computes both halves);
//  * the trailing update of the blocked Cholesky (C -= P P^T).
// A is column-major (rows contiguous), exactly the Cholesky-vector layout
// R(Q, ai) and the panel layout of a column-major lower Cholesky factor.
// CTA tile 64 x 64, 4 warps in 2 x 2, warp tile 32 x 32 (4 x 4 DMMA tiles),
// 16-deep K chunks streamed through a 3-stage cp.async pipeline.
#include "kernels.h"

namespace rpa {

namespace {
constexpr int BM = 64;
constexpr int BK = 16;
constexpr int LDS = BM + 8;  // 72 doubles: fragment loads hit each bank pair twice (optimal)
constexpr int kThreads = 128;

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// Tile b of the lower trapezoid of a T x T tile grid restricted to the first
// Tc tile columns, enumerated column by column: column tn holds rows tn..T-1.
__device__ __forceinline__ void trap_decode(int b, int T, int Tc, int& tm, int& tn) {
  // tiles before column c: c*T - c*(c-1)/2
  int lo = 0, hi = Tc - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (mid * T - mid * (mid - 1) / 2 <= b) lo = mid;
    else hi = mid - 1;
  }
  tn = lo;
  tm = tn + (b - (tn * T - tn * (tn - 1) / 2));
}

// One 64 x 64 tile (tm, tn) of C(lower trapezoid, ncols columns) for matrix z.
constexpr int kStages = 3;  // cp.async pipeline depth
constexpr size_t kTileSmem = sizeof(double) * (size_t)kStages * (2 * BK * LDS + BK);

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
               "l"(gmem), "r"(valid ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// One 64 x 64 tile (tm, tn) of C(lower trapezoid, ncols columns) for matrix z.
// Operands stream global -> shared through a kStages-deep cp.async pipeline
// (out-of-range elements zero-filled); one barrier per 16-deep K chunk.
template <bool kScaled>
__device__ __forceinline__ void dsyrk_tile(const DsyrkArgs& a, const double* A, double* C, int ncols, int tm, int tn,
                                           int z) {
  extern __shared__ double tile_smem[];
  auto As = reinterpret_cast<double(*)[BK][LDS]>(tile_smem);                        // [kStages]
  auto Bs = reinterpret_cast<double(*)[BK][LDS]>(tile_smem + kStages * BK * LDS);   // [kStages]
  auto sS = reinterpret_cast<double(*)[BK]>(tile_smem + 2 * kStages * BK * LDS);    // [kStages]

  const int m0 = tm * BM, n0 = tn * BM;
  const int t = threadIdx.x;
  const int lane = t & 31, warp = t >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const double u2 = kScaled ? a.u2[z] : 0.0;

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  auto load_stage = [&](int st, int64_t k0) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int idx = t + kThreads * i;
      const int col = idx / BM, row = idx % BM;
      const int64_t k = k0 + col;
      const bool kin = k < a.kdim;
      const bool va = kin && m0 + row < a.n, vb = kin && n0 + row < a.n;
      cp_async8(&As[st][col][row], va ? A + (int64_t)(m0 + row) + a.lda * k : A, va);
      cp_async8(&Bs[st][col][row], vb ? A + (int64_t)(n0 + row) + a.lda * k : A, vb);
    }
    if (kScaled && t < BK) {
      const int64_t k = k0 + t;
      double sc = 0.0;
      if (k < a.kdim) {
        const double d = a.D[k];
        sc = a.alpha * d / (d * d + u2);
      }
      sS[st][t] = sc;
    }
  };

  const int64_t nch = (a.kdim + BK - 1) / BK;
#pragma unroll
  for (int st = 0; st < kStages - 1; ++st) {
    if (st < nch) load_stage(st, (int64_t)st * BK);
    cp_async_commit();
  }
  for (int64_t c = 0; c < nch; ++c) {
    cp_async_wait<kStages - 2>();
    __syncthreads();
    const int64_t cn = c + kStages - 1;
    if (cn < nch) load_stage((int)(cn % kStages), cn * BK);
    cp_async_commit();
    const int buf = (int)(c % kStages);
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      const int kr = kk + (lane & 3);
      double af[4], bf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) af[i] = As[buf][kr][wm * 32 + i * 8 + (lane >> 2)];
      const double sc = kScaled ? sS[buf][kr] : 1.0;
#pragma unroll
      for (int j = 0; j < 4; ++j) bf[j] = Bs[buf][kr][wn * 32 + j * 8 + (lane >> 2)] * sc;
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
  }
  cp_async_wait<0>();

#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int row = m0 + wm * 32 + i * 8 + (lane >> 2);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int v = 0; v < 2; ++v) {
        const int col = n0 + wn * 32 + j * 8 + 2 * (lane & 3) + v;
        if (row < a.n && col < ncols && row >= col) {
          double* p = C + (int64_t)row + a.ldc * (int64_t)col;
          if (kScaled) *p = acc[i][j][v];
          else *p -= acc[i][j][v];
        }
      }
    }
  }
}

template <bool kScaled>
__global__ void __launch_bounds__(kThreads, 4) dsyrk_lower_kernel(const DsyrkArgs a, const int T, const int Tc) {
  int tm, tn;
  trap_decode(blockIdx.x, T, Tc, tm, tn);
  const int ncols = a.ncols > 0 ? a.ncols : a.n;
  const int z = blockIdx.y;
  dsyrk_tile<kScaled>(a, a.A + (int64_t)z * a.strideA, a.C + (int64_t)z * a.strideC, ncols, tm, tn, z);
}

// Variable-size batch: step of the two-level blocked Cholesky.
//   mode 0 (panel update): C = A[j0+64:, j0+64:], n = N - j0 - 64, ncols = min(N, J0+256) - (j0+64), K = 64
//   mode 1 (trailing):     C = A[J1:, J1:],       n = N - J1, J1 = min(N, J0+256), K = J1 - J0
__global__ void __launch_bounds__(kThreads, 4) dsyrk_varlen_kernel(const MatDesc* mats, int mode, int J0, int j0) {
  const MatDesc md = mats[blockIdx.y];
  const int N = md.n;
  const int J1 = min(N, J0 + 256);
  DsyrkArgs a{};
  int ncols;
  if (mode == 0) {
    a.n = N - j0 - BM;
    ncols = J1 - (j0 + BM);
    a.kdim = BM;
    a.A = md.A + (int64_t)(j0 + BM) + md.ld * (int64_t)j0;
    a.C = md.A + (int64_t)(j0 + BM) + md.ld * (int64_t)(j0 + BM);
  } else {
    a.n = N - J1;
    ncols = a.n;
    a.kdim = J1 - J0;
    a.A = md.A + (int64_t)J1 + md.ld * (int64_t)J0;
    a.C = md.A + (int64_t)J1 + md.ld * (int64_t)J1;
  }
  if (a.n <= 0 || ncols <= 0 || a.kdim <= 0) return;
  a.lda = md.ld;
  a.ldc = md.ld;
  const int T = (a.n + BM - 1) / BM;
  const int Tc = (min(ncols, a.n) + BM - 1) / BM;
  const int tiles = Tc * T - Tc * (Tc - 1) / 2;
  if ((int)blockIdx.x >= tiles) return;
  int tm, tn;
  trap_decode(blockIdx.x, T, Tc, tm, tn);
  dsyrk_tile<false>(a, a.A, a.C, min(ncols, a.n), tm, tn, 0);
}
}  // namespace

cudaError_t launch_dsyrk_varlen(const MatDesc* mats, int nmat, int mode, int J0, int j0, int max_tiles,
                                cudaStream_t stream) {
  if (nmat <= 0 || max_tiles <= 0) return cudaSuccess;
  cudaError_t e0 = cudaFuncSetAttribute(dsyrk_varlen_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmem);
  if (e0 != cudaSuccess) return e0;
  dsyrk_varlen_kernel<<<dim3((unsigned)max_tiles, (unsigned)nmat), kThreads, kTileSmem, stream>>>(mats, mode, J0, j0);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_dsyrk_lower(const DsyrkArgs& a, cudaStream_t stream) {
  if (a.n <= 0 || a.batch <= 0) return cudaSuccess;
  const int T = (a.n + BM - 1) / BM;
  const int nc = (a.ncols > 0 && a.ncols < a.n) ? a.ncols : a.n;
  const int Tc = (nc + BM - 1) / BM;
  const int64_t tiles = (int64_t)Tc * T - (int64_t)Tc * (Tc - 1) / 2;
  dim3 grid((unsigned)tiles, (unsigned)a.batch);
  cudaError_t e0 = a.D ? cudaFuncSetAttribute(dsyrk_lower_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)kTileSmem)
                       : cudaFuncSetAttribute(dsyrk_lower_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)kTileSmem);
  if (e0 != cudaSuccess) return e0;
  if (a.D) dsyrk_lower_kernel<true><<<grid, kThreads, kTileSmem, stream>>>(a, T, Tc);
  else dsyrk_lower_kernel<false><<<grid, kThreads, kTileSmem, stream>>>(a, T, Tc);
  ++g_launches;
  return cudaGetLastError();
}

}  // namespace rpa
