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
// Two CTA tiles (the tile tuner picks one per matrix-size bucket):
//   kW = 2: 64 x 64, 4 warps (2 x 2), 4 CTAs per SM;
//   kW = 4: 128 x 128, 16 warps (4 x 4), 1 CTA per SM (half the operand
//           traffic per flop, coarser tiles on the triangle's diagonal).
// Warp tile 32 x 32 (4 x 4 DMMA tiles) in both; 16-deep K chunks streamed
// through a 3-stage cp.async pipeline.
#include <algorithm>

#include "kernels.h"

namespace rpa {

namespace {
constexpr int BK = 16;
// Tile geometry of the kW x kW-warp CTA.  Row pitch BM + 8 doubles (72 or 136): the m8n8k4
// fragment loads hit each bank pair twice (optimal) in both.
template <int kW>
struct Geo {
  static constexpr int BM = 32 * kW;
  static constexpr int LDS = BM + 8;
  static constexpr int kThreads = 32 * kW * kW;
  static constexpr int kMinBlocks = kW == 2 ? 4 : 1;
};

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

constexpr int kStages = 3;  // cp.async pipeline depth
template <int kW>
constexpr size_t tile_smem() {
  return sizeof(double) * (size_t)kStages * (2 * BK * Geo<kW>::LDS + BK);
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
               "l"(gmem), "r"(valid ? 8 : 0)
               : "memory");
}
// 16 bytes (two consecutive rows of one column), the first `bytes` of them copied (16, 8 or 0),
// the rest zero-filled.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
               "l"(gmem), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// One BM x BM tile (tm, tn) of C(lower trapezoid, ncols columns) for matrix z.
// Operands stream global -> shared through a kStages-deep cp.async pipeline
// (out-of-range elements zero-filled); one barrier per 16-deep K chunk.
// kCopy: 8 (8-byte copies), 16 (16-byte copies; the caller checked the alignment) or 0 (decide
// per operand from its alignment).
template <bool kScaled, int kW, int kCopy>
__device__ __forceinline__ void dsyrk_tile(const DsyrkArgs& a, const double* A, double* C, int ncols, int tm, int tn,
                                           int z) {
  constexpr int BM = Geo<kW>::BM, LDS = Geo<kW>::LDS, kThreads = Geo<kW>::kThreads;
  constexpr int kLoads = BK * BM / kThreads;  // elements of each operand per thread and stage
  extern __shared__ double dyn_smem[];
  auto As = reinterpret_cast<double(*)[BK][LDS]>(dyn_smem);                        // [kStages]
  auto Bs = reinterpret_cast<double(*)[BK][LDS]>(dyn_smem + kStages * BK * LDS);   // [kStages]
  auto sS = reinterpret_cast<double(*)[BK]>(dyn_smem + 2 * kStages * BK * LDS);    // [kStages]

  const int m0 = tm * BM, n0 = tn * BM;
  const int t = threadIdx.x;
  const int lane = t & 31, warp = t >> 5;
  const int wm = warp / kW, wn = warp % kW;
  const double u2 = kScaled ? a.u2[z] : 0.0;

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  // 16-byte copies of row pairs when every column of the operand starts 16-byte aligned (aligned
  // base, even leading dimension; m0, n0 and the pair index are even): half the copy
  // instructions, 12-16 % faster than 8-byte copies on B200
  const bool vec = kCopy == 16 || (kCopy == 0 && ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && ((a.lda & 1) == 0));
  auto load_stage = [&](int st, int64_t k0) {
    if (vec) {
#pragma unroll
      for (int i = 0; i < kLoads / 2; ++i) {
        const int idx = t + kThreads * i;
        const int col = idx / (BM / 2), row = 2 * (idx % (BM / 2));
        const int64_t k = k0 + col;
        const bool kin = k < a.kdim;
        const int ba = kin ? 8 * max(0, min(2, a.n - (m0 + row))) : 0;
        const int bb = kin ? 8 * max(0, min(2, a.n - (n0 + row))) : 0;
        cp_async16(&As[st][col][row], ba ? A + (int64_t)(m0 + row) + a.lda * k : A, ba);
        cp_async16(&Bs[st][col][row], bb ? A + (int64_t)(n0 + row) + a.lda * k : A, bb);
      }
    } else {
#pragma unroll
      for (int i = 0; i < kLoads; ++i) {
        const int idx = t + kThreads * i;
        const int col = idx / BM, row = idx % BM;
        const int64_t k = k0 + col;
        const bool kin = k < a.kdim;
        const bool va = kin && m0 + row < a.n, vb = kin && n0 + row < a.n;
        cp_async8(&As[st][col][row], va ? A + (int64_t)(m0 + row) + a.lda * k : A, va);
        cp_async8(&Bs[st][col][row], vb ? A + (int64_t)(n0 + row) + a.lda * k : A, vb);
      }
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

  // Subtract mode reads the C fragment of two row groups at a time before storing any of it:
  // a load-subtract-store per element would wait out one memory round trip per element, since
  // the compiler cannot move a load of C above a store to C.
#pragma unroll
  for (int i0 = 0; i0 < 4; i0 += 2) {
    double cv[2][4][2];
    if (!kScaled) {
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int row = m0 + wm * 32 + (i0 + i) * 8 + (lane >> 2);
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int v = 0; v < 2; ++v) {
            const int col = n0 + wn * 32 + j * 8 + 2 * (lane & 3) + v;
            cv[i][j][v] =
                (row < a.n && col < ncols && row >= col) ? C[(int64_t)row + a.ldc * (int64_t)col] : 0.0;
          }
      }
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int row = m0 + wm * 32 + (i0 + i) * 8 + (lane >> 2);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
#pragma unroll
        for (int v = 0; v < 2; ++v) {
          const int col = n0 + wn * 32 + j * 8 + 2 * (lane & 3) + v;
          if (row < a.n && col < ncols && row >= col) {
            double* p = C + (int64_t)row + a.ldc * (int64_t)col;
            if (kScaled) *p = acc[i0 + i][j][v];
            else *p = cv[i][j][v] - acc[i0 + i][j][v];
          }
        }
      }
    }
  }
}

template <bool kScaled, int kW, int kCopy>
__global__ void __launch_bounds__(Geo<kW>::kThreads, Geo<kW>::kMinBlocks)
    dsyrk_lower_kernel(const DsyrkArgs a, const int T, const int Tc) {
  int tm, tn;
  trap_decode(blockIdx.x, T, Tc, tm, tn);
  const int ncols = a.ncols > 0 ? a.ncols : a.n;
  const int z = blockIdx.y;
  dsyrk_tile<kScaled, kW, kCopy>(a, a.A + (int64_t)z * a.strideA, a.C + (int64_t)z * a.strideC, ncols, tm, tn, z);
}

// Shape of one step of the two-level blocked Cholesky for a matrix of order N
// (outer block nb2, inner block kCholNB; J1 = min(N, J0+nb2), J2 = min(N, J1+nb2)):
//   mode 0 (panel update):  C = A[j0+NB:, j0+NB:], n = N - j0 - NB, ncols = J1 - (j0+NB), K = NB
//   mode 1 (trailing):      C = A[J1:, J1:],       n = N - J1, ncols = n,       K = J1 - J0
//   mode 2 (next block):    C = A[J1:, J1:J2],     n = N - J1, ncols = J2 - J1, K = J1 - J0
//   mode 3 (rest):          C = A[J2:, J2:],       n = N - J2, ncols = n,       K = J1 - J0
// with the panel A[row0:, J0:J1] (row0 = the first row of C) as the SYRK operand.
__host__ __device__ __forceinline__ void varlen_step(int N, int mode, int J0, int j0, int nb2, int& n, int& ncols,
                                                     int& kdim, int& arow, int& acol) {
  const int J1 = N < J0 + nb2 ? N : J0 + nb2;
  const int J2 = N < J1 + nb2 ? N : J1 + nb2;
  if (mode == 0) {
    n = N - j0 - kCholNB;
    ncols = J1 - (j0 + kCholNB);
    kdim = kCholNB;
    arow = j0 + kCholNB;
    acol = j0;
  } else if (mode == 3) {
    n = N - J2;
    ncols = n;
    kdim = J1 - J0;
    arow = J2;
    acol = J0;
  } else {
    n = N - J1;
    ncols = mode == 2 ? J2 - J1 : n;
    kdim = J1 - J0;
    arow = J1;
    acol = J0;
  }
  if (ncols > n) ncols = n;
}

template <int kW>
__global__ void __launch_bounds__(Geo<kW>::kThreads, Geo<kW>::kMinBlocks)
    dsyrk_varlen_kernel(const MatDesc* mats, int mode, int J0, int j0, int nb2) {
  constexpr int BM = Geo<kW>::BM;
  const MatDesc md = mats[blockIdx.y];
  int n, ncols, kdim, arow, acol;
  varlen_step(md.n, mode, J0, j0, nb2, n, ncols, kdim, arow, acol);
  if (n <= 0 || ncols <= 0 || kdim <= 0) return;
  const int T = (n + BM - 1) / BM;
  const int Tc = (ncols + BM - 1) / BM;
  const int tiles = Tc * T - Tc * (Tc - 1) / 2;
  if ((int)blockIdx.x >= tiles) return;
  DsyrkArgs a{};
  a.n = n;
  a.kdim = kdim;
  a.A = md.A + (int64_t)arow + md.ld * (int64_t)acol;
  a.C = md.A + (int64_t)arow + md.ld * (int64_t)arow;
  a.lda = md.ld;
  a.ldc = md.ld;
  int tm, tn;
  trap_decode(blockIdx.x, T, Tc, tm, tn);
  dsyrk_tile<false, kW, 0>(a, a.A, a.C, ncols, tm, tn, 0);
}

int trap_tiles(int n, int ncols, int bm) {
  if (n <= 0 || ncols <= 0) return 0;
  const int T = (n + bm - 1) / bm, Tc = (std::min(ncols, n) + bm - 1) / bm;
  return Tc * T - Tc * (Tc - 1) / 2;
}

template <int kW>
cudaError_t launch_varlen_w(const MatDesc* mats, int nmat, int mode, int J0, int j0, int nb2, int nmax,
                            cudaStream_t stream) {
  int n, ncols, kdim, arow, acol;
  varlen_step(nmax, mode, J0, j0, nb2, n, ncols, kdim, arow, acol);  // the largest order has the most tiles
  const int tiles = trap_tiles(n, ncols, Geo<kW>::BM);
  if (tiles <= 0 || kdim <= 0) return cudaSuccess;
  constexpr size_t smem = tile_smem<kW>();
  cudaError_t e0 = cudaFuncSetAttribute(dsyrk_varlen_kernel<kW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem);
  if (e0 != cudaSuccess) return e0;
  dsyrk_varlen_kernel<kW><<<dim3((unsigned)tiles, (unsigned)nmat), Geo<kW>::kThreads, smem, stream>>>(mats, mode, J0,
                                                                                                     j0, nb2);
  ++g_launches;
  return cudaGetLastError();
}

template <bool kScaled, int kW, int kCopy>
cudaError_t launch_lower_wc(const DsyrkArgs& a, cudaStream_t stream) {
  constexpr int BM = Geo<kW>::BM;
  const int T = (a.n + BM - 1) / BM;
  const int nc = (a.ncols > 0 && a.ncols < a.n) ? a.ncols : a.n;
  const int Tc = (nc + BM - 1) / BM;
  const int64_t tiles = (int64_t)Tc * T - (int64_t)Tc * (Tc - 1) / 2;
  constexpr size_t smem = tile_smem<kW>();
  cudaError_t e0 = cudaFuncSetAttribute(dsyrk_lower_kernel<kScaled, kW, kCopy>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e0 != cudaSuccess) return e0;
  dsyrk_lower_kernel<kScaled, kW, kCopy><<<dim3((unsigned)tiles, (unsigned)a.batch), Geo<kW>::kThreads, smem,
                                          stream>>>(a, T, Tc);
  ++g_launches;
  return cudaGetLastError();
}

// 16-byte copies when every column of every matrix of the batch starts 16-byte aligned.
template <bool kScaled, int kW>
cudaError_t launch_lower_w(const DsyrkArgs& a, cudaStream_t stream) {
  const bool vec = ((reinterpret_cast<uintptr_t>(a.A) & 15) == 0) && ((a.lda & 1) == 0) && ((a.strideA & 1) == 0);
  return vec ? launch_lower_wc<kScaled, kW, 16>(a, stream) : launch_lower_wc<kScaled, kW, 8>(a, stream);
}
}  // namespace

// One step of the variable-size blocked Cholesky over nmat matrices of orders <= nmax.
cudaError_t launch_dsyrk_varlen(const MatDesc* mats, int nmat, int mode, int J0, int j0, int nb2, int tile_w,
                                int nmax, cudaStream_t stream) {
  if (nmat <= 0) return cudaSuccess;
  return tile_w == 4 ? launch_varlen_w<4>(mats, nmat, mode, J0, j0, nb2, nmax, stream)
                     : launch_varlen_w<2>(mats, nmat, mode, J0, j0, nb2, nmax, stream);
}

cudaError_t launch_dsyrk_lower(const DsyrkArgs& a, cudaStream_t stream) {
  if (a.n <= 0 || a.batch <= 0) return cudaSuccess;
  if (a.tile_w == 4) return a.D ? launch_lower_w<true, 4>(a, stream) : launch_lower_w<false, 4>(a, stream);
  return a.D ? launch_lower_w<true, 2>(a, stream) : launch_lower_w<false, 2>(a, stream);
}

}  // namespace rpa
