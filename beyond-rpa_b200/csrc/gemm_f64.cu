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
// CTA tile 64 x 64, 4 warps (2 x 2) of 32 x 32 (4 x 4 DMMA tiles each), K chunks
// of 16 streamed through a 3-stage cp.async pipeline, 4 CTAs per SM.  Each
// operand's shared-memory tile follows its unit-stride index: [k][m] with row
// pitch 72 when m (or n) is contiguous, [m][k] with pitch 18 when k is; both
// pitches make the m8n8k4 fragment loads hit every bank pair exactly twice.
#include <atomic>

#include "kernels.h"

namespace rpa {

namespace {
constexpr int BM = 64;
constexpr int BK = 16;
constexpr int LDM = BM + 8;   // [k][m] pitch
constexpr int LDK = BK + 2;   // [m][k] pitch
constexpr int kTileWords = BK * LDM;  // == BM * LDK = 1152
static_assert(BK * LDM == BM * LDK, "both tile layouts take the same space");
constexpr int kThreads = 128;
constexpr int kStages = 3;
constexpr size_t kSmem = sizeof(double) * (size_t)kStages * (2 * kTileWords + BK);

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
               "l"(gmem), "r"(valid ? 8 : 0)
               : "memory");
}
// 16 bytes (two consecutive elements), the first `bytes` of them copied, the rest zero-filled.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
               "l"(gmem), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// kMC: the operand's row index (m for A, n for B) is the contiguous one -> [k][r] tile;
// otherwise k is contiguous -> [r][k] tile.
template <bool kMC>
__device__ __forceinline__ int tile_off(int r, int k) {
  return kMC ? k * LDM + r : r * LDK + k;
}

// One 64 x 64 output tile (m0, n0) of problem g; b is the batch index (or the split-K index).
// kVec: both operands are copied in 16-byte pairs along their unit-stride index (the launcher
// checked unit strides, even other strides and 16-byte aligned bases).
template <bool kAM, bool kBN, bool kVec = false>
__device__ __forceinline__ void gemm_tile(const GemmF64Args& g, const int m0, const int n0, const int b) {
  extern __shared__ double smem[];
  double* As = smem;                              // [kStages][kTileWords]
  double* Bs = smem + kStages * kTileWords;       // [kStages][kTileWords]
  double* Ss = smem + 2 * kStages * kTileWords;   // [kStages][BK]
  const bool split = g.splitk > 1;
  // split-K: blockIdx.z selects the K range [kbeg, kend) and its partial-product buffer
  int64_t kbeg = 0, kend = g.K;
  if (split) {
    const int64_t kc = ((g.K + g.splitk - 1) / g.splitk + BK - 1) / BK * BK;
    kbeg = (int64_t)b * kc;
    kend = min(g.K, kbeg + kc);
  }
  const double* A = g.A + (split ? 0 : (int64_t)b * g.sA);
  const double* B = g.B + (split ? 0 : (int64_t)b * g.sB);
  double* C = split ? g.work + (int64_t)b * g.M * g.N : g.C + (int64_t)b * g.sC;
  const int64_t ldc = split ? g.M : g.ldc;
  const double* ks = g.kscale ? g.kscale + (split ? 0 : (int64_t)b * g.ks_stride) : nullptr;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int wm = warp >> 1, wn = warp & 1;

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  auto load_stage = [&](int st, int64_t k0) {
    if (kVec) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int idx = t + kThreads * i;
        // pairs along the unit-stride index: (ra, ra+1) or (ca, ca+1)
        const int ra = kAM ? 2 * (idx % (BM / 2)) : idx / (BK / 2), ca = kAM ? idx / (BM / 2) : 2 * (idx % (BK / 2));
        const int64_t ka = k0 + ca;
        const int na = kAM ? ((ka < kend) ? max(0, min(2, g.M - (m0 + ra))) : 0)
                           : ((m0 + ra < g.M) ? (int)max((int64_t)0, min((int64_t)2, kend - ka)) : 0);
        cp_async16(As + st * kTileWords + tile_off<kAM>(ra, ca),
                   na ? A + (int64_t)(m0 + ra) * g.a_m + ka * g.a_k : A, 8 * na);
        const int rb = kBN ? 2 * (idx % (BM / 2)) : idx / (BK / 2), cb = kBN ? idx / (BM / 2) : 2 * (idx % (BK / 2));
        const int64_t kb = k0 + cb;
        const int nb = kBN ? ((kb < kend) ? max(0, min(2, g.N - (n0 + rb))) : 0)
                           : ((n0 + rb < g.N) ? (int)max((int64_t)0, min((int64_t)2, kend - kb)) : 0);
        cp_async16(Bs + st * kTileWords + tile_off<kBN>(rb, cb),
                   nb ? B + kb * g.b_k + (int64_t)(n0 + rb) * g.b_n : B, 8 * nb);
      }
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int idx = t + kThreads * i;
        // consecutive threads walk the operand's unit-stride index
        const int ra = kAM ? idx % BM : idx / BK, ca = kAM ? idx / BM : idx % BK;
        const int64_t ka = k0 + ca;
        const bool va = (m0 + ra < g.M) && (ka < kend);
        cp_async8(As + st * kTileWords + tile_off<kAM>(ra, ca),
                  va ? A + (int64_t)(m0 + ra) * g.a_m + ka * g.a_k : A, va);
        const int rb = kBN ? idx % BM : idx / BK, cb = kBN ? idx / BM : idx % BK;
        const int64_t kb = k0 + cb;
        const bool vb = (n0 + rb < g.N) && (kb < kend);
        cp_async8(Bs + st * kTileWords + tile_off<kBN>(rb, cb),
                  vb ? B + kb * g.b_k + (int64_t)(n0 + rb) * g.b_n : B, vb);
      }
    }
    if (ks && t < BK) {
      const int64_t k = k0 + t;
      Ss[st * BK + t] = k < kend ? ks[k] : 0.0;
    }
  };

  const int64_t nch = kend > kbeg ? (kend - kbeg + BK - 1) / BK : 0;
#pragma unroll
  for (int st = 0; st < kStages - 1; ++st) {
    if (st < nch) load_stage(st, kbeg + (int64_t)st * BK);
    cp_async_commit();
  }
  for (int64_t c = 0; c < nch; ++c) {
    cp_async_wait<kStages - 2>();
    __syncthreads();
    const int64_t cn = c + kStages - 1;
    if (cn < nch) load_stage((int)(cn % kStages), kbeg + cn * BK);
    cp_async_commit();
    const int st = (int)(c % kStages);
    const double* at = As + st * kTileWords;
    const double* bt = Bs + st * kTileWords;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      const int kr = kk + (lane & 3);
      double af[4], bf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) af[i] = at[tile_off<kAM>(wm * 32 + i * 8 + (lane >> 2), kr)];
      const double sc = ks ? Ss[st * BK + kr] : 1.0;
#pragma unroll
      for (int j = 0; j < 4; ++j) bf[j] = bt[tile_off<kBN>(wn * 32 + j * 8 + (lane >> 2), kr)] * sc;
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
  }
  cp_async_wait<0>();

  // With beta != 0 the C fragment of a row group is read before any of it is stored: a
  // load-update-store per element would wait out one memory round trip per element, since the
  // compiler cannot move a load of C above a store to C.
  const bool keep = !split && g.beta != 0.0;
  constexpr int kEpiRows = 1;  // row groups per read-then-write pass (2 spills in the grouped kernel)
#pragma unroll
  for (int i0 = 0; i0 < 4; i0 += kEpiRows) {
    double cv[kEpiRows][4][2];
#pragma unroll
    for (int i = 0; i < kEpiRows; ++i) {
      const int m = m0 + wm * 32 + (i0 + i) * 8 + (lane >> 2);
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int v = 0; v < 2; ++v) {
          const int n = n0 + wn * 32 + j * 8 + 2 * (lane & 3) + v;
          cv[i][j][v] = (keep && m < g.M && n < g.N) ? C[(int64_t)m + ldc * (int64_t)n] : 0.0;
        }
    }
#pragma unroll
    for (int i = 0; i < kEpiRows; ++i) {
      const int m = m0 + wm * 32 + (i0 + i) * 8 + (lane >> 2);
      if (m >= g.M) continue;
      const double rsm = g.rowscale ? g.rowscale[m] : 1.0;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
#pragma unroll
        for (int v = 0; v < 2; ++v) {
          const int n = n0 + wn * 32 + j * 8 + 2 * (lane & 3) + v;
          if (n >= g.N) continue;
          double* p = C + (int64_t)m + ldc * (int64_t)n;
          if (split) {
            *p = acc[i0 + i][j][v];
          } else {
            const double val = g.alpha * rsm * acc[i0 + i][j][v];
            *p = keep ? val + g.beta * cv[i][j][v] : val;
          }
        }
      }
    }
  }
}

template <bool kAM, bool kBN, bool kVec>
__global__ void __launch_bounds__(kThreads, 4) gemm_f64_kernel(const GemmF64Args g) {
  gemm_tile<kAM, kBN, kVec>(g, blockIdx.y * BM, blockIdx.x * BM, blockIdx.z);
}

// Many independent problems of one operand layout in one launch: CTA x works on tile
// x - tile_start[p] of the problem p with tile_start[p] <= x < tile_start[p + 1].
template <bool kAM, bool kBN>
__global__ void __launch_bounds__(kThreads, 4) gemm_f64_grouped_kernel(const GemmF64Args* __restrict__ probs,
                                                                       const int* __restrict__ tile_start,
                                                                       int nprob) {
  const int x = blockIdx.x;
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tile_start[mid] <= x) lo = mid;
    else hi = mid - 1;
  }
  const GemmF64Args& g = probs[lo];  // read through L1 when needed (a register copy would spill)
  const int tiles_n = (g.N + BM - 1) / BM;
  const int t = x - tile_start[lo];
  gemm_tile<kAM, kBN>(g, (t / tiles_n) * BM, (t % tiles_n) * BM, 0);
}

// C = alpha rs(m) sum_s P_s + beta C, partials summed in a fixed order.
__global__ void splitk_reduce_kernel(const GemmF64Args g) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t mn = (int64_t)g.M * g.N;
  if (idx >= mn) return;
  const int64_t m = idx % g.M, n = idx / g.M;
  double s = 0.0;
  for (int z = 0; z < g.splitk; ++z) s += g.work[z * mn + idx];
  double* p = g.C + m + g.ldc * n;
  const double val = g.alpha * (g.rowscale ? g.rowscale[m] : 1.0) * s;
  *p = (g.beta == 0.0) ? val : val + g.beta * *p;
}

template <bool kAM, bool kBN, bool kVec>
cudaError_t launch_variant(const GemmF64Args& g, cudaStream_t stream) {
  // per-variant bit per device: dynamic shared memory opted in (atomic: handles on different
  // devices may launch from different host threads)
  static std::atomic<uint64_t> attr_set{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 64 || !(attr_set.load(std::memory_order_relaxed) >> dev & 1)) {
    e = cudaFuncSetAttribute(gemm_f64_kernel<kAM, kBN, kVec>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kSmem);
    if (e != cudaSuccess) return e;
    if (dev < 64) attr_set.fetch_or(1ull << dev, std::memory_order_relaxed);
  }
  const bool split = g.splitk > 1;
  dim3 grid((unsigned)((g.N + BM - 1) / BM), (unsigned)((g.M + BM - 1) / BM),
            (unsigned)(split ? g.splitk : g.batch));
  gemm_f64_kernel<kAM, kBN, kVec><<<grid, kThreads, kSmem, stream>>>(g);
  if (split) {
    const int64_t mn = (int64_t)g.M * g.N;
    splitk_reduce_kernel<<<(unsigned)((mn + 255) / 256), 256, 0, stream>>>(g);
  }
  return cudaGetLastError();
}
}  // namespace

template <bool kAM, bool kBN>
cudaError_t set_smem_attr() {
  static std::atomic<uint64_t> done{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 64 && (done.load(std::memory_order_relaxed) >> dev & 1)) return cudaSuccess;
  e = cudaFuncSetAttribute(gemm_f64_grouped_kernel<kAM, kBN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem);
  if (e == cudaSuccess && dev < 64) done.fetch_or(1ull << dev, std::memory_order_relaxed);
  return e;
}

template <bool kAM, bool kBN>
cudaError_t launch_grouped_variant(const GemmF64Args* probs, const int* tile_start, int nprob, int ntiles,
                                   cudaStream_t stream) {
  cudaError_t e = set_smem_attr<kAM, kBN>();
  if (e != cudaSuccess) return e;
  gemm_f64_grouped_kernel<kAM, kBN><<<ntiles, kThreads, kSmem, stream>>>(probs, tile_start, nprob);
  return cudaGetLastError();
}

cudaError_t launch_gemm_f64_grouped(const std::vector<GemmF64Args>& probs, void* dev_buf, size_t dev_bytes,
                                    cudaStream_t stream) {
  if (probs.empty()) return cudaSuccess;
  const bool am = (probs[0].a_m == 1), bn = (probs[0].b_n == 1);
  std::vector<int> start(probs.size() + 1, 0);
  for (size_t p = 0; p < probs.size(); ++p) {
    const GemmF64Args& g = probs[p];
    // the layout template only chooses the load mapping (loads use the general strides), so
    // problems whose unit strides differ from the first one's stay correct, just less coalesced
    if (g.batch != 1 || g.splitk > 1) return cudaErrorInvalidValue;
    const int t = (g.M > 0 && g.N > 0) ? ((g.M + BM - 1) / BM) * ((g.N + BM - 1) / BM) : 0;
    start[p + 1] = start[p] + t;
  }
  const int ntiles = start.back();
  if (ntiles == 0) return cudaSuccess;
  const size_t pb = probs.size() * sizeof(GemmF64Args);
  const size_t need = pb + start.size() * sizeof(int);
  if (need > dev_bytes) return cudaErrorInvalidValue;
  // stream-ordered uploads: a later upload into the same buffer waits for this launch
  char* base = static_cast<char*>(dev_buf);
  cudaError_t e = cudaMemcpyAsync(base, probs.data(), pb, cudaMemcpyHostToDevice, stream);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(base + pb, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice, stream);
  if (e != cudaSuccess) return e;
  const GemmF64Args* dp = reinterpret_cast<const GemmF64Args*>(base);
  const int* ds = reinterpret_cast<const int*>(base + pb);
  const int np = (int)probs.size();
  if (am) e = bn ? launch_grouped_variant<true, true>(dp, ds, np, ntiles, stream)
                 : launch_grouped_variant<true, false>(dp, ds, np, ntiles, stream);
  else e = bn ? launch_grouped_variant<false, true>(dp, ds, np, ntiles, stream)
              : launch_grouped_variant<false, false>(dp, ds, np, ntiles, stream);
  ++g_launches;
  return e;
}

cudaError_t launch_gemm_f64_grouped_dev(const GemmF64Args* probs_dev, const int* tile_start_dev, int nprob,
                                        int ntiles, bool a_m_unit, bool b_n_unit, cudaStream_t stream) {
  if (nprob <= 0 || ntiles <= 0) return cudaSuccess;
  cudaError_t e;
  if (a_m_unit) e = b_n_unit ? launch_grouped_variant<true, true>(probs_dev, tile_start_dev, nprob, ntiles, stream)
                             : launch_grouped_variant<true, false>(probs_dev, tile_start_dev, nprob, ntiles, stream);
  else e = b_n_unit ? launch_grouped_variant<false, true>(probs_dev, tile_start_dev, nprob, ntiles, stream)
                    : launch_grouped_variant<false, false>(probs_dev, tile_start_dev, nprob, ntiles, stream);
  ++g_launches;
  return e;
}

int gemm_f64_tiles(const GemmF64Args& g) {
  return (g.M > 0 && g.N > 0) ? ((g.M + BM - 1) / BM) * ((g.N + BM - 1) / BM) : 0;
}

namespace {
// 16-byte pair copies: unit stride along the pair, the other stride and the batch stride even,
// a 16-byte aligned base (split-K ranges start at multiples of 16).
bool pairable(const double* p, int64_t unit, int64_t other, int64_t batch_stride, bool batched) {
  return unit == 1 && (other & 1) == 0 && (!batched || (batch_stride & 1) == 0) &&
         (reinterpret_cast<uintptr_t>(p) & 15) == 0;
}
template <bool kAM, bool kBN>
cudaError_t launch_layout(const GemmF64Args& g, cudaStream_t stream) {
  const bool batched = g.batch > 1 && g.splitk <= 1;
  const bool vec = pairable(g.A, kAM ? g.a_m : g.a_k, kAM ? g.a_k : g.a_m, g.sA, batched) &&
                   pairable(g.B, kBN ? g.b_n : g.b_k, kBN ? g.b_k : g.b_n, g.sB, batched);
  return vec ? launch_variant<kAM, kBN, true>(g, stream) : launch_variant<kAM, kBN, false>(g, stream);
}
}  // namespace

cudaError_t launch_gemm_f64(const GemmF64Args& g, cudaStream_t stream) {
  if (g.M <= 0 || g.N <= 0 || g.batch <= 0) return cudaSuccess;
  if (g.splitk > 1 && (g.batch != 1 || !g.work)) return cudaErrorInvalidValue;
  const bool am = (g.a_m == 1), bn = (g.b_n == 1);
  cudaError_t e;
  if (am) e = bn ? launch_layout<true, true>(g, stream) : launch_layout<true, false>(g, stream);
  else e = bn ? launch_layout<false, true>(g, stream) : launch_layout<false, false>(g, stream);
  g_launches += g.splitk > 1 ? 2 : 1;
  return e;
}

}  // namespace rpa
