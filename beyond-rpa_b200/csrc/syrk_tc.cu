// Split-BF16 SYRK on the 5th-generation tensor cores (tcgen05 + TMEM + TMA).
//
//   Pi_k(m, n) = sum_ai X_k(m, ai) X_k(n, ai),   m >= n,
//   X = H + L (bf16 hi/lo):  Pi ~= H H^T + H L^T + L H^T   (FP32 accumulate)
// and the diagonal is replaced by the exact FP64 value from the scale/split
// pass (the dropped L L^T term only biases the diagonal systematically).
// This is the contraction of rpa_THC_PiU_BlockAlgo (src/rpa/rpa_THC.f90:
// 313-339, DGEMM real_abT_x of a 500-column block, repeated per frequency),
// done as one lower-triangle SYRK per frequency over all ai at once.
//
// Persistent kernel, one CTA per SM, 576 threads:
//   warp 0      TMA producer (one elected lane)
//   warp 1      TMEM allocator + MMA issuer (one elected lane)
//   warps 2..17 epilogue: TMEM -> registers -> FP64 global stores
//               (warp w reads TMEM lanes 32*(w%4).. and 64 accumulator columns)
// Work unit = (frequency k, 128-row tile tm, 256-column tile tn) with
// tm*128 + 127 >= tn*256 (touches the lower triangle); a unit whose last
// columns lie above the diagonal or beyond NQ issues a narrower MMA (N = the
// columns that can hold lower-triangle entries, rounded up to 16).  Segmented
// accumulation: the ai range of a unit is cut into segments of
// `seg_chunks` x 32 columns; each segment accumulates into a fresh 128 x 256
// FP32 TMEM accumulator (two of them, 512 columns, alternate), and the
// epilogue warps add the segment partials in IEEE FP32 registers.  The
// tensor-core accumulator rounds toward zero, so its relative bias grows
// with the accumulation depth; segmenting bounds that depth (at NQ = 4096,
// nov = 65536 an unsegmented accumulator biases E_c by ~1e-5 Eh).
// Smem pipeline: 4 stages of {A_hi, A_lo (128x32), B_hi, B_lo (256x32)}
// bf16, 64-byte swizzle.
#include <vector>

#include "kernels.h"

namespace rpa {

namespace {
constexpr int TM = kSyrkTcTM, TN = kSyrkTcTN, TK = kSyrkTcTK;
constexpr int kStages = 4;
constexpr int kATileBytes = TM * TK * 2;  // 8 KB
constexpr int kBTileBytes = TN * TK * 2;  // 16 KB
constexpr int kStageBytes = 2 * kATileBytes + 2 * kBTileBytes;  // 48 KB
constexpr int kThreads = 576;
constexpr int kEpiWarps = 16;
constexpr int kEpiCols = TN / 4;  // accumulator columns per epilogue warp
constexpr uint32_t kTmemCols = 512;
constexpr int kSmemBytes = kStages * kStageBytes + 1024 /*align slack*/ + 256 /*barriers*/;

struct UnitCoord {
  int k, tm, tn;
};

__device__ __forceinline__ UnitCoord decode_unit(int u, int nblocks, int ntm) {
  UnitCoord c;
  c.k = u / nblocks;
  int b = u - c.k * nblocks;
  int tn = 0;
  while (true) {
    const int cnt = ntm - 2 * tn;
    if (b < cnt) break;
    b -= cnt;
    ++tn;
  }
  c.tn = tn;
  c.tm = 2 * tn + b;
  return c;
}

// What a CTA needs to know about one work unit.
struct Unit {
  int k, tm, tn, NQ, nchunks;
  int chunk0;          // first 32-column chunk of X
  bool accumulate;     // Pi += contribution instead of Pi = contribution
  double* Pk;          // Pi of this frequency
  int64_t ldPi;
  const double* dk;    // exact diagonal of this frequency
  const CUtensorMap* map[4];  // A_hi, A_lo, B_hi, B_lo
  // full GEMM units (tri == false): C(m, n) = alpha sum_k A(m,k) B(n,k) + beta C(m, n),
  // m < NQ (rows of A), n < N (rows of B); C = Pk with leading dimension ldPi
  bool tri = true;
  int N = 0;
  double alpha = 1.0, beta = 0.0;
};

// Single instance: tensor maps are kernel parameters, units are decoded.
struct SingleSource {
  const CUtensorMap* maps[4];
  SyrkTcArgs a;
  int nblocks, ntm, nchunks, nunits;
  __device__ __forceinline__ int* sync_counters() const { return a.sync; }
  __device__ __forceinline__ int sync_every() const { return a.sync_every; }
  __device__ __forceinline__ int sync_lag() const { return a.sync_lag; }
  __device__ __forceinline__ int max_chunks() const { return nchunks; }
  __device__ __forceinline__ Unit get(int u) const {
    const UnitCoord c = decode_unit(u, nblocks, ntm);
    Unit x;
    x.k = c.k;
    x.tm = c.tm;
    x.tn = c.tn;
    x.NQ = a.NQ;
    x.nchunks = nchunks;
    x.chunk0 = a.chunk0;
    x.accumulate = a.accumulate != 0;
    x.Pk = a.Pi + (int64_t)c.k * a.piStride;
    x.ldPi = a.ldPi;
    x.dk = a.diag ? a.diag + (int64_t)c.k * a.NQ : nullptr;
    for (int i = 0; i < 4; ++i) x.map[i] = maps[i];
    return x;
  }
};

// Many instances: per-instance descriptors (tensor maps in global memory) and a work list.
struct MultiSource {
  const SyrkInst* insts;
  const uint4* work;  // (instance, k, tm, tn)
  int nunits;
  int* sync;
  int sync_every_, sync_lag_, max_chunks_;
  __device__ __forceinline__ int* sync_counters() const { return sync; }
  __device__ __forceinline__ int sync_every() const { return sync_every_; }
  __device__ __forceinline__ int sync_lag() const { return sync_lag_; }
  __device__ __forceinline__ int max_chunks() const { return max_chunks_; }
  __device__ __forceinline__ Unit get(int u) const {
    const uint4 w = work[u];
    const SyrkInst& in = insts[w.x];
    Unit x;
    x.k = (int)w.y;
    x.tm = (int)w.z;
    x.tn = (int)w.w;
    x.NQ = in.NQ;
    x.nchunks = in.nchunks;
    x.chunk0 = 0;
    x.accumulate = false;
    x.Pk = in.Pi + (int64_t)x.k * in.piStride;
    x.ldPi = in.ldPi;
    x.dk = in.diag + (int64_t)x.k * in.NQ;
    x.map[0] = &in.tmAh;
    x.map[1] = &in.tmAl;
    x.map[2] = &in.tmBh;
    x.map[3] = &in.tmBl;
    return x;
  }
};

// General GEMM: tensor maps are kernel parameters; units (tm, tn) over the full tile grid,
// tm-major (consecutive units share an A band).
struct GemmSource {
  const CUtensorMap* maps[4];
  GemmSplitArgs a;
  int ntn, nchunks, nunits;
  __device__ __forceinline__ int* sync_counters() const { return a.sync; }
  __device__ __forceinline__ int sync_every() const { return a.sync_every; }
  __device__ __forceinline__ int sync_lag() const { return a.sync_lag; }
  __device__ __forceinline__ int max_chunks() const { return nchunks; }
  __device__ __forceinline__ Unit get(int u) const {
    Unit x;
    x.k = 0;
    x.tm = u / ntn;
    x.tn = u - x.tm * ntn;
    x.NQ = a.M;
    x.N = a.N;
    x.nchunks = nchunks;
    x.chunk0 = 0;
    x.accumulate = false;
    x.Pk = a.C;
    x.ldPi = a.ldc;
    x.dk = nullptr;
    x.tri = false;
    x.alpha = a.alpha;
    x.beta = a.beta;
    for (int i = 0; i < 4; ++i) x.map[i] = maps[i];
    return x;
  }
};

// Bounded wait until *c >= target (acquire); false when it gave up (~70 ms).
__device__ __noinline__ bool wait_count(const int* c, int target) {
  for (uint32_t it = 0; it < (1u << 20); ++it) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(c) : "memory");
    if (v >= target) return true;
    __nanosleep(64);
  }
  return false;
}

template <class Source>
__device__ __forceinline__ void syrk_body(const Source& src, int* err, const int seg_chunks) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* acc_full = empty + kStages;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* drain = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int nunits = src.nunits;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], kEpiWarps);
    }
    mbar_init(drain, 1);
    fence_mbar_init();
  }
  if (warp == 1) tmem_alloc(tmem_slot, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  auto a_hi = [&](int s) { return smem + s * kStageBytes; };
  auto a_lo = [&](int s) { return smem + s * kStageBytes + kATileBytes; };
  auto b_hi = [&](int s) { return smem + s * kStageBytes + 2 * kATileBytes; };
  auto b_lo = [&](int s) { return smem + s * kStageBytes + 2 * kATileBytes + kBTileBytes; };

  if (warp == 0) {
    if (lane == 0) {
      // ------------------------------------------------------------ producer
      int stage = 0;
      uint32_t phase = 0;
      uint32_t issued = 0, issued_par = 0;  // per-stage bit masks: issued, parity of the last issue
      bool ok = true;
      const CUtensorMap* last = nullptr;
      int* const sync = src.sync_counters();
      const int sync_every = src.sync_every(), sync_lag = src.sync_lag();
      const int nmile = sync ? (src.max_chunks() + sync_every - 1) / sync_every : 0;
      bool sync_wait = true;  // cleared for good if a wait ever runs out of time
      for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
        const Unit x = src.get(u);
        if (x.map[0] != last) {
          for (int i = 0; i < 4; ++i) tma_prefetch_desc(x.map[i]);
          last = x.map[0];
        }
        const int wave = (u - (int)blockIdx.x) / (int)gridDim.x;
        const int members = min((int)gridDim.x, nunits - wave * (int)gridDim.x);
        // a lower-triangle unit whose live columns fit 128 rows (the first 128-row tile of a
        // 256-column block on the diagonal, a ragged last block) loads B through the 128-row box
        // of the same tensor (the A maps): half the B bytes, and the MMA reads only those rows
        const bool narrowB = x.tri && min(x.NQ, (x.tm + 1) * TM) - x.tn * TN <= TM;
        const CUtensorMap* mbh = narrowB ? x.map[0] : x.map[2];
        const CUtensorMap* mbl = narrowB ? x.map[1] : x.map[3];
        const uint32_t stage_bytes = narrowB ? 4 * kATileBytes : kStageBytes;
        for (int ch = 0; ch < x.nchunks; ++ch) {
          if (sync && ch % sync_every == 0) {
            const int mi = ch / sync_every;
            int* row = sync + (int64_t)wave * nmile;
            asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(row + mi) : "memory");
            if (sync_wait && mi >= sync_lag) sync_wait = wait_count(row + mi - sync_lag, members);
          }
          if (!mbar_wait(&empty[stage], phase ^ 1u, err, kDevTimeoutTmaEmpty)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&full[stage], stage_bytes);
          const int c0 = (x.chunk0 + ch) * TK;
          tma_load_3d(a_hi(stage), x.map[0], &full[stage], c0, x.tm * TM, x.k);
          tma_load_3d(a_lo(stage), x.map[1], &full[stage], c0, x.tm * TM, x.k);
          tma_load_3d(b_hi(stage), mbh, &full[stage], c0, x.tn * TN, x.k);
          tma_load_3d(b_lo(stage), mbl, &full[stage], c0, x.tn * TN, x.k);
          issued |= 1u << stage;
          issued_par = (issued_par & ~(1u << stage)) | (phase << stage);
          if (++stage == kStages) {
            stage = 0;
            phase ^= 1u;
          }
        }
        if (sync && ok) {  // a unit shorter than the longest of the launch: release the later milestones
          int* row = sync + (int64_t)wave * nmile;
          for (int mi = (x.nchunks + sync_every - 1) / sync_every; mi < nmile; ++mi)
            asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(row + mi) : "memory");
        }
      }
      // make sure no bulk copy is still landing in shared memory at exit
      for (int s = 0; s < kStages; ++s)
        if (issued & (1u << s)) mbar_wait(&full[s], (issued_par >> s) & 1u, err, kDevTimeoutDrain);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ------------------------------------------------------------ MMA issuer
      int stage = 0;
      uint32_t phase = 0;
      int it = 0;  // segment counter (selects the TMEM accumulator)
      bool ok = true;
      for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
        const Unit x = src.get(u);
        const int nchunks = x.nchunks;
        // MMA width of this unit: only columns n < min(NQ, (tm+1)*TM) can hold lower-triangle
        // entries (the first 128 rows of a 256-column block on the diagonal, the ragged last
        // block), rounded up to the N granularity (16) of a 128-row MMA
        const int live = x.tri ? min(x.NQ, (x.tm + 1) * TM) - x.tn * TN : x.N - x.tn * TN;
        const int nmma = min(TN, max(16, (live + 15) & ~15));
        const uint32_t idesc = umma_idesc_bf16_f32(TM, nmma);
        for (int c0 = 0; c0 < nchunks && ok; c0 += seg_chunks, ++it) {
          const int b = it & 1;
          const uint32_t acc_phase = (uint32_t)((it >> 1) & 1);
          if (!mbar_wait(&acc_empty[b], acc_phase ^ 1u, err, kDevTimeoutAccEmpty)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d_tmem = tmem_base + (uint32_t)(b * TN);
          const int c1 = min(nchunks, c0 + seg_chunks);
          for (int ch = c0; ch < c1; ++ch) {
            if (!mbar_wait(&full[stage], phase, err, kDevTimeoutTmaFull)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t ah = smem_u32(a_hi(stage)), al = smem_u32(a_lo(stage));
            const uint32_t bh = smem_u32(b_hi(stage)), bl = smem_u32(b_lo(stage));
#pragma unroll
            for (int kk = 0; kk < TK / 16; ++kk) {
              const uint32_t off = (uint32_t)(kk * 32);  // 16 bf16 = 32 bytes along K
              const uint64_t dah = umma_desc_k_sw64(ah + off), dal = umma_desc_k_sw64(al + off);
              const uint64_t dbh = umma_desc_k_sw64(bh + off), dbl = umma_desc_k_sw64(bl + off);
              tc_mma_bf16(d_tmem, dah, dbh, idesc, (ch > c0 || kk > 0) ? 1u : 0u);
              tc_mma_bf16(d_tmem, dah, dbl, idesc, 1u);
              tc_mma_bf16(d_tmem, dal, dbh, idesc, 1u);
            }
            tc_commit(&empty[stage]);
            if (++stage == kStages) {
              stage = 0;
              phase ^= 1u;
            }
          }
          if (!ok) break;
          tc_commit(&acc_full[b]);
        }
      }
      // drain: wait until every issued MMA has completed before TMEM is freed
      tc_commit(drain);
      mbar_wait(drain, 0, err, kDevTimeoutDrain);
    }
  } else {
    // -------------------------------------------------------------- epilogue
    const int quarter = warp & 3;            // TMEM lanes quarter*32 .. +31
    const int colq = (warp - 2) >> 2;        // accumulator columns colq*64 .. +63
    int it = 0;
    bool ok = true;
    float run[kEpiCols];
    for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
      const Unit x = src.get(u);
      const int m = x.tm * TM + quarter * 32 + lane;
      const int warp_max_m = x.tm * TM + quarter * 32 + 31;
      const int nbase = x.tn * TN + colq * kEpiCols;
      for (int c0 = 0; c0 < x.nchunks; c0 += seg_chunks, ++it) {
        const int b = it & 1;
        const uint32_t acc_phase = (uint32_t)((it >> 1) & 1);
        if (!mbar_wait(&acc_full[b], acc_phase, err, kDevTimeoutAccFull)) {
          ok = false;
          break;
        }
        tc_fence_after();
#pragma unroll
        for (int cc = 0; cc < kEpiCols / 8; ++cc) {
          const int n0 = nbase + cc * 8;
          if (x.tri ? (n0 <= warp_max_m && n0 < x.NQ) : n0 < x.N)  // warp-uniform: skip columns above
                                                                      // the diagonal or beyond N
            tmem_ld_add_x8(tmem_base + (uint32_t)(b * TN + colq * kEpiCols + cc * 8) + ((uint32_t)(quarter * 32) << 16),
                           &run[cc * 8], c0 == 0);
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&acc_empty[b]);
      }
      if (!ok) break;
      if (!x.tri) {
        if (m < x.NQ) {
          double* p = x.Pk + (int64_t)m + (int64_t)nbase * x.ldPi;
          const int ncol = min(kEpiCols, x.N - nbase);
#pragma unroll
          for (int j = 0; j < kEpiCols; ++j) {
            if (j < ncol) *p = x.beta == 0.0 ? x.alpha * (double)run[j] : fma(x.alpha, (double)run[j], x.beta * *p);
            p += x.ldPi;
          }
        }
      } else if (m < x.NQ && nbase <= m) {
        double* p = x.Pk + (int64_t)m + (int64_t)nbase * x.ldPi;
        const int jd = m - nbase;  // column index of the diagonal element (may be >= kEpiCols)
        if (x.accumulate) {
#pragma unroll
          for (int j = 0; j < kEpiCols; ++j) {
            if (j < jd) *p += (double)run[j];
            p += x.ldPi;
          }
        } else {
#pragma unroll
          for (int j = 0; j < kEpiCols; ++j) {
            if (j < jd) *p = (double)run[j];
            p += x.ldPi;
          }
        }
        if (jd < kEpiCols && x.dk) x.Pk[(int64_t)m * (x.ldPi + 1)] = x.dk[m];
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, kTmemCols);
  }
}

__global__ void __launch_bounds__(kThreads, 1)
    syrk_split_bf16_kernel(const __grid_constant__ CUtensorMap tmA_hi, const __grid_constant__ CUtensorMap tmA_lo,
                           const __grid_constant__ CUtensorMap tmB_hi, const __grid_constant__ CUtensorMap tmB_lo,
                           const SyrkTcArgs args, const int nblocks, const int ntm, const int nunits,
                           const int nchunks, const int seg_chunks) {
  SingleSource src;
  src.maps[0] = &tmA_hi;
  src.maps[1] = &tmA_lo;
  src.maps[2] = &tmB_hi;
  src.maps[3] = &tmB_lo;
  src.a = args;
  src.nblocks = nblocks;
  src.ntm = ntm;
  src.nchunks = nchunks;
  src.nunits = nunits;
  syrk_body(src, args.err, seg_chunks);
}

// Many instances (fragments) in one persistent launch.
__global__ void __launch_bounds__(kThreads, 1)
    syrk_split_bf16_multi_kernel(const SyrkInst* __restrict__ insts, const uint4* __restrict__ work, const int nunits,
                                 int* err, const int seg_chunks, int* sync, const int sync_every, const int sync_lag,
                                 const int max_chunks) {
  MultiSource src;
  src.insts = insts;
  src.work = work;
  src.nunits = nunits;
  src.sync = sync;
  src.sync_every_ = sync_every > 0 ? sync_every : 1;
  src.sync_lag_ = sync_lag;
  src.max_chunks_ = max_chunks;
  syrk_body(src, err, seg_chunks);
}
__global__ void __launch_bounds__(kThreads, 1)
    gemm_split_bf16_kernel(const __grid_constant__ CUtensorMap tmA_hi, const __grid_constant__ CUtensorMap tmA_lo,
                           const __grid_constant__ CUtensorMap tmB_hi, const __grid_constant__ CUtensorMap tmB_lo,
                           const GemmSplitArgs args, const int ntn, const int nunits, const int nchunks) {
  GemmSource src;
  src.maps[0] = &tmA_hi;
  src.maps[1] = &tmA_lo;
  src.maps[2] = &tmB_hi;
  src.maps[3] = &tmB_lo;
  src.a = args;
  src.ntn = ntn;
  src.nchunks = nchunks;
  src.nunits = nunits;
  syrk_body(src, args.err, args.seg_chunks > 0 ? args.seg_chunks : nchunks);
}
}  // namespace

int64_t gemm_split_sync_words(int M, int N, int64_t K, int num_sms, int sync_every) {
  if (sync_every <= 0) return 0;
  const int64_t nunits = (int64_t)((M + TM - 1) / TM) * ((N + TN - 1) / TN);
  const int64_t grid = nunits < num_sms ? nunits : num_sms;
  if (grid <= 0) return 0;
  const int64_t nchunks = (K + TK - 1) / TK;
  return (nunits + grid - 1) / grid * ((nchunks + sync_every - 1) / sync_every);
}

cudaError_t launch_gemm_split_bf16(const CUtensorMap* maps, const GemmSplitArgs& a, int num_sms,
                                   cudaStream_t stream) {
  const int64_t ntm = (a.M + TM - 1) / TM, ntn = (a.N + TN - 1) / TN;
  const int64_t nunits = ntm * ntn;
  const int64_t nchunks = (a.K + TK - 1) / TK;
  if (a.M <= 0 || a.N <= 0 || a.K <= 0) return cudaSuccess;
  if (nunits > INT32_MAX || nchunks > INT32_MAX) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(gemm_split_bf16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kSmemBytes);
  if (e != cudaSuccess) return e;
  const int grid = nunits < num_sms ? (int)nunits : num_sms;
  gemm_split_bf16_kernel<<<grid, kThreads, kSmemBytes, stream>>>(maps[0], maps[1], maps[2], maps[3], a, (int)ntn,
                                                                  (int)nunits, (int)nchunks);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_syrk_split_bf16(const CUtensorMap* tmA_hi, const CUtensorMap* tmA_lo, const CUtensorMap* tmB_hi,
                                   const CUtensorMap* tmB_lo, const SyrkTcArgs& a, int num_sms,
                                   cudaStream_t stream) {
  const int ntm = (a.NQ + TM - 1) / TM;
  const int ntn = (a.NQ + TN - 1) / TN;
  int nblocks = 0;
  for (int tn = 0; tn < ntn; ++tn) nblocks += (ntm - 2 * tn > 0) ? (ntm - 2 * tn) : 0;
  const int nunits = nblocks * a.kg;
  const int64_t span = a.nov_part > 0 ? a.nov_part : a.nov;
  const int nchunks = (int)((span + TK - 1) / TK);
  if (a.chunk0 < 0 || (int64_t)a.chunk0 * TK + span > ((a.nov + TK - 1) / TK) * TK) return cudaErrorInvalidValue;
  if (nunits == 0 || nchunks == 0) return cudaSuccess;
  cudaError_t e =
      cudaFuncSetAttribute(syrk_split_bf16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
  if (e != cudaSuccess) return e;
  const int grid = nunits < num_sms ? nunits : num_sms;
  const int seg_chunks = a.seg_chunks > 0 ? a.seg_chunks : nchunks;
  syrk_split_bf16_kernel<<<grid, kThreads, kSmemBytes, stream>>>(*tmA_hi, *tmA_lo, *tmB_hi, *tmB_lo, a, nblocks,
                                                                  ntm, nunits, nchunks, seg_chunks);
  ++g_launches;
  return cudaGetLastError();
}

int64_t syrk_tc_sync_words(int NQ, int kg, int64_t nov_part, int num_sms, int sync_every) {
  if (sync_every <= 0) return 0;
  const int nunits = syrk_tc_blocks(NQ) * kg;
  const int grid = nunits < num_sms ? nunits : num_sms;
  if (grid <= 0) return 0;
  const int64_t waves = (nunits + grid - 1) / grid;
  const int64_t nchunks = (nov_part + TK - 1) / TK;
  return waves * ((nchunks + sync_every - 1) / sync_every);
}

int syrk_tc_blocks(int NQ) {
  const int ntm = (NQ + TM - 1) / TM;
  const int ntn = (NQ + TN - 1) / TN;
  int nblocks = 0;
  for (int tn = 0; tn < ntn; ++tn) nblocks += (ntm - 2 * tn > 0) ? (ntm - 2 * tn) : 0;
  return nblocks;
}

void syrk_tc_block_coords(int NQ, std::vector<uint2>& out) {
  const int ntm = (NQ + TM - 1) / TM;
  const int ntn = (NQ + TN - 1) / TN;
  out.clear();
  for (int tn = 0; tn < ntn; ++tn)
    for (int tm = 2 * tn; tm < ntm; ++tm) out.push_back(make_uint2((unsigned)tm, (unsigned)tn));
}

int64_t syrk_tc_multi_sync_words(int nunits, int max_chunks, int num_sms, int sync_every) {
  if (sync_every <= 0 || nunits <= 0) return 0;
  const int grid = nunits < num_sms ? nunits : num_sms;
  const int64_t waves = (nunits + grid - 1) / grid;
  return waves * ((max_chunks + sync_every - 1) / sync_every);
}

cudaError_t launch_syrk_split_bf16_multi(const SyrkInst* insts, const uint4* work, int nunits, int seg_chunks,
                                         int* err, int num_sms, cudaStream_t stream, int* sync, int sync_every,
                                         int sync_lag, int max_chunks) {
  if (nunits == 0) return cudaSuccess;
  cudaError_t e =
      cudaFuncSetAttribute(syrk_split_bf16_multi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
  if (e != cudaSuccess) return e;
  const int grid = nunits < num_sms ? nunits : num_sms;
  syrk_split_bf16_multi_kernel<<<grid, kThreads, kSmemBytes, stream>>>(insts, work, nunits, err, seg_chunks, sync,
                                                                       sync_every, sync_lag, max_chunks);
  ++g_launches;
  return cudaGetLastError();
}

}  // namespace rpa
