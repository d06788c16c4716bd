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
// Persistent kernel, one CTA per SM, 192 threads:
//   warp 0      TMA producer (one elected lane)
//   warp 1      TMEM allocator + MMA issuer (one elected lane)
//   warps 2..5  epilogue: TMEM -> registers -> FP64 global stores
// Work unit = (frequency k, 128-row tile tm, 256-column tile tn) with
// tm*128 + 127 >= tn*256 (touches the lower triangle).  The 128 x 256 FP32
// accumulator lives in TMEM; two accumulators (512 columns) let the epilogue
// of one unit overlap the main loop of the next.  Smem pipeline: 4 stages of
// {A_hi, A_lo (128x32), B_hi, B_lo (256x32)} bf16, 64-byte swizzle.
#include "kernels.h"

namespace rpa {

namespace {
constexpr int TM = kSyrkTcTM, TN = kSyrkTcTN, TK = kSyrkTcTK;
constexpr int kStages = 4;
constexpr int kATileBytes = TM * TK * 2;  // 8 KB
constexpr int kBTileBytes = TN * TK * 2;  // 16 KB
constexpr int kStageBytes = 2 * kATileBytes + 2 * kBTileBytes;  // 48 KB
constexpr int kThreads = 192;
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kIdesc = umma_idesc_bf16_f32(TM, TN);
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

__global__ void __launch_bounds__(kThreads, 1)
    syrk_split_bf16_kernel(const __grid_constant__ CUtensorMap tmA_hi, const __grid_constant__ CUtensorMap tmA_lo,
                           const __grid_constant__ CUtensorMap tmB_hi, const __grid_constant__ CUtensorMap tmB_lo,
                           const SyrkTcArgs args, const int nblocks, const int ntm, const int nunits,
                           const int nchunks) {
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
  int* err = args.err;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 4);
    }
    mbar_init(drain, 1);
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    tma_prefetch_desc(&tmA_hi);
    tma_prefetch_desc(&tmA_lo);
    tma_prefetch_desc(&tmB_hi);
    tma_prefetch_desc(&tmB_lo);
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
      int issued_parity[kStages];
      for (int s = 0; s < kStages; ++s) issued_parity[s] = -1;
      bool ok = true;
      for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
        const UnitCoord c = decode_unit(u, nblocks, ntm);
        for (int ch = 0; ch < nchunks; ++ch) {
          if (!mbar_wait(&empty[stage], phase ^ 1u, err, kDevTimeoutTmaEmpty)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&full[stage], kStageBytes);
          const int x = ch * TK;
          tma_load_3d(a_hi(stage), &tmA_hi, &full[stage], x, c.tm * TM, c.k);
          tma_load_3d(a_lo(stage), &tmA_lo, &full[stage], x, c.tm * TM, c.k);
          tma_load_3d(b_hi(stage), &tmB_hi, &full[stage], x, c.tn * TN, c.k);
          tma_load_3d(b_lo(stage), &tmB_lo, &full[stage], x, c.tn * TN, c.k);
          issued_parity[stage] = (int)phase;
          if (++stage == kStages) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      // make sure no bulk copy is still landing in shared memory at exit
      for (int s = 0; s < kStages; ++s)
        if (issued_parity[s] >= 0) mbar_wait(&full[s], (uint32_t)issued_parity[s], err, kDevTimeoutDrain);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ------------------------------------------------------------ MMA issuer
      int stage = 0;
      uint32_t phase = 0;
      int it = 0;
      bool ok = true;
      for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x, ++it) {
        const int b = it & 1;
        const uint32_t acc_phase = (uint32_t)((it >> 1) & 1);
        if (!mbar_wait(&acc_empty[b], acc_phase ^ 1u, err, kDevTimeoutAccEmpty)) break;
        tc_fence_after();
        const uint32_t d_tmem = tmem_base + (uint32_t)(b * TN);
        for (int ch = 0; ch < nchunks; ++ch) {
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
            tc_mma_bf16(d_tmem, dah, dbh, kIdesc, (ch > 0 || kk > 0) ? 1u : 0u);
            tc_mma_bf16(d_tmem, dah, dbl, kIdesc, 1u);
            tc_mma_bf16(d_tmem, dal, dbh, kIdesc, 1u);
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
      // drain: wait until every issued MMA has completed before TMEM is freed
      tc_commit(drain);
      mbar_wait(drain, 0, err, kDevTimeoutDrain);
    }
  } else {
    // -------------------------------------------------------------- epilogue
    const int quarter = warp & 3;  // TMEM lanes quarter*32 .. +31
    int it = 0;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x, ++it) {
      const int b = it & 1;
      const uint32_t acc_phase = (uint32_t)((it >> 1) & 1);
      if (!mbar_wait(&acc_full[b], acc_phase, err, kDevTimeoutAccFull)) break;
      tc_fence_after();
      const UnitCoord c = decode_unit(u, nblocks, ntm);
      const int m = c.tm * TM + quarter * 32 + lane;
      const int warp_max_m = c.tm * TM + quarter * 32 + 31;
      double* Pk = args.Pi + (int64_t)c.k * args.piStride;
      const double* dk = args.diag + (int64_t)c.k * args.NQ;
      const double dm = (m < args.NQ) ? dk[m] : 0.0;
#pragma unroll 1
      for (int cc = 0; cc < TN; cc += 32) {
        const int n0 = c.tn * TN + cc;
        if (n0 > warp_max_m || n0 >= args.NQ) break;  // warp-uniform: rest is above the diagonal
        float v[32];
        tmem_ld_32x32b_x32(tmem_base + (uint32_t)(b * TN + cc) + ((uint32_t)(quarter * 32) << 16), v);
        if (m < args.NQ) {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int n = n0 + j;
            if (n < m) Pk[(int64_t)m + (int64_t)n * args.ldPi] = (double)v[j];
            else if (n == m) Pk[(int64_t)m + (int64_t)n * args.ldPi] = dm;
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[b]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, kTmemCols);
  }
}
}  // namespace

cudaError_t launch_syrk_split_bf16(const CUtensorMap* tmA_hi, const CUtensorMap* tmA_lo, const CUtensorMap* tmB_hi,
                                   const CUtensorMap* tmB_lo, const SyrkTcArgs& a, int num_sms,
                                   cudaStream_t stream) {
  const int ntm = (a.NQ + TM - 1) / TM;
  const int ntn = (a.NQ + TN - 1) / TN;
  int nblocks = 0;
  for (int tn = 0; tn < ntn; ++tn) nblocks += (ntm - 2 * tn > 0) ? (ntm - 2 * tn) : 0;
  const int nunits = nblocks * a.kg;
  const int nchunks = (int)((a.nov + TK - 1) / TK);
  if (nunits == 0 || nchunks == 0) return cudaSuccess;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e =
        cudaFuncSetAttribute(syrk_split_bf16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  const int grid = nunits < num_sms ? nunits : num_sms;
  syrk_split_bf16_kernel<<<grid, kThreads, kSmemBytes, stream>>>(*tmA_hi, *tmA_lo, *tmB_hi, *tmB_lo, a, nblocks,
                                                                  ntm, nunits, nchunks);
  ++g_launches;
  return cudaGetLastError();
}

}  // namespace rpa
