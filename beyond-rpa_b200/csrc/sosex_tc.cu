// Split-BF16 SOSEX pair contraction on the 5th-generation tensor cores
// (rpa_CC_Exchange_SOSEX + rpa_CC_EcExchange1, src/rpa/rpa_CC_Exchange.f90:36-116):
//
//   E_x = -alpha * sum_{i>=j} (2 - delta_ij) sum_{Q,mu} B_mu W_ij(Q,mu) W_ji(Q,mu),
//   W_ij = R_i U_j^T,  R_i = R(:, nv*i .. nv*i+nv-1),  U_j = U(nv*j .. nv*j+nv-1, :),
//
// and the Tr(XK) contraction of the MBPT3 exchange (W_ji from U2 = U X, B = 1).
// R and U are split once into bf16 pairs (R = Rh + Rl, U = Uh + Ul), stored
// K-major (one row per Q or mu, the virtual index contiguous) with every
// occupied block padded to nvp (a multiple of 32) columns of zeros, so that a
// TMA box of 32 columns never straddles two occupied orbitals and every x
// coordinate is a multiple of 32 elements (64 B).  Then
//   W ~= Rh Uh^T + Rh Ul^T + Rl Uh^T       (three BF16 products, FP32 accumulate)
// with the products of one 128 x 128 (Q, mu) tile of W_ij and of W_ji in
// two TMEM accumulators.  The tensor-core accumulator rounds toward zero, so
// the virtual index is cut into segments of seg_chunks x 32 columns, each
// accumulated afresh and added in IEEE FP32 registers by the epilogue (the
// bias of one accumulator grows with the number of additions it takes).
// The epilogue forms sum_mu B_mu W_ij W_ji in FP64 and writes one partial per
// epilogue warp and unit (reduced in a fixed order afterwards: deterministic).
//
// Persistent kernel, one CTA per SM, 576 threads:
//   warp 0      TMA producer (one elected lane)
//   warp 1      TMEM allocator + MMA issuer (one elected lane)
//   warps 2..17 epilogue (warp w: TMEM lanes 32*(w%4).., 32 accumulator columns)
// Work unit = (pair i >= j, 128-row Q tile, 128-column mu tile), pair-major,
// so the CTAs of one wave share the pair's operand tiles in L2.
// Smem pipeline: 3 stages of {Ri_hi, Ri_lo, Uj_hi, Uj_lo, Rj_hi, Rj_lo, Ui_hi,
// Ui_lo}, each 128 x 32 bf16 with 64-byte swizzle (the diagonal pairs of SOSEX
// need only the first four).
#include <algorithm>

#include "kernels.h"

namespace rpa {

namespace {
constexpr int TM = 128, TN = 128, TK = 32;
constexpr int kStages = 3;
constexpr int kTile = TM * TK * 2;        // 8 KB
constexpr int kStageBytes = 8 * kTile;    // 64 KB
constexpr int kThreads = 576;
constexpr int kEpiWarps = 16;
constexpr int kEpiCols = TN / 4;          // 32 accumulator columns per epilogue warp
constexpr uint32_t kTmemCols = 512;       // 2 buffers x (W_ij, W_ji) x 128 columns
constexpr uint32_t kIdesc = umma_idesc_bf16_f32(TM, TN);
constexpr int kSmemBytes = kStages * kStageBytes + 1024 /*align slack*/ + 256 /*barriers*/;

__device__ __forceinline__ void pair_of(int p, int& i, int& j) {
  // p enumerates (i, j) with i >= j: p = i*(i+1)/2 + j
  int t = (int)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
  while ((t + 1) * (t + 2) / 2 <= p) ++t;
  while (t * (t + 1) / 2 > p) --t;
  i = t;
  j = p - t * (t + 1) / 2;
}

struct PairUnit {
  int i, j, qt, mt;
  bool diag;  // W_ii W_ii: one accumulator, four operand tiles
};

__device__ __forceinline__ PairUnit unit_of(int u, const SosexTcArgs& a) {
  PairUnit x;
  const int per = a.nqt * a.nmt;
  const int p = u / per;
  const int r = u - p * per;
  pair_of(p, x.i, x.j);
  x.qt = r / a.nmt;
  x.mt = r - x.qt * a.nmt;
  x.diag = (x.i == x.j) && a.same;
  return x;
}

__global__ void __launch_bounds__(kThreads, 1)
    sosex_split_bf16_kernel(const __grid_constant__ CUtensorMap tRh, const __grid_constant__ CUtensorMap tRl,
                            const __grid_constant__ CUtensorMap tUh, const __grid_constant__ CUtensorMap tUl,
                            const __grid_constant__ CUtensorMap tU2h, const __grid_constant__ CUtensorMap tU2l,
                            const SosexTcArgs a) {
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
  const int nch = a.nvp / TK;
  const int seg = a.seg_chunks > 0 ? a.seg_chunks : nch;

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

  // tile t of stage s: 0 Ri_hi, 1 Ri_lo, 2 Uj_hi, 3 Uj_lo, 4 Rj_hi, 5 Rj_lo, 6 Ui_hi, 7 Ui_lo
  auto tile = [&](int s, int t) { return smem + s * kStageBytes + t * kTile; };

  if (warp == 0) {
    if (lane == 0) {
      // ------------------------------------------------------------ producer
      for (const CUtensorMap* m : {&tRh, &tRl, &tUh, &tUl, &tU2h, &tU2l}) tma_prefetch_desc(m);
      int stage = 0;
      uint32_t phase = 0;
      uint32_t issued = 0, issued_par = 0;
      bool ok = true;
      for (int u = blockIdx.x; u < a.nunits && ok; u += gridDim.x) {
        const PairUnit x = unit_of(u, a);
        const int q0 = x.qt * TM, m0 = x.mt * TN;
        for (int c = 0; c < nch; ++c) {
          if (!mbar_wait(&empty[stage], phase ^ 1u, a.err, kDevTimeoutTmaEmpty)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&full[stage], (x.diag ? 4 : 8) * kTile);
          const int ci = x.i * a.nvp + c * TK, cj = x.j * a.nvp + c * TK;
          tma_load_3d(tile(stage, 0), &tRh, &full[stage], ci, q0, 0);
          tma_load_3d(tile(stage, 1), &tRl, &full[stage], ci, q0, 0);
          tma_load_3d(tile(stage, 2), &tUh, &full[stage], cj, m0, 0);
          tma_load_3d(tile(stage, 3), &tUl, &full[stage], cj, m0, 0);
          if (!x.diag) {
            tma_load_3d(tile(stage, 4), &tRh, &full[stage], cj, q0, 0);
            tma_load_3d(tile(stage, 5), &tRl, &full[stage], cj, q0, 0);
            tma_load_3d(tile(stage, 6), &tU2h, &full[stage], ci, m0, 0);
            tma_load_3d(tile(stage, 7), &tU2l, &full[stage], ci, m0, 0);
          }
          issued |= 1u << stage;
          issued_par = (issued_par & ~(1u << stage)) | (phase << stage);
          if (++stage == kStages) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      // no bulk copy may still be landing in shared memory at exit
      for (int s = 0; s < kStages; ++s)
        if (issued & (1u << s)) mbar_wait(&full[s], (issued_par >> s) & 1u, a.err, kDevTimeoutDrain);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ------------------------------------------------------------ MMA issuer
      int stage = 0;
      uint32_t phase = 0;
      int it = 0;  // segment counter (selects the TMEM buffer)
      bool ok = true;
      for (int u = blockIdx.x; u < a.nunits && ok; u += gridDim.x) {
        const PairUnit x = unit_of(u, a);
        for (int c0 = 0; c0 < nch && ok; c0 += seg, ++it) {
          const int b = it & 1;
          const uint32_t acc_phase = (uint32_t)((it >> 1) & 1);
          if (!mbar_wait(&acc_empty[b], acc_phase ^ 1u, a.err, kDevTimeoutAccEmpty)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d1 = tmem_base + (uint32_t)(b * 2 * TN), d2 = d1 + (uint32_t)TN;
          const int c1 = min(nch, c0 + seg);
          for (int ch = c0; ch < c1; ++ch) {
            if (!mbar_wait(&full[stage], phase, a.err, kDevTimeoutTmaFull)) {
              ok = false;
              break;
            }
            tc_fence_after();
#pragma unroll
            for (int kk = 0; kk < TK / 16; ++kk) {
              const uint32_t off = (uint32_t)(kk * 32);  // 16 bf16 = 32 bytes along K
              const uint32_t acc = (ch > c0 || kk > 0) ? 1u : 0u;
              const uint64_t rih = umma_desc_k_sw64(smem_u32(tile(stage, 0)) + off);
              const uint64_t ril = umma_desc_k_sw64(smem_u32(tile(stage, 1)) + off);
              const uint64_t ujh = umma_desc_k_sw64(smem_u32(tile(stage, 2)) + off);
              const uint64_t ujl = umma_desc_k_sw64(smem_u32(tile(stage, 3)) + off);
              tc_mma_bf16(d1, rih, ujh, kIdesc, acc);
              tc_mma_bf16(d1, rih, ujl, kIdesc, 1u);
              tc_mma_bf16(d1, ril, ujh, kIdesc, 1u);
              if (!x.diag) {
                const uint64_t rjh = umma_desc_k_sw64(smem_u32(tile(stage, 4)) + off);
                const uint64_t rjl = umma_desc_k_sw64(smem_u32(tile(stage, 5)) + off);
                const uint64_t uih = umma_desc_k_sw64(smem_u32(tile(stage, 6)) + off);
                const uint64_t uil = umma_desc_k_sw64(smem_u32(tile(stage, 7)) + off);
                tc_mma_bf16(d2, rjh, uih, kIdesc, acc);
                tc_mma_bf16(d2, rjh, uil, kIdesc, 1u);
                tc_mma_bf16(d2, rjl, uih, kIdesc, 1u);
              }
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
      // every issued MMA must complete before TMEM is freed
      tc_commit(drain);
      mbar_wait(drain, 0, a.err, kDevTimeoutDrain);
    }
  } else {
    // -------------------------------------------------------------- epilogue
    const int quarter = warp & 3;      // TMEM lanes quarter*32 .. +31
    const int colq = (warp - 2) >> 2;  // accumulator columns colq*32 .. +31
    const int ew = warp - 2;
    int it = 0;
    bool ok = true;
    float r1[kEpiCols], r2[kEpiCols];
    for (int u = blockIdx.x; u < a.nunits && ok; u += gridDim.x) {
      const PairUnit x = unit_of(u, a);
      for (int c0 = 0; c0 < nch; c0 += seg, ++it) {
        const int b = it & 1;
        const uint32_t acc_phase = (uint32_t)((it >> 1) & 1);
        if (!mbar_wait(&acc_full[b], acc_phase, a.err, kDevTimeoutAccFull)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t t1 =
            tmem_base + (uint32_t)(b * 2 * TN + colq * kEpiCols) + ((uint32_t)(quarter * 32) << 16);
#pragma unroll
        for (int cc = 0; cc < kEpiCols / 8; ++cc) tmem_ld_add_x8(t1 + (uint32_t)(cc * 8), &r1[cc * 8], c0 == 0);
        if (!x.diag) {
#pragma unroll
          for (int cc = 0; cc < kEpiCols / 8; ++cc)
            tmem_ld_add_x8(t1 + (uint32_t)(TN + cc * 8), &r2[cc * 8], c0 == 0);
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&acc_empty[b]);
      }
      if (!ok) break;
      // Hadamard reduction in FP64 (rows beyond NQ and columns beyond NT hold zeros)
      double s = 0.0;
      const int mbase = x.mt * TN + colq * kEpiCols;
#pragma unroll
      for (int c = 0; c < kEpiCols; ++c) {
        const int mu = mbase + c;
        const double bm = mu < a.NT ? a.Bmu[mu] : 0.0;
        const double w1 = (double)r1[c];
        s += bm * w1 * (x.diag ? w1 : (double)r2[c]);
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
      if (lane == 0) a.partial[(int64_t)u * kEpiWarps + ew] = (x.i == x.j ? 1.0 : 2.0) * s;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, kTmemCols);
  }
}

// R (NQ x nov, column-major, ld) -> Xh/Xl rows q of P = no*nvp bf16: column a + nv*i goes to
// i*nvp + a (the padding is zeroed by the caller).  32 x 32 tiles transposed through shared memory.
__global__ void __launch_bounds__(256) split_rows_kernel(const double* __restrict__ R, int64_t ldR, int NQ, int nv,
                                                         int64_t nov, int nvp, int64_t P, __nv_bfloat16* Xh,
                                                         __nv_bfloat16* Xl) {
  __shared__ double t[32][33];
  const int64_t ai0 = (int64_t)blockIdx.x * 32;
  const int q0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int r = ty; r < 32; r += 8) {
    const int64_t ai = ai0 + r;
    const int q = q0 + tx;
    t[r][tx] = (ai < nov && q < NQ) ? R[(int64_t)q + ldR * ai] : 0.0;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int q = q0 + r;
    const int64_t ai = ai0 + tx;
    if (q < NQ && ai < nov) {
      const float f = (float)t[tx][r];
      const __nv_bfloat16 hi = __float2bfloat16_rn(f);
      const int64_t i = ai / nv, av = ai - i * nv;
      const int64_t dst = (int64_t)q * P + i * nvp + av;
      Xh[dst] = hi;
      Xl[dst] = __float2bfloat16_rn(f - __bfloat162float(hi));
    }
  }
}

// U (nov x NT, column-major, ld) -> Xh/Xl rows mu of P bf16 with the same padding.
__global__ void __launch_bounds__(256) split_cols_kernel(const double* __restrict__ U, int64_t ldU, int NT, int nv,
                                                         int64_t nov, int nvp, int64_t P, __nv_bfloat16* Xh,
                                                         __nv_bfloat16* Xl) {
  const int64_t ai = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (ai >= nov) return;
  const int64_t i = ai / nv, av = ai - i * nv;
  for (int64_t mu = blockIdx.y; mu < NT; mu += gridDim.y) {
    const float f = (float)U[ai + ldU * mu];
    const __nv_bfloat16 hi = __float2bfloat16_rn(f);
    const int64_t dst = mu * P + i * nvp + av;
    Xh[dst] = hi;
    Xl[dst] = __float2bfloat16_rn(f - __bfloat162float(hi));
  }
}

// Fixed-order block sums: out[b] = sum of x[b*chunk .. (b+1)*chunk) (tree order, blockDim 256).
__global__ void __launch_bounds__(256) chunk_sum_kernel(const double* __restrict__ x, int64_t n, int64_t chunk,
                                                        double* out) {
  __shared__ double sh[256];
  const int64_t b0 = (int64_t)blockIdx.x * chunk, b1 = min(n, b0 + chunk);
  double s = 0.0;
  for (int64_t k = b0 + threadIdx.x; k < b1; k += 256) s += x[k];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}
}  // namespace

int sosex_tc_nvp(int nv) { return (nv + TK - 1) / TK * TK; }

int64_t sosex_tc_units(int NQ, int no, int NT) {
  return (int64_t)no * (no + 1) / 2 * ((NQ + TM - 1) / TM) * ((NT + TN - 1) / TN);
}

int64_t sosex_tc_partials(int NQ, int no, int NT) { return sosex_tc_units(NQ, no, NT) * kEpiWarps; }

cudaError_t launch_split_rows(const double* R, int64_t ldR, int NQ, int no, int nv, __nv_bfloat16* Xh,
                              __nv_bfloat16* Xl, cudaStream_t stream) {
  const int nvp = sosex_tc_nvp(nv);
  const int64_t nov = (int64_t)no * nv, P = (int64_t)no * nvp;
  cudaError_t e = cudaMemsetAsync(Xh, 0, (size_t)NQ * P * 2, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(Xl, 0, (size_t)NQ * P * 2, stream);
  if (e != cudaSuccess) return e;
  split_rows_kernel<<<dim3((unsigned)((nov + 31) / 32), (unsigned)((NQ + 31) / 32)), 256, 0, stream>>>(
      R, ldR, NQ, nv, nov, nvp, P, Xh, Xl);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_split_cols(const double* U, int64_t ldU, int NT, int no, int nv, __nv_bfloat16* Xh,
                              __nv_bfloat16* Xl, cudaStream_t stream) {
  const int nvp = sosex_tc_nvp(nv);
  const int64_t nov = (int64_t)no * nv, P = (int64_t)no * nvp;
  cudaError_t e = cudaMemsetAsync(Xh, 0, (size_t)NT * P * 2, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(Xl, 0, (size_t)NT * P * 2, stream);
  if (e != cudaSuccess) return e;
  split_cols_kernel<<<dim3((unsigned)((nov + 255) / 256), (unsigned)std::min(NT, 65535)), 256, 0, stream>>>(
      U, ldU, NT, nv, nov, nvp, P, Xh, Xl);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_sosex_split_bf16(const CUtensorMap* maps, const SosexTcArgs& a, int num_sms, cudaStream_t stream) {
  if (a.nunits <= 0) return cudaSuccess;
  if (a.nvp <= 0 || a.nvp % TK != 0) return cudaErrorInvalidValue;
  cudaError_t e =
      cudaFuncSetAttribute(sosex_split_bf16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
  if (e != cudaSuccess) return e;
  const int grid = a.nunits < num_sms ? a.nunits : num_sms;
  sosex_split_bf16_kernel<<<grid, kThreads, kSmemBytes, stream>>>(maps[0], maps[1], maps[2], maps[3], maps[4],
                                                                   maps[5], a);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_chunk_sum(const double* x, int64_t n, int64_t chunk, double* out, int64_t* nout,
                             cudaStream_t stream) {
  *nout = n > 0 ? (n + chunk - 1) / chunk : 0;
  if (*nout == 0) return cudaSuccess;
  chunk_sum_kernel<<<(unsigned)*nout, 256, 0, stream>>>(x, n, chunk, out);
  ++g_launches;
  return cudaGetLastError();
}

}  // namespace rpa
