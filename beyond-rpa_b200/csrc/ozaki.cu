// FP64-accurate trailing updates of the blocked Cholesky on the int8 tensor cores.
//
// The log-det of 1 + Pi(u) is an FP64 Cholesky whose cost is the rank-nb2 trailing updates
//   C(r, c) -= sum_k P(r, k) P(c, k),   r >= c,
// with P the just-factored column panel (nb2 = 256 columns).  On DMMA these run near the FP64
// peak (~35 TFLOP/s on B200).  Here they can run as exact integer products on tcgen05 (kind::i8),
// the splitting scheme of Ozaki, Ogita, Oishi and Rump (Numer. Algorithms 59, 2012) with
// integer slices (Ootomo, Ozaki and Yokota, IJHPCA 2024):
//
//  * slicing (ozaki_slice_kernel): every row r of P gets an exponent e_r with
//    max_k |P(r, k)| < 2^e_r and S signed digits d_{r,s,k} in [-64, 64] taken by round-to-nearest,
//      P(r, k) = 2^(e_r - 6) * sum_{s<S} d_{r,s,k} 2^(-7 s)  +  (remainder < 2^(e_r - 7 S)),
//    all exact in FP64 (scalings by powers of two, remainders of rint);
//  * products (ozaki_syrk_kernel): for each 128 x 64 tile of C and each digit pair (s, t) with
//    s + t < S, one int8 MMA per 32 k adds D_s D_t^T into the int32 TMEM accumulator of group
//    g = s + t (S groups x 64 columns <= 512 TMEM columns).  |d| <= 64 and k <= 512 keep every
//    group sum below 2^31: the products are exact;
//  * epilogue: v = sum_g ACC_g 2^(-7 g) in FP64 (Horner from the smallest group), and
//    C(r, c) -= v 2^(e_r + e_c - 12) for r >= c, read-ahead of the C fragment as in the DMMA path.
//
// Dropped pairs (s + t >= S) and the digit remainders leave a relative error of about
// S 2^(-7 S) of |P(r)|_max |P(c)|_max per product: 1.2e-14 for S = 7, 1.5e-16 for S = 8.
//
// Kernel roles (persistent, one CTA per SM, 320 threads): warp 0 issues the TMA loads of the
// digit planes (one 3-D box of all S planes per operand and 64-wide k chunk), warp 1 owns TMEM
// and issues the MMAs from one lane, warps 2..9 drain TMEM.  Every wait is bounded.
#include <cstdlib>

#include "kernels.h"

namespace rpa {

namespace {
constexpr int OZ_TM = 128;      // rows of C per tile (TMEM lanes)
constexpr int OZ_TN = 64;       // columns of C per tile (TMEM columns per digit group)
constexpr int OZ_TK = 64;       // k bytes per stage (one 64-byte swizzle row)
constexpr int OZ_STAGES = 2;
constexpr int OZ_THREADS = 320;  // producer, MMA issuer, 8 epilogue warps
constexpr uint32_t OZ_TMEM_COLS = 512;

template <int S>
struct OzShape {
  static constexpr int kABytes = S * OZ_TM * OZ_TK;
  static constexpr int kBBytes = S * OZ_TN * OZ_TK;
  static constexpr int kStageBytes = kABytes + kBBytes;
  static constexpr int kSmem = OZ_STAGES * kStageBytes + 1024 + 256;
  static_assert(S * OZ_TN <= (int)OZ_TMEM_COLS, "one TMEM accumulator of 64 columns per digit group");
};

// Instruction descriptor: kind::i8, A = B = signed 8-bit, D = signed 32-bit, both K-major, M x N.
constexpr uint32_t umma_idesc_s8_s32(int M, int N) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tc_mma_s8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// 32 lanes x 32 consecutive 32-bit TMEM columns per warp, as signed integers.
__device__ __forceinline__ void tmem_ld_s32_x32(uint32_t taddr, int* v) {
  float f[32];
  tmem_ld_32x32b_x32(taddr, f);  // load + wait::ld
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __float_as_int(f[i]);
}

// 4-D tiled bulk tensor load global -> shared (dims: 64 k bytes, rows, k chunk, plane); the box
// spans all S digit planes of one k chunk: S contiguous (rows x 64 B) tiles in shared memory.
__device__ __forceinline__ void tma_load_planes(void* dst, const void* tmap, uint64_t* bar, int row, int kc,
                                                int plane0) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(0), "r"(row), "r"(kc), "r"(plane0), "r"(smem_u32(bar))
      : "memory");
}

// 2^e as a double for |e| < 1022 (exponent field arithmetic; exact)
__device__ __forceinline__ double pow2i(int e) { return __longlong_as_double((long long)(1023 + e) << 52); }

// ---------------------------------------------------------------- slicing
// Rows r0 .. n-1 of the panel P = A(:, c0 .. c0 + K - 1) of every matrix: exponents and S digit
// planes.  Block: 256 threads = 8 warps over 32 rows; warp w handles columns 32 w .. of every
// 256-column group of the panel, lane l the row r0 + 32 blockIdx.x + l.
template <int S>
__global__ void __launch_bounds__(256) ozaki_slice_kernel(const double* __restrict__ A, int64_t ld, int64_t stride,
                                                          int n, int r0, int c0, int K, int8_t* __restrict__ slices,
                                                          int* __restrict__ expo) {
  __shared__ double red[8][32];
  const int z = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = r0 + blockIdx.x * 32 + lane;
  const double* Az = A + (int64_t)z * stride;
  double m = 0.0;
  for (int c = warp; c < K; c += 8) m = fmax(m, r < n ? fabs(Az[r + ld * (int64_t)(c0 + c)]) : 0.0);
  red[warp][lane] = m;
  __syncthreads();
  m = 0.0;
#pragma unroll
  for (int w = 0; w < 8; ++w) m = fmax(m, red[w][lane]);
  int e = 0;
  if (m > 0.0) frexp(m, &e);  // m = f 2^e, 0.5 <= f < 1: every |P(r, k)| < 2^e
  if (warp == 0 && r < n) expo[(int64_t)z * n + r] = e;
  if (r >= n) return;
  const double scale = pow2i(6 - e);
  // warp w: 32-column groups g = w, w + 8, ...; 32 digits per plane -> two 16-byte stores
  for (int c = 32 * warp; c < K; c += 256) {
    double y[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) y[j] = (c + j < K) ? Az[r + ld * (int64_t)(c0 + c + j)] * scale : 0.0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
      uint32_t wd[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        uint32_t packed = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const double d = rint(y[4 * q + b]);
          y[4 * q + b] = (y[4 * q + b] - d) * 128.0;
          packed |= ((uint32_t)((int)d & 0xFF)) << (8 * b);
        }
        wd[q] = packed;
      }
      // layout [z][s][k chunk][row][64 k]: every (plane, chunk) is a contiguous array of 64-byte rows
      int8_t* dst = slices + ((((int64_t)z * S + s) * (K / OZ_TK) + c / OZ_TK) * n + r) * OZ_TK + c % OZ_TK;
      *reinterpret_cast<uint4*>(dst) = make_uint4(wd[0], wd[1], wd[2], wd[3]);
      *reinterpret_cast<uint4*>(dst + 16) = make_uint4(wd[4], wd[5], wd[6], wd[7]);
    }
  }
}

// ---------------------------------------------------------------- products
struct OzUpdate {
  double* A;  // matrices (column-major, ld, stride); C is the block below
  int64_t ld, stride;
  int n, nmat;
  int row0, col0;     // C block: rows row0 .., columns col0 .. (global indices)
  int nrows, ncols;
  int nchunks;        // K / 64
  const int* expo;    // [z][n]
  int ntm, ntn, nunits;
};

__device__ __forceinline__ bool unit_live(const OzUpdate& u, int tm, int tn) {
  // the tile holds a lower-triangle entry of C iff its last row is at or below its first column
  return u.row0 + tm * OZ_TM + OZ_TM - 1 >= u.col0 + tn * OZ_TN;
}

template <int S>
__global__ void __launch_bounds__(OZ_THREADS, 1)
    ozaki_syrk_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      const OzUpdate u, int* err) {
  using Sh = OzShape<S>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + OZ_STAGES * Sh::kStageBytes);
  uint64_t* empty = full + OZ_STAGES;
  uint64_t* acc_full = empty + OZ_STAGES;
  uint64_t* acc_empty = acc_full + 1;
  uint64_t* drain = acc_empty + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < OZ_STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, 8);
    mbar_init(drain, 1);
    fence_mbar_init();
  }
  if (warp == 1) tmem_alloc(tmem_slot, OZ_TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  auto a_tile = [&](int st) { return smem + st * Sh::kStageBytes; };
  auto b_tile = [&](int st) { return smem + st * Sh::kStageBytes + Sh::kABytes; };

  if (warp == 0) {
    if (lane == 0) {
      // ------------------------------------------------------------ producer
      tma_prefetch_desc(&tmA);
      tma_prefetch_desc(&tmB);
      int stage = 0;
      uint32_t phase = 0, issued = 0, issued_par = 0;
      bool ok = true;
      for (int w = blockIdx.x; w < u.nunits && ok; w += gridDim.x) {
        const int z = w / (u.ntm * u.ntn), rem = w - z * u.ntm * u.ntn;
        const int tm = rem / u.ntn, tn = rem - tm * u.ntn;
        if (!unit_live(u, tm, tn)) continue;
        for (int ch = 0; ch < u.nchunks; ++ch) {
          if (!mbar_wait(&empty[stage], phase ^ 1u, err, kDevTimeoutTmaEmpty)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&full[stage], Sh::kStageBytes);
          tma_load_planes(a_tile(stage), &tmA, &full[stage], u.row0 + tm * OZ_TM, ch, z * S);
          tma_load_planes(b_tile(stage), &tmB, &full[stage], u.col0 + tn * OZ_TN, ch, z * S);
          issued |= 1u << stage;
          issued_par = (issued_par & ~(1u << stage)) | (phase << stage);
          if (++stage == OZ_STAGES) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      for (int s = 0; s < OZ_STAGES; ++s)
        if (issued & (1u << s)) mbar_wait(&full[s], (issued_par >> s) & 1u, err, kDevTimeoutDrain);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ------------------------------------------------------------ MMA issuer
      constexpr uint32_t idesc = umma_idesc_s8_s32(OZ_TM, OZ_TN);
      int stage = 0;
      uint32_t phase = 0, acc_phase = 0;
      bool ok = true;
      for (int w = blockIdx.x; w < u.nunits && ok; w += gridDim.x) {
        const int rem = w % (u.ntm * u.ntn);
        const int tm = rem / u.ntn, tn = rem - tm * u.ntn;
        if (!unit_live(u, tm, tn)) continue;
        if (!mbar_wait(acc_empty, acc_phase ^ 1u, err, kDevTimeoutAccEmpty)) break;
        tc_fence_after();
        for (int ch = 0; ch < u.nchunks; ++ch) {
          if (!mbar_wait(&full[stage], phase, err, kDevTimeoutTmaFull)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a0 = smem_u32(a_tile(stage)), b0 = smem_u32(b_tile(stage));
#pragma unroll
          for (int kk = 0; kk < OZ_TK / 32; ++kk) {
#pragma unroll
            for (int s = 0; s < S; ++s) {
              const uint64_t da = umma_desc_k_sw64(a0 + (uint32_t)(s * OZ_TM * OZ_TK + kk * 32));
#pragma unroll
              for (int t = 0; t < S - s; ++t) {
                const uint64_t db = umma_desc_k_sw64(b0 + (uint32_t)(t * OZ_TN * OZ_TK + kk * 32));
                // group g = s + t; its first product of the unit (ch = kk = s = 0) overwrites
                tc_mma_s8(tmem_base + (uint32_t)((s + t) * OZ_TN), da, db, idesc,
                          (ch > 0 || kk > 0 || s > 0) ? 1u : 0u);
              }
            }
          }
          tc_commit(&empty[stage]);
          if (++stage == OZ_STAGES) {
            stage = 0;
            phase ^= 1u;
          }
        }
        if (!ok) break;
        tc_commit(acc_full);
        acc_phase ^= 1u;
      }
      tc_commit(drain);
      mbar_wait(drain, 0, err, kDevTimeoutDrain);
    }
  } else {
    // -------------------------------------------------------------- epilogue (warps 2..9)
    // warp w reads TMEM lanes 32 (w mod 4) .. + 31 (its rows) and the column half (w - 2) / 4 of the
    // tile: 32 columns.  The C fragment is read before the accumulator is ready (under the MMAs);
    // TMEM is released once the 32 x 32 block of every digit group has been read.
    const int quarter = warp & 3;
    const int half = (warp - 2) >> 2;
    const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
    uint32_t acc_phase = 0;
    for (int w = blockIdx.x; w < u.nunits; w += gridDim.x) {
      const int z = w / (u.ntm * u.ntn), rem = w - z * u.ntm * u.ntn;
      const int tm = rem / u.ntn, tn = rem - tm * u.ntn;
      if (!unit_live(u, tm, tn)) continue;
      const int r = u.row0 + tm * OZ_TM + quarter * 32 + lane;
      const int c0 = u.col0 + tn * OZ_TN + half * 32;
      const bool row_ok = r < u.row0 + u.nrows;
      double* Cz = u.A + (int64_t)z * u.stride;
      double old[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const bool live = row_ok && c0 + j < u.col0 + u.ncols && r >= c0 + j;
        old[j] = live ? Cz[r + u.ld * (int64_t)(c0 + j)] : 0.0;
      }
      const int er = row_ok ? u.expo[(int64_t)z * u.n + r] : 0;
      if (!mbar_wait(acc_full, acc_phase, err, kDevTimeoutAccFull)) break;
      acc_phase ^= 1u;
      tc_fence_after();
      double v[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] = 0.0;
#pragma unroll
      for (int g = S - 1; g >= 0; --g) {  // Horner over the digit groups, smallest weight first
        int acc[32];
        tmem_ld_s32_x32(tmem_base + lane_addr + (uint32_t)(g * OZ_TN + half * 32), acc);
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = fma(v[j], 1.0 / 128.0, (double)acc[j]);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acc_empty);
      if (row_ok) {
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int c = c0 + j;
          if (c < u.col0 + u.ncols && r >= c) {
            const int ex = er + __ldg(u.expo + (int64_t)z * u.n + c) - 12;
            // below 2^-1000 the update is far under the rounding of C
            Cz[r + u.ld * (int64_t)c] = old[j] - (ex < -1000 ? 0.0 : v[j] * pow2i(ex));
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, OZ_TMEM_COLS);
  }
}

template <int S>
cudaError_t launch_update_s(const OzakiWork& w, int buf, double* A, int64_t ld, int64_t stride, int n, int nmat,
                            int row0, int col0, int nrows, int ncols, int* err, int num_sms, cudaStream_t stream) {
  OzUpdate u;
  u.A = A;
  u.ld = ld;
  u.stride = stride;
  u.n = n;
  u.nmat = nmat;
  u.row0 = row0;
  u.col0 = col0;
  u.nrows = nrows;
  u.ncols = ncols;
  u.nchunks = w.K / OZ_TK;
  u.expo = w.expo[buf];
  u.ntm = (nrows + OZ_TM - 1) / OZ_TM;
  u.ntn = (ncols + OZ_TN - 1) / OZ_TN;
  const int64_t units = (int64_t)u.ntm * u.ntn * nmat;
  if (units == 0) return cudaSuccess;
  if (units > INT32_MAX) return cudaErrorInvalidValue;
  u.nunits = (int)units;
  int live = 0;
  for (int tm = 0; tm < u.ntm; ++tm)
    for (int tn = 0; tn < u.ntn; ++tn) live += u.row0 + tm * OZ_TM + OZ_TM - 1 >= u.col0 + tn * OZ_TN;
  const int64_t live_units = (int64_t)live * nmat;
  const int grid = (int)(live_units < num_sms ? live_units : num_sms);
  if (grid <= 0) return cudaSuccess;
  const int smem = OzShape<S>::kSmem;
  cudaError_t e = cudaFuncSetAttribute(ozaki_syrk_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  ozaki_syrk_kernel<S><<<grid, OZ_THREADS, smem, stream>>>(w.mapA[buf], w.mapB[buf], u, err);
  ++g_launches;
  return cudaGetLastError();
}
}  // namespace

// Off by default: at order 4096 the int8 updates give E(u) bit-identical to the DMMA updates but
// take longer (log-det 15.7 vs 14.7 ms for 16 matrices on B200).  With S = 7 digit groups the
// 512 TMEM columns allow N = 64 per MMA, and 128 x 64 x 32 int8 MMAs ran at about a quarter of the
// int8 peak (the 28 pair products of a tile take ~125 cycles each); the FP64 read-modify-write of
// C adds the same traffic as the DMMA path.  RPA_B200_OZAKI_SLICES = 7 or 8 turns them on.
int ozaki_slices_default() {
  const char* e = std::getenv("RPA_B200_OZAKI_SLICES");
  const int v = e ? std::atoi(e) : 0;
  return (v == 7 || v == 8) ? v : 0;
}

size_t ozaki_buffer_bytes(int n, int nmat, int K, int S) {
  return (size_t)S * nmat * n * K + 256 + ((size_t)nmat * n * sizeof(int) + 255) / 256 * 256;
}

cudaError_t ozaki_setup(OzakiWork& w, PFN_cuTensorMapEncodeTiled_v12000 encode, void* const buf[2], int n, int nmat,
                        int K, int S) {
  if ((S != 7 && S != 8) || K % OZ_TK != 0 || K > 512 || n < 1 || nmat < 1) return cudaErrorInvalidValue;
  w.S = S;
  w.K = K;
  const size_t slice_bytes = (size_t)S * nmat * n * K;
  for (int b = 0; b < 2; ++b) {
    uint8_t* base = static_cast<uint8_t*>(buf[b]);
    w.slices[b] = reinterpret_cast<int8_t*>(base);
    w.expo[b] = reinterpret_cast<int*>(base + (slice_bytes + 255) / 256 * 256);
    const cuuint64_t nkc = (cuuint64_t)(K / OZ_TK);
    cuuint64_t dims[4] = {(cuuint64_t)OZ_TK, (cuuint64_t)n, nkc, (cuuint64_t)nmat * S};
    cuuint64_t strides[3] = {(cuuint64_t)OZ_TK, (cuuint64_t)OZ_TK * n, (cuuint64_t)OZ_TK * n * nkc};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    cuuint32_t boxA[4] = {OZ_TK, OZ_TM, 1, (cuuint32_t)S};
    cuuint32_t boxB[4] = {OZ_TK, OZ_TN, 1, (cuuint32_t)S};
    if (encode(&w.mapA[b], CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, base, dims, strides, boxA, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS ||
        encode(&w.mapB[b], CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, base, dims, strides, boxB, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return cudaErrorInvalidValue;
  }
  return cudaSuccess;
}

cudaError_t launch_ozaki_slices(const OzakiWork& w, int buf, const double* A, int64_t ld, int64_t stride, int n,
                                int nmat, int r0, int c0, cudaStream_t stream) {
  if (r0 >= n) return cudaSuccess;
  dim3 grid((unsigned)((n - r0 + 31) / 32), (unsigned)nmat);
  if (w.S == 8)
    ozaki_slice_kernel<8><<<grid, 256, 0, stream>>>(A, ld, stride, n, r0, c0, w.K, w.slices[buf], w.expo[buf]);
  else
    ozaki_slice_kernel<7><<<grid, 256, 0, stream>>>(A, ld, stride, n, r0, c0, w.K, w.slices[buf], w.expo[buf]);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_ozaki_update(const OzakiWork& w, int buf, double* A, int64_t ld, int64_t stride, int n, int nmat,
                                int row0, int col0, int nrows, int ncols, int* err, int num_sms, cudaStream_t stream) {
  if (nrows <= 0 || ncols <= 0) return cudaSuccess;
  return w.S == 8 ? launch_update_s<8>(w, buf, A, ld, stride, n, nmat, row0, col0, nrows, ncols, err, num_sms, stream)
                  : launch_update_s<7>(w, buf, A, ld, stride, n, nmat, row0, col0, nrows, ncols, err, num_sms, stream);
}

}  // namespace rpa
