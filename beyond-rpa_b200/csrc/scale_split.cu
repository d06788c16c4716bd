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
//
// The pass is HBM-bound: 8 B read + 4 B written per element and frequency, so
// the writes (hi + lo for every frequency) are ~90 % of the traffic.  They
// leave through the tensor memory accelerator: eight compute warps fill a
// ring of shared-memory stages (one frequency of a 32-row x 128-column tile
// per stage, in the 128-byte swizzled layout of the store's tensor map) and
// one store warp issues bulk tensor stores of each full stage, so no compute
// warp ever waits on a global store or on a CTA-wide barrier per frequency.
// Stage hand-over uses mbarriers (full: 256 compute-thread arrivals; free:
// the store thread, once the bulk store has finished reading the stage);
// every wait is bounded.
#include "kernels.h"

namespace rpa {

namespace {
constexpr int kTQ = 32;                // Q rows per tile: lane l of every compute warp owns row q0 + l
constexpr int kTA = 128;               // ai columns per chunk: two 64-column (128-byte) store boxes
constexpr int kComputeWarps = 8;       // warp w owns the 16 columns 16 w .. 16 w + 15 of a chunk
constexpr int kCols = kTA / kComputeWarps;
constexpr int kComputeThreads = 32 * kComputeWarps;
constexpr int kThreads = kComputeThreads + 32;  // + the store warp
constexpr int kStages = 4;
// bulk-store groups still reading shared memory while the next is issued: a stage is freed as soon
// as the group after it has been committed (1: 4.23-4.31 ms at NQ 4096 / 65536 ai / 16 frequencies;
// 2: 4.28-4.34 ms; 3: 4.74-4.84 ms, each later free stalls the compute warps)
constexpr int kStoreLag = 1;
constexpr int kBoxBytes = kTQ * 128;            // 32 rows x 64 bf16
constexpr int kStageBytes = 4 * kBoxBytes;      // hi box 0, hi box 1, lo box 0, lo box 1
constexpr int kFacBytes = kComputeWarps * kCols * kMaxKgLaunch * 8;
// the diagonal sums of the first kRegAcc frequencies stay in registers, the others in shared memory
// ([warp][k - kRegAcc][lane]): at the 96 registers two CTAs of nine warps allow, this removes most of
// the compute warps' spills (split pass 4.04-4.10 ms against 4.25-4.39 ms with all sums in registers,
// NQ 4096 / 65536 ai / 16 frequencies)
constexpr int kRegAcc = 8;
constexpr int kAccBytes = kComputeWarps * (kMaxKgLaunch - kRegAcc) * 32 * 8;
// smem: stages (1024-byte aligned for the 128-byte swizzle) | per-warp scale factors | mbarriers
constexpr size_t kSplitSmem = 1024 + (size_t)kStages * kStageBytes + kFacBytes + kAccBytes + 2 * kStages * 8;
static_assert(2 * (kSplitSmem + 1024) <= 233472, "two CTAs per SM must fit in shared memory");
static_assert(kComputeWarps * kTQ * kMaxKgLaunch * 8 <= kStages * kStageBytes,
              "the diagonal reduction reuses the stage ring");

__device__ __forceinline__ uint32_t pack_bf162(float a, float b) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ float2 unpack_bf162(uint32_t w) {
  return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xFFFF0000u));
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tma_store_3d(const void* tmap, uint32_t src, int c0, int c1, int c2) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
                   reinterpret_cast<uint64_t>(tmap)),
               "r"(src), "r"(c0), "r"(c1), "r"(c2)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<uint64_t>(p)));
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void named_barrier(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

__device__ __forceinline__ void scale_split_body(const double* __restrict__ R, int64_t ldR, int NQ, int64_t nov,
                                                 const double* __restrict__ D, const FreqGroup& fg, double alpha,
                                                 const CUtensorMap* tm_hi, const CUtensorMap* tm_lo,
                                                 double* __restrict__ diag_part, int64_t ai_per_split, int qtile,
                                                 int split, int* err) {
  extern __shared__ uint8_t dyn_smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(dyn_smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* stages = smem;
  double* fac_all = reinterpret_cast<double*>(smem + kStages * kStageBytes);
  double* acc_all = reinterpret_cast<double*>(smem + kStages * kStageBytes + kFacBytes);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes + kFacBytes + kAccBytes);
  uint64_t* freeb = full + kStages;

  const int t = threadIdx.x;
  const int warp = t >> 5, lane = t & 31;
  const int q0 = qtile * kTQ;
  const int kg = fg.n;
  const int64_t a_begin = (int64_t)split * ai_per_split;
  const int64_t a_end = min(nov, a_begin + ai_per_split);
  const int nchunks = (int)((a_end - a_begin + kTA - 1) / kTA);

  if (t == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], kComputeThreads);
      mbar_init(&freeb[s], 1);
    }
    fence_mbar_init();
  }
  __syncthreads();

  double acc[kRegAcc];
#pragma unroll
  for (int k = 0; k < kRegAcc; ++k) acc[k] = 0.0;
  double* accs = acc_all + (warp < kComputeWarps ? warp : 0) * ((kMaxKgLaunch - kRegAcc) * 32);
  if (warp < kComputeWarps) {
#pragma unroll
    for (int k = 0; k < kMaxKgLaunch - kRegAcc; ++k) accs[k * 32 + lane] = 0.0;
  }

  if (warp < kComputeWarps) {
    const int q = q0 + lane;
    double* fac = fac_all + warp * (kCols * kMaxKgLaunch);  // [k][16 columns], this warp's own
    const uint32_t row_off = (uint32_t)lane * 128u;
    const uint32_t box = (uint32_t)(warp >> 2);                 // columns 0..63 -> box 0, 64..127 -> box 1
    const uint32_t chunk16 = (uint32_t)(2 * (warp & 3));        // first 16-byte chunk of the row in the box
    const uint32_t sw = (uint32_t)(lane & 7);                   // 128-byte swizzle: chunk ^= row mod 8
    const uint32_t off0 = box * kBoxBytes + row_off + (((chunk16 + 0) ^ sw) << 4);
    const uint32_t off1 = box * kBoxBytes + row_off + (((chunk16 + 1) ^ sw) << 4);
    const uint32_t stage0 = smem_u32(stages);
    uint32_t it = 0;
    bool ok = true;
    for (int c = 0; c < nchunks && ok; ++c) {
      const int64_t a0 = a_begin + (int64_t)c * kTA + warp * kCols;
      // R(q, a0 + j): for each j the warp reads 32 consecutive Q of one column (256 bytes).  Issued
      // before the scale-factor arithmetic, whose latency covers part of theirs.
      double r[kCols];
#pragma unroll
      for (int j = 0; j < kCols; ++j) {
        const int64_t a = a0 + j;
        r[j] = (q < NQ && a < a_end) ? __ldg(R + (int64_t)q + ldR * a) : 0.0;
      }
      // scale factors of this warp's 16 columns for every frequency (FP64), into its own slice:
      // sqrt(alpha d / (d^2 + u^2)) = sqrt(alpha d) / sqrt(d^2 + u^2), the first per column (lanes
      // j and j + 16 each take column j), the second one reciprocal square root per (k, j)
      __syncwarp();
      const int jl = lane & (kCols - 1);
      const double dl = (a0 + jl < a_end) ? D[a0 + jl] : 0.0;
      const double sad = sqrt(alpha * dl);
      // lane takes frequencies k = 2m + (lane >> 4); the u_k^2 are picked with constant indexes so
      // that the parameter array is never indexed dynamically (which would copy it to the stack)
#pragma unroll
      for (int m = 0; m < kMaxKgLaunch / 2; ++m) {
        const int k = 2 * m + (lane >> 4);
        const double u2 = (lane >> 4) ? fg.u2[2 * m + 1] : fg.u2[2 * m];
        if (k < kg) fac[k * kCols + jl] = (a0 + jl < a_end) ? sad * rsqrt(fma(dl, dl, u2)) : 0.0;
      }
      // warm L2 with the next chunk's 16 columns (two 128-byte lines each) while this one is split
      {
        const int64_t an = a0 + kTA + (lane & 15);
        const int qn = q0 + 16 * (lane >> 4);
        if (an < a_end && qn < NQ) prefetch_l2(R + (int64_t)qn + ldR * an);
      }
      __syncwarp();
#pragma unroll
      for (int k = 0; k < kMaxKgLaunch; ++k) {
        if (k < kg) {
          const double* fk = fac + k * kCols;
          uint32_t hw[kCols / 2], lw[kCols / 2];
          double s = 0.0;
#pragma unroll
          for (int p = 0; p < kCols / 2; ++p) {
            const double2 f2 = *reinterpret_cast<const double2*>(fk + 2 * p);
            const double x0 = r[2 * p] * f2.x, x1 = r[2 * p + 1] * f2.y;
            s = fma(x0, x0, s);
            s = fma(x1, x1, s);
            // hi = bf16(x), lo = bf16(x - hi); x - hi is exact in FP32
            const float g0 = (float)x0, g1 = (float)x1;
            hw[p] = pack_bf162(g0, g1);
            const float2 hf = unpack_bf162(hw[p]);
            lw[p] = pack_bf162(g0 - hf.x, g1 - hf.y);
          }
          if (k < kRegAcc) acc[k] += s;
          else accs[(k - kRegAcc) * 32 + lane] += s;
          const uint32_t st = it % kStages;
          if (!mbar_wait(&freeb[st], ((it / kStages) & 1u) ^ 1u, err, kDevTimeoutTmaEmpty)) {
            ok = false;
            break;
          }
          const uint32_t base = stage0 + st * kStageBytes;
          st_shared_v4(base + off0, hw[0], hw[1], hw[2], hw[3]);
          st_shared_v4(base + off1, hw[4], hw[5], hw[6], hw[7]);
          st_shared_v4(base + 2 * kBoxBytes + off0, lw[0], lw[1], lw[2], lw[3]);
          st_shared_v4(base + 2 * kBoxBytes + off1, lw[4], lw[5], lw[6], lw[7]);
          fence_proxy_async_smem();  // make the stores visible to the bulk-copy engine
          mbar_arrive(&full[st]);
          ++it;
        }
      }
    }
  } else if (lane == 0) {
    // store thread: one bulk tensor store per 64-column box of each full stage
    tma_prefetch_desc(tm_hi);
    tma_prefetch_desc(tm_lo);
    uint32_t it = 0;
    bool ok = true;
    for (int c = 0; c < nchunks && ok; ++c) {
      const int a0 = (int)(a_begin + (int64_t)c * kTA);
      for (int k = 0; k < kg; ++k) {
        const uint32_t st = it % kStages;
        if (!mbar_wait(&full[st], (it / kStages) & 1u, err, kDevTimeoutTmaFull)) {
          ok = false;
          break;
        }
        const uint32_t base = smem_u32(stages) + st * kStageBytes;
        // a box may run past nov (the map clips it) but never starts past it
        tma_store_3d(tm_hi, base, a0, q0, k);
        tma_store_3d(tm_lo, base + 2 * kBoxBytes, a0, q0, k);
        if (a0 + 64 < nov) {
          tma_store_3d(tm_hi, base + kBoxBytes, a0 + 64, q0, k);
          tma_store_3d(tm_lo, base + 3 * kBoxBytes, a0 + 64, q0, k);
        }
        bulk_commit();
        // a stage may be refilled once the engine has read it: keep kStoreLag groups reading
        if (it >= (uint32_t)kStoreLag) {
          bulk_wait_read<kStoreLag>();
          mbar_arrive(&freeb[(it - kStoreLag) % kStages]);
        }
        ++it;
      }
    }
    bulk_wait_all();
  }
  // every stage has been read by its store (the store thread waited for that before arriving
  // here): reuse the ring for the deterministic reduction of the 8 column owners of each row
  named_barrier(1, kThreads);
  double* red = reinterpret_cast<double*>(stages);  // [w][k][lane]
  if (warp < kComputeWarps) {
#pragma unroll
    for (int k = 0; k < kMaxKgLaunch; ++k)
      if (k < kg) red[(warp * kMaxKgLaunch + k) * 32 + lane] = k < kRegAcc ? acc[k] : accs[(k - kRegAcc) * 32 + lane];
  }
  named_barrier(1, kThreads);
  for (int idx = t; idx < kg * kTQ; idx += kThreads) {
    const int k = idx / kTQ, row = idx % kTQ;
    if (q0 + row < NQ) {
      double sum = 0.0;
#pragma unroll
      for (int w = 0; w < kComputeWarps; ++w) sum += red[(w * kMaxKgLaunch + k) * 32 + row];
      diag_part[((int64_t)split * kg + k) * NQ + q0 + row] = sum;
    }
  }
}

__global__ void __launch_bounds__(kThreads, 2) scale_split_kernel(
    const double* __restrict__ R, int64_t ldR, int NQ, int64_t nov, const double* __restrict__ D, FreqGroup fg,
    double alpha, const __grid_constant__ CUtensorMap tm_hi, const __grid_constant__ CUtensorMap tm_lo,
    double* __restrict__ diag_part, int64_t ai_per_split, int split0, int* err) {
  scale_split_body(R, ldR, NQ, nov, D, fg, alpha, &tm_hi, &tm_lo, diag_part, ai_per_split, blockIdx.x,
                   split0 + (int)blockIdx.y, err);
}

// Many instances in one launch: CTA b handles (instance, q tile, ai split) = work[b].
__global__ void __launch_bounds__(kThreads, 2) scale_split_multi_kernel(const SplitJob* __restrict__ jobs,
                                                                        const int4* __restrict__ work, int* err) {
  const int4 w = work[blockIdx.x];
  const SplitJob& j = jobs[w.x];
  scale_split_body(j.R, j.ldR, j.NQ, j.nov, j.D, j.fg, j.alpha, &j.tm_hi, &j.tm_lo, j.diag_part, j.ai_per_split,
                   w.y, w.z, err);
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

cudaError_t encode_split_store_map(PFN_cuTensorMapEncodeTiled_v12000 encode, CUtensorMap* m, void* base,
                                   int64_t nov, int NQ, int kg, int64_t pitch) {
  cuuint64_t dims[3] = {(cuuint64_t)nov, (cuuint64_t)NQ, (cuuint64_t)kg};
  cuuint64_t strides[2] = {(cuuint64_t)pitch * 2, (cuuint64_t)pitch * 2 * (cuuint64_t)NQ};
  cuuint32_t box[3] = {64, (cuuint32_t)kTQ, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, base, dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t launch_scale_split_multi(const SplitJob* jobs, const int4* work, int nwork, const int64_t* offsets,
                                     int njobs, int64_t total, int* err, cudaStream_t stream) {
  cudaError_t e0 =
      cudaFuncSetAttribute(scale_split_multi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSplitSmem);
  if (e0 != cudaSuccess) return e0;
  if (nwork > 0) {
    scale_split_multi_kernel<<<nwork, kThreads, kSplitSmem, stream>>>(jobs, work, err);
    ++g_launches;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || total == 0) return e;
  diag_reduce_multi_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(jobs, offsets, njobs, total);
  ++g_launches;
  return cudaGetLastError();
}

cudaError_t launch_scale_split(const double* R, int64_t ldR, int NQ, int64_t nov, const double* D,
                               const FreqGroup& fg, double alpha, const CUtensorMap* tm_hi, const CUtensorMap* tm_lo,
                               double* diag_part, double* diag, const SplitPlan& plan, int* err, cudaStream_t stream) {
  cudaError_t e = launch_scale_split_part(R, ldR, NQ, nov, D, fg, alpha, tm_hi, tm_lo, diag_part, plan, 0,
                                          plan.nsplit, err, stream);
  if (e != cudaSuccess) return e;
  return launch_diag_reduce(diag_part, plan, fg.n, NQ, diag, stream);
}

cudaError_t launch_scale_split_part(const double* R, int64_t ldR, int NQ, int64_t nov, const double* D,
                                    const FreqGroup& fg, double alpha, const CUtensorMap* tm_hi,
                                    const CUtensorMap* tm_lo, double* diag_part, const SplitPlan& plan, int split0,
                                    int split1, int* err, cudaStream_t stream) {
  if (split0 < 0 || split1 > plan.nsplit || split1 <= split0) return cudaErrorInvalidValue;
  if (fg.n < 1 || fg.n > kMaxKgLaunch) return cudaErrorInvalidValue;
  cudaError_t e0 = cudaFuncSetAttribute(scale_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSplitSmem);
  if (e0 != cudaSuccess) return e0;
  dim3 grid(plan.qtiles, split1 - split0);
  scale_split_kernel<<<grid, kThreads, kSplitSmem, stream>>>(R, ldR, NQ, nov, D, fg, alpha, *tm_hi, *tm_lo, diag_part,
                                                             plan.ai_per_split, split0, err);
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
