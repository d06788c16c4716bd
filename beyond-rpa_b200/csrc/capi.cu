// C-ABI host layer of librpa_b200: handle, device workspace, staging of
// host/device arguments, and the orchestration of the sm_100a kernels.
// Entry points are declared (with the reference routines they replace) in
// include/rpa_b200.h.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <initializer_list>
#include <map>
#include <string>
#include <vector>

#include "abi_guard.h"
#include "kernels.h"

using rpa::dd;

namespace rpa {
thread_local int64_t g_launches = 0;
}

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

// Device-memory accounting of one handle: bytes its workspace holds, and the cap a caller may set
// (rpa_b200_set_workspace_limit; 0 = none).  Every workspace allocation of a call goes through
// dev_alloc / dev_free below, which charge the handle whose call is running on this thread.
struct WorkspaceAccount {
  size_t used = 0;
  size_t limit = 0;
};
namespace {
thread_local WorkspaceAccount* g_account = nullptr;

cudaError_t dev_alloc(void** p, size_t bytes) {
  WorkspaceAccount* a = g_account;
  if (a && a->limit && (bytes > a->limit || a->used > a->limit - bytes)) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;  // over the caller's cap: reported like a failed cudaMalloc
  }
  const cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaSuccess && a) a->used += bytes;
  return e;
}

void dev_free(void* p, size_t bytes) {
  if (!p) return;
  cudaFree(p);
  WorkspaceAccount* a = g_account;
  if (a) a->used = a->used > bytes ? a->used - bytes : 0;
}
}  // namespace

struct rpa_b200_handle {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;      // stream the calls run on
  cudaStream_t own_stream = nullptr;  // the handle's own stream
  cudaStream_t copy_stream = nullptr;  // host-to-device staging overlapped with compute
  std::string last_error;
  WorkspaceAccount account;  // device bytes of the workspace below and the caller's cap
  DevBuf R, D, eps, Xhi, Xlo, diag_part, diag, Pi, Ldiag, ddbuf;
  // direct-ring T2 / exchange workspace
  DevBuf tZ, tOm, tIOm, tP, tS, tV, tT, tTIT, tVt, tW, tU, tRU, tSmall, tPerm;
  // batched (many-instance) workspace: descriptors and per-batch results
  DevBuf bDesc, bRes;
  DevBuf gY, gD;  // adjoint workspace
  DevBuf xM;      // MBPT3 exchange: NT x NT matrices, R U and U X
  DevBuf eW, eA, eZ;  // symmetric eigensolver workspace, input and eigenvector buffers
  DevBuf thZ, thXa, thXi, thYX, thR;  // THC factors, Khatri-Rao block, Cholesky vectors formed from them
  DevBuf jU, jL, jX, jPno, jWork;      // particle-hole corrections: localised T2 vectors, PNOs, scratch
  DevBuf jPack, jQS, jS, jD;           // per-orbital PNO packs, QS slots, S blocks, grouped-GEMM descriptors
  DevBuf jT, jM, jV, jMap;             // batched PNO stage: T_ij, T T^T, eigenvectors, column map
  DevBuf jSK;                          // split-K partials of the G products
  DevBuf sxR, sxU, sxP;                // split-BF16 exchange: R and U (U2) hi/lo rows, partial sums
  DevBuf t2Z, t2M, t2Sync;             // split-BF16 ring contractions: Z (both layouts), M / P, milestones
  struct BatchGraph {
    uint64_t key;
    std::vector<cudaGraphExec_t> execs;
    std::vector<int64_t> launches;
  };
  BatchGraph bgraph{0, {}, {}};
  int* err_dev = nullptr;    // device error word
  int* count_dev = nullptr;  // non-finite counter
  PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  cudaEvent_t ev[5] = {};
  double timings[6] = {0, 0, 0, 0, 0, 0};
  int64_t launches = 0;
  int seg_chunks = 16;  // 512-column accumulation segments of the tensor-core SYRK
  int sync_every = 32;  // K chunks between the wave-progress milestones of the SYRK (0: off)
  DevBuf syncBuf;       // milestone counters of the SYRK waves
  // per-call event pairs around the scale/split pass and the contraction kernel
  std::vector<cudaEvent_t> pool;
  size_t pool_used = 0;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> split_ev, tc_ev;
  // CUDA graphs of the blocked Cholesky launch sequence, keyed by its arguments
  struct CholGraph {
    double* A;
    int64_t ld, stride;
    int n, nmat;
    double* Ldiag;
    cudaStream_t stream;
    int nb2, tile_w;
    int oz;  // digits of the int8 trailing updates (0: DMMA)
    cudaGraphExec_t exec;
    int64_t launches;
  };
  std::vector<CholGraph> chol_graphs;
  // int8 tensor-core trailing updates of the log-det (ozaki.cu): two digit-plane buffers and
  // their tensor maps, set up for one (order, matrices, panel width) at a time
  DevBuf ozBuf[2];
  rpa::OzakiWork ozw;
  int oz_n = 0, oz_nmat = 0;
  int ozaki_slices = 0;  // digits per entry of the int8 updates (RPA_B200_OZAKI_SLICES: 7 or 8; 0: DMMA)
  // tile plans of the FP64 log-det per bucket of 256 matrix orders (tuned or set)
  std::map<int, rpa::LogdetPlan> logdet_plans;
  uint64_t plans_version = 0;  // bumped on every change (part of the batched graph key)
  int autotune = 1;            // tune unseen order buckets on their first batched use (RPA_B200_AUTOTUNE=0: off)
  size_t batch_bytes = 0;      // device bytes per batch of the batched entry (0: 60% of free memory)
  size_t thc_piece_bytes = (size_t)2 << 30;  // device bytes of one piece of the THC Pi build (R, YX, hi + lo)
  int sosex_seg = 2;           // 32-column chunks per accumulation segment of the split exchange contraction
  int ring_seg = 2;            // the same for the split ring contractions of the T2 range finder
  DevBuf tune;                 // tuner workspace: descriptors and pivots of its test matrices
  // fork/join branches of the batched graph: [0] the next batch's scale/split pass, [1..2] log-det buckets
  cudaStream_t aux[3] = {};
  cudaEvent_t fork_ev[6] = {};
  // lookahead Cholesky schedules (one per log-det branch): high-priority critical-path stream,
  // default-priority stream for the rest of each trailing update (RPA_B200_LOOKAHEAD=0: off)
  bool lookahead = true;
  rpa::Lookahead la[3] = {};
};

namespace {

const double kPi = 3.14159265358979323846;

int fail(rpa_b200_handle* h, int status, const char* fmt, ...) {
  if (h) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    h->last_error = buf;
  }
  return status;
}

// RPA_ERR_NONFINITE for a NaN or Inf energy: entry points that do not screen every input array
// (the exchange and PNO energies) report a non-finite input through their result.
int finite_or_fail(rpa_b200_handle* h, std::initializer_list<double> xs, const char* what) {
  for (double x : xs)
    if (!std::isfinite(x)) return fail(h, RPA_ERR_NONFINITE, "non-finite %s (NaN or Inf in an input)", what);
  return RPA_OK;
}

#define RPA_CUDA(h, call)                                                                                   \
  do {                                                                                                      \
    cudaError_t e_ = (call);                                                                                \
    if (e_ != cudaSuccess) {                                                                                \
      if (e_ == cudaErrorMemoryAllocation) return fail(h, RPA_ERR_OOM, "%s: %s", #call, cudaGetErrorString(e_)); \
      return fail(h, RPA_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));                                \
    }                                                                                                       \
  } while (0)

// RPA_ERR_NONFINITE when a device result (rows x cols, column-major, ld) holds NaN or Inf: the array
// entry points that do not screen their inputs report a non-finite input through their output.
// Synchronises the stream.
int screen_result(rpa_b200_handle* h, const double* A, int64_t ld, int64_t rows, int64_t cols, const char* what) {
  RPA_CUDA(h, cudaMemsetAsync(h->count_dev, 0, sizeof(int), h->stream));
  RPA_CUDA(h, rpa::launch_count_nonfinite_cols(A, ld, rows, cols, h->count_dev, h->stream));
  int cnt = 0;
  RPA_CUDA(h, cudaMemcpyAsync(&cnt, h->count_dev, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  if (cnt) return fail(h, RPA_ERR_NONFINITE, "%d non-finite entries in %s (NaN or Inf in an input)", cnt, what);
  return RPA_OK;
}

cudaError_t ensure(DevBuf& b, size_t bytes) {
  if (b.bytes >= bytes && b.p) return cudaSuccess;
  if (b.p) {
    dev_free(b.p, b.bytes);
    b.p = nullptr;
    b.bytes = 0;
  }
  if (bytes == 0) bytes = 256;
  cudaError_t e = dev_alloc(&b.p, bytes);
  if (e == cudaSuccess) b.bytes = bytes;
  return e;
}

void release(DevBuf& b) {
  dev_free(b.p, b.bytes);
  b.p = nullptr;
  b.bytes = 0;
}

cudaEvent_t pool_event(rpa_b200_handle* h) {
  if (h->pool_used == h->pool.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    h->pool.push_back(e);
  }
  return h->pool[h->pool_used++];
}

bool is_device_ptr(const void* p) {
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

// Refuse array arguments that are device memory of a GPU other than the handle's (see
// rpa::classify_arg_memory).  Null pointers and pointers the runtime does not know are skipped
// here (the argument checks of each entry point handle them).
int check_arrays(rpa_b200_handle* h, std::initializer_list<const void*> arrays) {
  int index = 0;
  for (const void* p : arrays) {
    ++index;
    if (!p) continue;
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (rpa::classify_arg_memory((int)attr.type, attr.device, h->device) == rpa::ArgMemory::OtherDevice)
      return fail(h, RPA_ERR_INVALID_ARG,
                  "array argument %d is device memory of GPU %d; this handle runs on GPU %d (copy it first)", index,
                  attr.device, h->device);
  }
  return RPA_OK;
}

// Read a small array (host or device) into a host vector.
int fetch_small(rpa_b200_handle* h, const double* p, int64_t n, std::vector<double>& out) {
  out.resize((size_t)n);
  if (n == 0) return RPA_OK;
  if (is_device_ptr(p)) {
    RPA_CUDA(h, cudaMemcpyAsync(out.data(), p, (size_t)n * 8, cudaMemcpyDeviceToHost, h->stream));
    RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  } else {
    std::memcpy(out.data(), p, (size_t)n * 8);
  }
  return RPA_OK;
}

int check_device_error(rpa_b200_handle* h) {
  int err = 0;
  RPA_CUDA(h, cudaMemcpyAsync(&err, h->err_dev, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  if (err == rpa::kDevNotSPD) return fail(h, RPA_ERR_NOT_SPD, "1+Pi(u) is not positive definite (Cholesky pivot <= 0)");
  if (err != 0) return fail(h, RPA_ERR_TIMEOUT, "device-side bounded wait expired (code %d)", err);
  return RPA_OK;
}

struct Validated {
  int NQ;
  int64_t no, nv, nov;
  int K;
  std::vector<double> eo, ev, freqs, weights;
};

int validate_common(rpa_b200_handle* h, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* R, int64_t ldR,
                    const double* eo, const double* ev, int64_t NFreqs, const double* freqs, double alpha,
                    int64_t prec, Validated& v) {
  if (!h) return RPA_ERR_INVALID_ARG;
  if (NQ < 1 || NQ > (1 << 20)) return fail(h, RPA_ERR_INVALID_ARG, "NQ=%lld out of range", (long long)NQ);
  if (NOcc < 1 || NVirt < 1) return fail(h, RPA_ERR_INVALID_ARG, "NOcc and NVirt must be >= 1");
  if (NOcc > INT32_MAX / NVirt)
    return fail(h, RPA_ERR_TOO_LARGE, "NOcc*NVirt=%lld*%lld exceeds 2^31-1", (long long)NOcc, (long long)NVirt);
  if (NFreqs < 1 || NFreqs > 64) return fail(h, RPA_ERR_INVALID_ARG, "NFreqs=%lld not in [1,64]", (long long)NFreqs);
  if (ldR < NQ) return fail(h, RPA_ERR_INVALID_ARG, "ldR < NQ");
  if (!R || !eo || !ev || !freqs) return fail(h, RPA_ERR_INVALID_ARG, "NULL array argument");
  if (!(alpha > 0.0)) return fail(h, RPA_ERR_INVALID_ARG, "alpha must be > 0");
  if (prec != RPA_PREC_FP64 && prec != RPA_PREC_SPLIT_BF16)
    return fail(h, RPA_ERR_INVALID_ARG, "unknown precision mode %lld", (long long)prec);
  v.NQ = (int)NQ;
  v.no = NOcc;
  v.nv = NVirt;
  v.nov = NOcc * NVirt;
  v.K = (int)NFreqs;
  int s;
  if ((s = fetch_small(h, eo, NOcc, v.eo)) != RPA_OK) return s;
  if ((s = fetch_small(h, ev, NVirt, v.ev)) != RPA_OK) return s;
  if ((s = fetch_small(h, freqs, NFreqs, v.freqs)) != RPA_OK) return s;
  double emax = -INFINITY, vmin = INFINITY;
  for (double x : v.eo) {
    if (!std::isfinite(x)) return fail(h, RPA_ERR_NONFINITE, "non-finite occupied orbital energy");
    emax = std::max(emax, x);
  }
  for (double x : v.ev) {
    if (!std::isfinite(x)) return fail(h, RPA_ERR_NONFINITE, "non-finite virtual orbital energy");
    vmin = std::min(vmin, x);
  }
  if (!(vmin - emax > 0.0))
    return fail(h, RPA_ERR_INVALID_ARG, "Found invalid orbital energy gap. Cannot decompose energy denominators.");
  for (double x : v.freqs)
    if (!std::isfinite(x)) return fail(h, RPA_ERR_NONFINITE, "non-finite frequency");
  return RPA_OK;
}

// Stage R (NQ x nov, ldR) on the device; returns a device pointer and its ld.
// Orbital energies -> D(ai) on the device (no synchronisation).
int stage_eps(rpa_b200_handle* h, const Validated& v) {
  RPA_CUDA(h, ensure(h->eps, (size_t)(v.no + v.nv) * 8));
  double* ed = static_cast<double*>(h->eps.p);
  RPA_CUDA(h, cudaMemcpyAsync(ed, v.eo.data(), (size_t)v.no * 8, cudaMemcpyHostToDevice, h->stream));
  RPA_CUDA(h, cudaMemcpyAsync(ed + v.no, v.ev.data(), (size_t)v.nv * 8, cudaMemcpyHostToDevice, h->stream));
  RPA_CUDA(h, ensure(h->D, (size_t)v.nov * 8));
  RPA_CUDA(h, rpa::launch_dai(ed, ed + v.no, v.no, v.nv, static_cast<double*>(h->D.p), h->stream));
  return RPA_OK;
}

int stage_R(rpa_b200_handle* h, const Validated& v, const double* R, int64_t ldR, const double** Rd, int64_t* ldd) {
  if (is_device_ptr(R)) {
    *Rd = R;
    *ldd = ldR;
  } else {
    RPA_CUDA(h, ensure(h->R, (size_t)v.NQ * v.nov * 8));
    if (ldR == v.NQ)
      RPA_CUDA(h, cudaMemcpyAsync(h->R.p, R, (size_t)v.NQ * v.nov * 8, cudaMemcpyHostToDevice, h->stream));
    else
      RPA_CUDA(h, cudaMemcpy2DAsync(h->R.p, (size_t)v.NQ * 8, R, (size_t)ldR * 8, (size_t)v.NQ * 8, (size_t)v.nov,
                                    cudaMemcpyHostToDevice, h->stream));
    *Rd = static_cast<const double*>(h->R.p);
    *ldd = v.NQ;
  }
  // NaN/Inf screen of the Cholesky vectors: the NQ rows of every column (rows between NQ and ld
  // are the caller's padding, which no kernel reads)
  RPA_CUDA(h, cudaMemsetAsync(h->count_dev, 0, sizeof(int), h->stream));
  RPA_CUDA(h, rpa::launch_count_nonfinite_cols(*Rd, *ldd, v.NQ, v.nov, h->count_dev, h->stream));
  int s = stage_eps(h, v);
  if (s != RPA_OK) return s;
  int cnt = 0;
  RPA_CUDA(h, cudaMemcpyAsync(&cnt, h->count_dev, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  if (cnt) return fail(h, RPA_ERR_NONFINITE, "%d non-finite entries in the Cholesky vectors", cnt);
  return RPA_OK;
}

int encode_map(rpa_b200_handle* h, CUtensorMap* m, void* base, int64_t nov, int NQ, int kg, int64_t pitch, int rows) {
  cuuint64_t dims[3] = {(cuuint64_t)nov, (cuuint64_t)NQ, (cuuint64_t)kg};
  cuuint64_t strides[2] = {(cuuint64_t)pitch * 2, (cuuint64_t)pitch * 2 * (cuuint64_t)NQ};
  cuuint32_t box[3] = {(cuuint32_t)rpa::kSyrkTcTK, (cuuint32_t)rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = h->encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, base, dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(h, RPA_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return RPA_OK;
}

// Store views of X_hi / X_lo for the scale/split pass (boxes of 64 ai x 32 Q, 128-byte swizzle).
int encode_store_maps(rpa_b200_handle* h, CUtensorMap* hi, CUtensorMap* lo, void* xhi, void* xlo, int64_t nov, int NQ,
                      int kg, int64_t pitch) {
  if (rpa::encode_split_store_map(h->encode, hi, xhi, nov, NQ, kg, pitch) != cudaSuccess ||
      rpa::encode_split_store_map(h->encode, lo, xlo, nov, NQ, kg, pitch) != cudaSuccess)
    return fail(h, RPA_ERR_CUDA, "cuTensorMapEncodeTiled failed for the split operands' store views");
  return RPA_OK;
}

// Build the lower triangles of Pi_k (k = 0..K-1) into h->Pi (ld = NQ).
// Frequencies per split-BF16 group (all of them unless the device is short of memory).  The
// free-memory query can stall the host for tens of ms while the GPU idles: ask only when the
// buffers from an earlier call cannot already hold the largest group.  Returns -status on error.
int choose_kg(rpa_b200_handle* h, const Validated& v, int64_t pitch) {
  const size_t perFreq = (size_t)v.NQ * pitch * 2 * 2;  // hi + lo
  const int kmax = std::min(v.K, rpa::kMaxKgLaunch);
  if (h->Xhi.bytes >= (size_t)kmax * v.NQ * pitch * 2 && h->Xlo.bytes >= (size_t)kmax * v.NQ * pitch * 2) return kmax;
  size_t freeB = 0, totalB = 0;
  cudaError_t e = cudaMemGetInfo(&freeB, &totalB);
  if (e != cudaSuccess) {
    fail(h, RPA_ERR_CUDA, "CUDA error %s", cudaGetErrorString(e));
    return -RPA_ERR_CUDA;
  }
  const size_t have = h->Xhi.bytes + h->Xlo.bytes;
  const size_t budget = (size_t)((double)(freeB + have) * 0.7);
  return (int)std::min<size_t>((size_t)kmax, std::max<size_t>(1, budget / perFreq));
}

// Zeroed wave-progress counters for one tensor-core SYRK launch (nullptr: no synchronisation).
int prepare_sync(rpa_b200_handle* h, int NQ, int kg, int64_t nov_part, int** out) {
  *out = nullptr;
  const int64_t words = rpa::syrk_tc_sync_words(NQ, kg, nov_part, h->num_sms, h->sync_every);
  if (words <= 0) return RPA_OK;
  RPA_CUDA(h, ensure(h->syncBuf, (size_t)words * sizeof(int)));
  RPA_CUDA(h, cudaMemsetAsync(h->syncBuf.p, 0, (size_t)words * sizeof(int), h->stream));
  *out = static_cast<int*>(h->syncBuf.p);
  return RPA_OK;
}

int build_pi(rpa_b200_handle* h, const Validated& v, const double* Rd, int64_t ldR, double alpha, int64_t prec) {
  const int NQ = v.NQ;
  const int64_t nov = v.nov;
  const size_t piBytes = (size_t)v.K * NQ * NQ * 8;
  RPA_CUDA(h, ensure(h->Pi, piBytes));
  RPA_CUDA(h, ensure(h->diag, (size_t)v.K * NQ * 8));
  double* Pi = static_cast<double*>(h->Pi.p);
  const double* D = static_cast<const double*>(h->D.p);
  if (prec == RPA_PREC_FP64) {
    rpa::DsyrkArgs a{};
    a.A = Rd;
    a.lda = ldR;
    a.strideA = 0;
    a.C = Pi;
    a.ldc = NQ;
    a.strideC = (int64_t)NQ * NQ;
    a.n = NQ;
    a.kdim = nov;
    a.batch = v.K;
    a.D = D;
    a.alpha = alpha;
    for (int k = 0; k < v.K; ++k) a.u2[k] = v.freqs[k] * v.freqs[k];
    cudaEvent_t e0 = pool_event(h), e1 = pool_event(h);
    RPA_CUDA(h, cudaEventRecord(e0, h->stream));
    RPA_CUDA(h, rpa::launch_dsyrk_lower(a, h->stream));
    RPA_CUDA(h, cudaEventRecord(e1, h->stream));
    h->tc_ev.push_back({e0, e1});
    return RPA_OK;
  }
  // split-BF16: groups of frequencies sized to the free device memory
  const int64_t pitch = (nov + 7) / 8 * 8;
  int kg = 0;
  if ((kg = choose_kg(h, v, pitch)) <= 0) return -kg;
  RPA_CUDA(h, ensure(h->Xhi, (size_t)kg * NQ * pitch * 2));
  RPA_CUDA(h, ensure(h->Xlo, (size_t)kg * NQ * pitch * 2));
  const rpa::SplitPlan plan = rpa::plan_scale_split(NQ, nov, h->num_sms);
  RPA_CUDA(h, ensure(h->diag_part, (size_t)plan.nsplit * kg * NQ * 8));
  for (int g0 = 0; g0 < v.K; g0 += kg) {
    const int n = std::min(kg, v.K - g0);
    rpa::FreqGroup fg{};
    fg.n = n;
    for (int k = 0; k < n; ++k) fg.u2[k] = v.freqs[g0 + k] * v.freqs[g0 + k];
    double* diag = static_cast<double*>(h->diag.p) + (int64_t)g0 * NQ;
    CUtensorMap mAh, mAl, mBh, mBl, sHi, sLo;
    int s;
    if ((s = encode_store_maps(h, &sHi, &sLo, h->Xhi.p, h->Xlo.p, nov, NQ, n, pitch)) != RPA_OK) return s;
    cudaEvent_t e0 = pool_event(h), e1 = pool_event(h), e2 = pool_event(h);
    RPA_CUDA(h, cudaEventRecord(e0, h->stream));
    RPA_CUDA(h, rpa::launch_scale_split(Rd, ldR, NQ, nov, D, fg, alpha, &sHi, &sLo,
                                        static_cast<double*>(h->diag_part.p), diag, plan, h->err_dev, h->stream));
    RPA_CUDA(h, cudaEventRecord(e1, h->stream));
    h->split_ev.push_back({e0, e1});
    if ((s = encode_map(h, &mAh, h->Xhi.p, nov, NQ, n, pitch, rpa::kSyrkTcTM)) != RPA_OK) return s;
    if ((s = encode_map(h, &mAl, h->Xlo.p, nov, NQ, n, pitch, rpa::kSyrkTcTM)) != RPA_OK) return s;
    if ((s = encode_map(h, &mBh, h->Xhi.p, nov, NQ, n, pitch, rpa::kSyrkTcTN)) != RPA_OK) return s;
    if ((s = encode_map(h, &mBl, h->Xlo.p, nov, NQ, n, pitch, rpa::kSyrkTcTN)) != RPA_OK) return s;
    rpa::SyrkTcArgs a{};
    a.NQ = NQ;
    a.nov = nov;
    a.kg = n;
    a.Pi = Pi + (int64_t)g0 * NQ * NQ;
    a.ldPi = NQ;
    a.piStride = (int64_t)NQ * NQ;
    a.diag = diag;
    a.err = h->err_dev;
    a.seg_chunks = h->seg_chunks;
    if ((s = prepare_sync(h, NQ, n, nov, &a.sync)) != RPA_OK) return s;
    a.sync_every = h->sync_every;
    a.sync_lag = 2;
    RPA_CUDA(h, rpa::launch_syrk_split_bf16(&mAh, &mAl, &mBh, &mBl, a, h->num_sms, h->stream));
    RPA_CUDA(h, cudaEventRecord(e2, h->stream));
    h->tc_ev.push_back({e1, e2});
  }
  return RPA_OK;
}

// Split-BF16 Pi build from Cholesky vectors in host memory, all frequencies in one group: the ai
// columns are staged in kPipe pieces on the copy stream while the compute stream screens, scales,
// splits and contracts the pieces that have arrived (the tensor-core SYRK of piece c > 0 adds
// into Pi in FP64; the last piece writes the exact diagonal).  The diagonal partials are indexed
// by the global split, so the result equals the one-shot build.  count_dev collects the number of
// non-finite entries of R; the caller reads it after the stream has been synchronised.
// Returns 1 (nothing done) when the frequencies do not fit in one group.
// Relative sizes of the pieces R is staged in (RPA_B200_PIECES = comma-separated weights).
std::vector<int> piece_weights() {
  std::vector<int> w;
  if (const char* e = std::getenv("RPA_B200_PIECES")) {
    for (const char* p = e; *p;) {
      char* end = nullptr;
      const long x = std::strtol(p, &end, 10);
      if (end == p) break;
      if (x > 0 && x < 1000) w.push_back((int)x);
      p = (*end == ',') ? end + 1 : end;
    }
  }
  if (w.empty() || w.size() > 32) w = {1, 2, 3, 4, 5, 6};
  return w;
}

int build_pi_pipelined(rpa_b200_handle* h, const Validated& v, const double* Rh, int64_t ldR, double alpha) {
  // pieces of growing size (weights 1, 2, ..., 6 by default): the first copy, which nothing
  // hides, is short, and each later copy runs under the contraction of the pieces before it
  const std::vector<int> weights = piece_weights();
  const int kPipe = (int)weights.size();
  std::vector<int64_t> cum(kPipe + 1, 0);
  for (int c = 0; c < kPipe; ++c) cum[c + 1] = cum[c] + weights[c];
  const int64_t kWeightSum = cum[kPipe];
  const int NQ = v.NQ;
  const int64_t nov = v.nov;
  const int64_t pitch = (nov + 7) / 8 * 8;
  int kg = 0;
  if ((kg = choose_kg(h, v, pitch)) <= 0) return -kg;
  const rpa::SplitPlan plan = rpa::plan_scale_split(NQ, nov, h->num_sms);
  if (kg < v.K || plan.nsplit < 4 || plan.ai_per_split % 32 != 0) return 1;
  RPA_CUDA(h, ensure(h->R, (size_t)NQ * nov * 8));
  RPA_CUDA(h, ensure(h->Pi, (size_t)v.K * NQ * NQ * 8));
  RPA_CUDA(h, ensure(h->diag, (size_t)v.K * NQ * 8));
  RPA_CUDA(h, ensure(h->Xhi, (size_t)kg * NQ * pitch * 2));
  RPA_CUDA(h, ensure(h->Xlo, (size_t)kg * NQ * pitch * 2));
  RPA_CUDA(h, ensure(h->diag_part, (size_t)plan.nsplit * kg * NQ * 8));
  double* Rd = static_cast<double*>(h->R.p);
  double* Pi = static_cast<double*>(h->Pi.p);
  double* diag = static_cast<double*>(h->diag.p);
  const double* D = static_cast<const double*>(h->D.p);
  rpa::FreqGroup fg{};
  fg.n = v.K;
  for (int k = 0; k < v.K; ++k) fg.u2[k] = v.freqs[k] * v.freqs[k];
  CUtensorMap mAh, mAl, mBh, mBl, sHi, sLo;
  int s;
  if ((s = encode_store_maps(h, &sHi, &sLo, h->Xhi.p, h->Xlo.p, nov, NQ, v.K, pitch)) != RPA_OK) return s;
  if ((s = encode_map(h, &mAh, h->Xhi.p, nov, NQ, v.K, pitch, rpa::kSyrkTcTM)) != RPA_OK) return s;
  if ((s = encode_map(h, &mAl, h->Xlo.p, nov, NQ, v.K, pitch, rpa::kSyrkTcTM)) != RPA_OK) return s;
  if ((s = encode_map(h, &mBh, h->Xhi.p, nov, NQ, v.K, pitch, rpa::kSyrkTcTN)) != RPA_OK) return s;
  if ((s = encode_map(h, &mBl, h->Xlo.p, nov, NQ, v.K, pitch, rpa::kSyrkTcTN)) != RPA_OK) return s;
  RPA_CUDA(h, cudaMemsetAsync(h->count_dev, 0, sizeof(int), h->stream));
  // the copy stream starts after earlier work of this stream (R may still be read by it)
  cudaEvent_t start = pool_event(h);
  RPA_CUDA(h, cudaEventRecord(start, h->stream));
  RPA_CUDA(h, cudaStreamWaitEvent(h->copy_stream, start, 0));
  bool first = true;  // the first non-empty piece writes Pi, later ones add into it
  for (int c = 0; c < kPipe; ++c) {
    const int64_t w0 = cum[c], w1 = cum[c + 1];
    const int s0 = (int)(plan.nsplit * w0 / kWeightSum), s1 = (int)(plan.nsplit * w1 / kWeightSum);
    const int64_t a0 = (int64_t)s0 * plan.ai_per_split, a1 = std::min(nov, (int64_t)s1 * plan.ai_per_split);
    if (a1 <= a0) continue;
    cudaEvent_t arrived = pool_event(h);
    RPA_CUDA(h, cudaMemcpy2DAsync(Rd + a0 * NQ, (size_t)NQ * 8, Rh + a0 * ldR, (size_t)ldR * 8, (size_t)NQ * 8,
                                  (size_t)(a1 - a0), cudaMemcpyHostToDevice, h->copy_stream));
    RPA_CUDA(h, cudaEventRecord(arrived, h->copy_stream));
    RPA_CUDA(h, cudaStreamWaitEvent(h->stream, arrived, 0));
    RPA_CUDA(h, rpa::launch_count_nonfinite(Rd + a0 * NQ, (a1 - a0) * NQ, h->count_dev, h->stream));
    cudaEvent_t e0 = pool_event(h), e1 = pool_event(h), e2 = pool_event(h);
    RPA_CUDA(h, cudaEventRecord(e0, h->stream));
    RPA_CUDA(h, rpa::launch_scale_split_part(Rd, NQ, NQ, nov, D, fg, alpha, &sHi, &sLo,
                                             static_cast<double*>(h->diag_part.p), plan, s0, s1, h->err_dev,
                                             h->stream));
    const bool last = (s1 == plan.nsplit);
    if (last)
      RPA_CUDA(h, rpa::launch_diag_reduce(static_cast<double*>(h->diag_part.p), plan, v.K, NQ, diag, h->stream));
    RPA_CUDA(h, cudaEventRecord(e1, h->stream));
    h->split_ev.push_back({e0, e1});
    rpa::SyrkTcArgs a{};
    a.NQ = NQ;
    a.nov = nov;
    a.kg = v.K;
    a.Pi = Pi;
    a.ldPi = NQ;
    a.piStride = (int64_t)NQ * NQ;
    a.diag = last ? diag : nullptr;
    a.err = h->err_dev;
    a.seg_chunks = h->seg_chunks;
    a.chunk0 = (int)(a0 / 32);
    a.nov_part = a1 - a0;
    a.accumulate = first ? 0 : 1;
    first = false;
    if ((s = prepare_sync(h, NQ, v.K, a1 - a0, &a.sync)) != RPA_OK) return s;
    a.sync_every = h->sync_every;
    a.sync_lag = 2;
    RPA_CUDA(h, rpa::launch_syrk_split_bf16(&mAh, &mAl, &mBh, &mBl, a, h->num_sms, h->stream));
    RPA_CUDA(h, cudaEventRecord(e2, h->stream));
    h->tc_ev.push_back({e1, e2});
  }
  return RPA_OK;
}

// ---- tile plans of the FP64 log-det
// A plan is kept per bucket of 256 matrix orders; the tuner times every candidate on the
// matrices it is given and keeps the fastest (measured, not modelled: the best outer block and
// CTA tile depend on the order, the batch width and what runs beside the log-det).
constexpr int kPlanBucket = 256;
const rpa::LogdetPlan kLogdetCands[6] = {{128, 2}, {256, 2}, {512, 2}, {128, 4}, {256, 4}, {512, 4}};

int plan_bucket(int n) { return (n + kPlanBucket - 1) / kPlanBucket; }

rpa::LogdetPlan plan_for(const rpa_b200_handle* h, int n) {
  auto it = h->logdet_plans.find(plan_bucket(n));
  return it != h->logdet_plans.end() ? it->second : rpa::default_logdet_plan();
}

// Time every candidate on nmat matrices of orders <= nmax (device descriptors; contents are
// overwritten with seeded SPD test matrices), two runs each (the first also loads the variant's
// kernels), keep the fastest for the bucket of nmax.  ms (6 entries or null): each candidate's time.
int tune_logdet_on(rpa_b200_handle* h, const rpa::MatDesc* dmats, int nmat, int nmax, double* ms) {
  cudaEvent_t t0 = pool_event(h), t1 = pool_event(h);
  if (!t0 || !t1) return fail(h, RPA_ERR_CUDA, "event creation failed");
  int best = 0;
  float best_ms = 0.0f;
  for (int c = 0; c < 6; ++c) {
    float t = 0.0f;
    for (int rep = 0; rep < 2; ++rep) {
      RPA_CUDA(h, rpa::launch_fill_spd_varlen(dmats, nmat, nmax, 0x5eedull + (uint64_t)rep, h->stream));
      RPA_CUDA(h, cudaEventRecord(t0, h->stream));
      RPA_CUDA(h, rpa::launch_logdet_varlen(dmats, nmat, nmax, h->err_dev, h->stream, kLogdetCands[c],
                                            h->lookahead ? &h->la[0] : nullptr));
      RPA_CUDA(h, cudaEventRecord(t1, h->stream));
      RPA_CUDA(h, cudaEventSynchronize(t1));
      RPA_CUDA(h, cudaEventElapsedTime(&t, t0, t1));
    }
    if (ms) ms[c] = t;
    if (c == 0 || t < best_ms) {
      best_ms = t;
      best = c;
    }
  }
  int s = check_device_error(h);  // the test matrices are positive definite: a flag is a real fault
  if (s != RPA_OK) return s;
  h->logdet_plans[plan_bucket(nmax)] = kLogdetCands[best];
  ++h->plans_version;
  return RPA_OK;
}

// Tune the bucket of order n on nmat test matrices of that order stored at base (n*n doubles each).
int tune_uniform(rpa_b200_handle* h, int n, int nmat, double* base, double* ms) {
  RPA_CUDA(h, ensure(h->tune, (size_t)nmat * (sizeof(rpa::MatDesc) + 8 * ((size_t)n + 4)) + 512));
  std::vector<rpa::MatDesc> mats(nmat);
  rpa::MatDesc* dmats = static_cast<rpa::MatDesc*>(h->tune.p);
  double* scratch = reinterpret_cast<double*>(static_cast<uint8_t*>(h->tune.p) +
                                              ((size_t)nmat * sizeof(rpa::MatDesc) + 255) / 256 * 256);
  for (int z = 0; z < nmat; ++z) {
    mats[z].A = base + (size_t)z * n * n;
    mats[z].ld = n;
    mats[z].n = n;
    mats[z].Ldiag = scratch + (size_t)z * n;
    mats[z].tr_dd = scratch + (size_t)nmat * n + 4 * (size_t)z;
    mats[z].ld_dd = mats[z].tr_dd + 2;
  }
  RPA_CUDA(h, cudaMemcpyAsync(dmats, mats.data(), sizeof(rpa::MatDesc) * nmat, cudaMemcpyHostToDevice, h->stream));
  int s = tune_logdet_on(h, dmats, nmat, n, ms);
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));  // mats must outlive its copy
  return s;
}

// First use of an order bucket by a single-system log-det (autotune on, order >= 512): tune it
// on as many test matrices as the call factors, in a temporary buffer (fewer, down to 4, when
// memory is short; the default plan stays when even that fails).  Returns a status.
int tune_single(rpa_b200_handle* h, int n, int nmat) {
  if (!h->autotune || n < 512 || h->logdet_plans.count(plan_bucket(n))) return RPA_OK;
  for (int m = nmat; m >= 1; m = m > 4 ? 4 : 0) {
    void* tmp = nullptr;
    if (dev_alloc(&tmp, (size_t)m * n * n * 8) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    int s = tune_uniform(h, n, m, static_cast<double*>(tmp), nullptr);
    cudaStreamSynchronize(h->stream);
    dev_free(tmp, (size_t)m * n * n * 8);
    if (s == RPA_OK) RPA_CUDA(h, cudaMemsetAsync(h->err_dev, 0, sizeof(int), h->stream));
    return s;
  }
  return RPA_OK;
}

// Blocked Cholesky of nmat matrices through a cached CUDA graph (the launch
// sequence depends only on the arguments; ~6 launches per 64 columns would
// otherwise leave the GPU idle between the small late-step kernels).
// The int8 digit-plane buffers for nmat matrices of order n and the plan's panel width (nullptr:
// the trailing updates stay on DMMA).  Reallocating them invalidates the captured Cholesky graphs,
// which hold their addresses.
const rpa::OzakiWork* ozaki_for(rpa_b200_handle* h, int n, int nmat, const rpa::LogdetPlan& plan) {
  const int S = h->ozaki_slices;
  if (S == 0 || n < 2 * plan.nb2 || plan.nb2 > 512) return nullptr;
  if (h->ozw.S == S && h->ozw.K == plan.nb2 && h->oz_n == n && h->oz_nmat == nmat) return &h->ozw;
  const size_t bytes = rpa::ozaki_buffer_bytes(n, nmat, plan.nb2, S);
  bool grew = false;
  for (DevBuf& b : h->ozBuf)
    if (b.bytes < bytes) {
      cudaStreamSynchronize(h->stream);
      if (ensure(b, bytes) != cudaSuccess) {
        cudaGetLastError();
        h->ozw.S = 0;
        return nullptr;  // no room: DMMA updates
      }
      grew = true;
    }
  if (grew) {
    for (auto& g : h->chol_graphs) cudaGraphExecDestroy(g.exec);
    h->chol_graphs.clear();
  }
  void* bufs[2] = {h->ozBuf[0].p, h->ozBuf[1].p};
  if (rpa::ozaki_setup(h->ozw, h->encode, bufs, n, nmat, plan.nb2, S) != cudaSuccess) {
    h->ozw.S = 0;
    return nullptr;
  }
  h->ozw.num_sms = h->num_sms;
  h->oz_n = n;
  h->oz_nmat = nmat;
  return &h->ozw;
}

int cholesky(rpa_b200_handle* h, double* A, int64_t ld, int64_t stride, int n, int nmat, double* Ldiag) {
  if (int ts = tune_single(h, n, nmat)) return ts;
  const rpa::LogdetPlan plan = plan_for(h, n);
  const rpa::OzakiWork* oz = ozaki_for(h, n, nmat, plan);
  for (auto& g : h->chol_graphs) {
    if (g.A == A && g.ld == ld && g.stride == stride && g.n == n && g.nmat == nmat && g.Ldiag == Ldiag &&
        g.stream == h->stream && g.nb2 == plan.nb2 && g.tile_w == plan.tile_w && g.oz == (oz ? oz->S : 0)) {
      RPA_CUDA(h, cudaGraphLaunch(g.exec, h->stream));
      rpa::g_launches += g.launches;
      return RPA_OK;
    }
  }
  const int64_t before = rpa::g_launches;
  cudaGraph_t graph = nullptr;
  if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
    cudaError_t e = rpa::launch_cholesky_lower(A, ld, stride, n, nmat, Ldiag, h->err_dev, h->stream, plan,
                                               h->lookahead ? &h->la[0] : nullptr, oz);
    cudaError_t e2 = cudaStreamEndCapture(h->stream, &graph);
    const int64_t count = rpa::g_launches - before;
    rpa::g_launches = before;
    cudaGraphExec_t exec = nullptr;
    if (e == cudaSuccess && e2 == cudaSuccess && graph &&
        cudaGraphInstantiate(&exec, graph, cudaGraphInstantiateFlagUseNodePriority) == cudaSuccess) {
      cudaGraphDestroy(graph);
      if (h->chol_graphs.size() >= 8) {
        cudaGraphExecDestroy(h->chol_graphs.front().exec);
        h->chol_graphs.erase(h->chol_graphs.begin());
      }
      h->chol_graphs.push_back(
          {A, ld, stride, n, nmat, Ldiag, h->stream, plan.nb2, plan.tile_w, oz ? oz->S : 0, exec, count});
      RPA_CUDA(h, cudaGraphLaunch(exec, h->stream));
      rpa::g_launches += count;
      return RPA_OK;
    }
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
  } else {
    cudaGetLastError();
  }
  // capture unavailable on this stream: launch the same kernels directly
  RPA_CUDA(h, rpa::launch_cholesky_lower(A, ld, stride, n, nmat, Ldiag, h->err_dev, h->stream, plan, nullptr, oz));
  return RPA_OK;
}

// Energy from the lower triangles of K matrices Pi_k stored in h->Pi (ld = NQ).
int energy_from_workspace(rpa_b200_handle* h, int NQ, int K, const std::vector<double>& w, double* Ec, double* Eu) {
  double* Pi = static_cast<double*>(h->Pi.p);
  RPA_CUDA(h, ensure(h->Ldiag, (size_t)K * NQ * 8));
  RPA_CUDA(h, ensure(h->ddbuf, (size_t)4 * K * 8));
  double* tr = static_cast<double*>(h->ddbuf.p);
  double* ld = tr + 2 * K;
  RPA_CUDA(h, rpa::launch_trace_shift(Pi, NQ, (int64_t)NQ * NQ, NQ, K, nullptr, tr, h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[2], h->stream));
  int cs = cholesky(h, Pi, NQ, (int64_t)NQ * NQ, NQ, K, static_cast<double*>(h->Ldiag.p));
  if (cs != RPA_OK) return cs;
  RPA_CUDA(h, rpa::launch_logdet_sum(static_cast<double*>(h->Ldiag.p), NQ, K, ld, h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[3], h->stream));
  std::vector<double> host(4 * (size_t)K);
  RPA_CUDA(h, cudaMemcpyAsync(host.data(), tr, (size_t)4 * K * 8, cudaMemcpyDeviceToHost, h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  int s = check_device_error(h);
  if (s != RPA_OK) return s;
  dd ec{0.0, 0.0};
  for (int k = 0; k < K; ++k) {
    dd trk{host[2 * k], host[2 * k + 1]};
    dd ldk{host[2 * K + 2 * k], host[2 * K + 2 * k + 1]};
    dd eu = rpa::dd_add_dd(ldk, {-trk.hi, -trk.lo});
    if (!std::isfinite(eu.hi)) return fail(h, RPA_ERR_NONFINITE, "non-finite E(u) at frequency %d", k + 1);
    if (Eu) Eu[k] = eu.hi + eu.lo;
    // w_k/(2 pi) * E(u): exact product in double-double
    const double f = w[k] / (2.0 * kPi);
    const double p = eu.hi * f;
    const double pe = std::fma(eu.hi, f, -p) + eu.lo * f;
    ec = rpa::dd_add_dd(ec, {p, pe});
  }
  *Ec = ec.hi + ec.lo;
  return RPA_OK;
}


// ------------------------------------------------------------------ direct-ring T2
// I(1) M = -(1/4pi) sum_k Z_k^T (Z_k M),  Z_k = sqrt(w_k) L_k^{-1} R diag(chi_k),
// chi_k = -alpha D/(D^2+u_k^2), L_k the Cholesky factor of 1 + Pi_k (kept in h->Pi
// by the energy step).  This is rpa_CC_IM_v5 (src/rpa/rpa_CC_Doubles.f90:369-422)
// with Q diag(1/(1+pi)) Q^T = (1+Pi)^{-1} = L^{-T} L^{-1}: no eigen-decomposition
// of Pi(u) is needed for lambda = 1.
struct T2Ctx {
  int NQ, K;
  int64_t nov;
  const double* R;
  int64_t ldR;
  double alpha;
  std::vector<double> u2, w;
  int zk;             // frequencies per Z group
  bool z_resident;    // all groups built once
  // split-BF16 ring contractions (prec split with Z resident): Z split once in both K-major
  // layouts, Zt (rows K*NQ, nov contiguous, pitch p1) for P = Z M and Z (rows nov, K*NQ
  // contiguous, pitch p2) for Z^T P
  bool split = false;
  int64_t p1 = 0, p2 = 0;
  CUtensorMap mZt[2], mZ[2];
};

// Split-BF16 operands of the ring contractions, once per T2 call (Z resident in h->tZ).
int prepare_split_z(rpa_b200_handle* h, T2Ctx& c) {
  const int64_t rows = (int64_t)c.K * c.NQ;
  if (rows > INT32_MAX || c.nov > INT32_MAX) return fail(h, RPA_ERR_TOO_LARGE, "T2 split operands too large");
  c.p1 = rpa::sosex_tc_nvp((int)c.nov);
  c.p2 = rpa::sosex_tc_nvp((int)rows);
  const size_t b1 = (size_t)rows * c.p1 * 2, b2 = (size_t)c.nov * c.p2 * 2;  // bytes of one bf16 part
  RPA_CUDA(h, ensure(h->t2Z, 2 * b1 + 2 * b2 + 512));
  auto* base = static_cast<uint8_t*>(h->t2Z.p);
  auto* zth = reinterpret_cast<__nv_bfloat16*>(base);
  auto* ztl = reinterpret_cast<__nv_bfloat16*>(base + b1);
  auto* zh = reinterpret_cast<__nv_bfloat16*>(base + 2 * b1);
  auto* zl = reinterpret_cast<__nv_bfloat16*>(base + 2 * b1 + b2);
  const double* Z = static_cast<const double*>(h->tZ.p);
  RPA_CUDA(h, rpa::launch_split_rows(Z, rows, (int)rows, 1, (int)c.nov, zth, ztl, h->stream));
  RPA_CUDA(h, rpa::launch_split_cols(Z, rows, (int)c.nov, 1, (int)rows, zh, zl, h->stream));
  int s;
  if ((s = encode_map(h, &c.mZt[0], zth, c.p1, (int)rows, 1, c.p1, rpa::kSyrkTcTM))) return s;
  if ((s = encode_map(h, &c.mZt[1], ztl, c.p1, (int)rows, 1, c.p1, rpa::kSyrkTcTM))) return s;
  if ((s = encode_map(h, &c.mZ[0], zh, c.p2, (int)c.nov, 1, c.p2, rpa::kSyrkTcTM))) return s;
  if ((s = encode_map(h, &c.mZ[1], zl, c.p2, (int)c.nov, 1, c.p2, rpa::kSyrkTcTM))) return s;
  c.split = true;
  return RPA_OK;
}

// C (M x N, ld ldc) = alpha A B^T with A given by two maps (M rows) and B (N x K, column-major
// K x N in memory, ld ldb) split here into bf16 rows of pitch = the A maps' pitch.
int gemm_split_t2(rpa_b200_handle* h, const CUtensorMap* amaps, int M, int64_t K, int64_t pitch, const double* B,
                  int64_t ldb, int N, double* C, int64_t ldc, double alpha) {
  const size_t bb = (size_t)N * pitch * 2;
  RPA_CUDA(h, ensure(h->t2M, 2 * bb + 256));
  auto* bh = static_cast<__nv_bfloat16*>(h->t2M.p);
  auto* bl = reinterpret_cast<__nv_bfloat16*>(static_cast<uint8_t*>(h->t2M.p) + bb);
  RPA_CUDA(h, rpa::launch_split_cols(B, ldb, N, 1, (int)K, bh, bl, h->stream));
  CUtensorMap maps[4] = {amaps[0], amaps[1]};
  int s;
  if ((s = encode_map(h, &maps[2], bh, pitch, N, 1, pitch, rpa::kSyrkTcTN))) return s;
  if ((s = encode_map(h, &maps[3], bl, pitch, N, 1, pitch, rpa::kSyrkTcTN))) return s;
  rpa::GemmSplitArgs g{};
  g.M = M;
  g.N = N;
  g.K = K;
  g.C = C;
  g.ldc = ldc;
  g.alpha = alpha;
  g.beta = 0.0;
  // short accumulation segments: each product feeds the Rayleigh-Ritz matrix, and the
  // round-toward-zero bias of a tensor-core accumulator grows with the additions it takes
  // (16-chunk segments bias A by ~3e-6 relative, 2-chunk segments by ~4e-7)
  g.seg_chunks = h->ring_seg;
  g.err = h->err_dev;
  g.sync_every = h->sync_every;
  g.sync_lag = 2;
  const int64_t words = rpa::gemm_split_sync_words(M, N, K, h->num_sms, h->sync_every);
  if (words > 0) {
    RPA_CUDA(h, ensure(h->t2Sync, (size_t)words * sizeof(int)));
    RPA_CUDA(h, cudaMemsetAsync(h->t2Sync.p, 0, (size_t)words * sizeof(int), h->stream));
    g.sync = static_cast<int*>(h->t2Sync.p);
  }
  RPA_CUDA(h, rpa::launch_gemm_split_bf16(maps, g, h->num_sms, h->stream));
  return RPA_OK;
}

int build_z_group(rpa_b200_handle* h, const T2Ctx& c, int g0, int n, double* Z) {
  rpa::ChiGroup cg{};
  cg.n = n;
  cg.alpha = c.alpha;
  for (int k = 0; k < n; ++k) {
    cg.u2[k] = c.u2[g0 + k];
    cg.sqrtw[k] = std::sqrt(c.w[g0 + k]);
  }
  const int64_t ldz = (int64_t)n * c.NQ;
  RPA_CUDA(h, rpa::launch_chi_scale(c.R, c.ldR, c.NQ, c.nov, static_cast<const double*>(h->D.p), cg, Z, ldz,
                                    h->stream));
  // L_k^{-1} on rows k*NQ.. of Z (batched over the group's frequencies)
  const double* L = static_cast<const double*>(h->Pi.p) + (int64_t)g0 * c.NQ * c.NQ;
  RPA_CUDA(h, rpa::launch_trsm_lower_left(L, c.NQ, (int64_t)c.NQ * c.NQ, Z, ldz, c.NQ, c.NQ, (int)c.nov, n,
                                          h->stream));
  return RPA_OK;
}

// out (nov x ncols, ld nov) = I M (M: nov x ncols, ld nov)
int apply_I(rpa_b200_handle* h, const T2Ctx& c, const double* M, int ncols, double* out) {
  double* Z = static_cast<double*>(h->tZ.p);
  double* P = static_cast<double*>(h->tP.p);
  if (c.split) {  // P = Z M, out = -(1/4 pi) Z^T P as split-BF16 GEMMs on the tensor cores
    const int64_t rows = (int64_t)c.K * c.NQ;
    int s = gemm_split_t2(h, c.mZt, (int)rows, c.nov, c.p1, M, c.nov, ncols, P, rows, 1.0);
    if (s == RPA_OK)
      s = gemm_split_t2(h, c.mZ, (int)c.nov, rows, c.p2, P, rows, ncols, out, c.nov, -1.0 / (4.0 * kPi));
    return s;
  }
  bool first = true;
  for (int g0 = 0; g0 < c.K; g0 += c.zk) {
    const int n = std::min(c.zk, c.K - g0);
    const int64_t ldz = (int64_t)n * c.NQ;
    double* Zg = c.z_resident ? Z + (int64_t)g0 * c.NQ * c.nov : Z;
    if (!c.z_resident) {
      int s = build_z_group(h, c, g0, n, Zg);
      if (s != RPA_OK) return s;
    }
    rpa::GemmF64Args g{};
    g.M = (int)ldz;
    g.N = ncols;
    g.K = c.nov;
    g.A = Zg;
    g.a_m = 1;
    g.a_k = ldz;
    g.B = M;
    g.b_k = 1;
    g.b_n = c.nov;
    g.C = P;
    g.ldc = ldz;
    g.alpha = 1.0;
    g.beta = 0.0;
    g.batch = 1;
    RPA_CUDA(h, rpa::launch_gemm_f64(g, h->stream));
    rpa::GemmF64Args g2{};
    g2.M = (int)c.nov;
    g2.N = ncols;
    g2.K = ldz;
    g2.A = Zg;
    g2.a_m = ldz;
    g2.a_k = 1;
    g2.B = P;
    g2.b_k = 1;
    g2.b_n = ldz;
    g2.C = out;
    g2.ldc = c.nov;
    g2.alpha = -1.0 / (4.0 * kPi);
    g2.beta = first ? 0.0 : 1.0;
    g2.batch = 1;
    RPA_CUDA(h, rpa::launch_gemm_f64(g2, h->stream));
    first = false;
  }
  return RPA_OK;
}

// Normalise the columns of X (rows x cols, ld rows) on the device.
int normalize_columns(rpa_b200_handle* h, double* X, int64_t rows, int cols) {
  double* nrm = static_cast<double*>(h->tSmall.p);
  RPA_CUDA(h, rpa::launch_col_sqnorm(X, rows, cols, rows, nrm, h->stream));
  RPA_CUDA(h, rpa::launch_scale_cols(X, rows, cols, rows, nrm, true, h->stream));
  return RPA_OK;
}

// Symmetric eigen-decomposition of A (n x n, ld n; destroyed) on the GPU (Householder
// tridiagonalisation + divide and conquer, syevd.cu): V receives the eigenvectors, evals their
// eigenvalues (in V's column order) and order the permutation that sorts them ascending.
int sym_eig(rpa_b200_handle* h, double* A, double* V, int n, std::vector<double>& evals, std::vector<int>& order) {
  RPA_CUDA(h, ensure(h->eW, rpa::syevd_workspace_bytes(n)));
  bool converged = false;
  RPA_CUDA(h, rpa::syevd(A, n, V, h->eW.p, h->eW.bytes, evals, converged, h->stream));
  if (!converged) return fail(h, RPA_ERR_NOT_CONVERGED, "symmetric eigensolver: a leaf did not converge (n=%d)", n);
  for (double x : evals)
    if (!std::isfinite(x)) return fail(h, RPA_ERR_NONFINITE, "symmetric eigensolver: non-finite eigenvalue (n=%d)", n);
  order.resize(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return evals[a] < evals[b]; });
  return RPA_OK;
}

// dst(:, j) = src(:, cols[j]) * scale[j] on the device (cols/scale from the host)
int gather(rpa_b200_handle* h, const double* src, int64_t rows, double* dst, const std::vector<int>& cols,
           const std::vector<double>* scale) {
  const int nc = (int)cols.size();
  if (nc == 0) return RPA_OK;
  int* perm = static_cast<int*>(h->tPerm.p);
  double* sc = static_cast<double*>(h->tSmall.p);
  RPA_CUDA(h, cudaMemcpyAsync(perm, cols.data(), (size_t)nc * sizeof(int), cudaMemcpyHostToDevice, h->stream));
  if (scale)
    RPA_CUDA(h, cudaMemcpyAsync(sc, scale->data(), (size_t)nc * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  RPA_CUDA(h, rpa::launch_gather_cols(src, rows, dst, rows, rows, nc, perm, scale ? sc : nullptr, h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));  // host vectors must outlive the copies
  return RPA_OK;
}

rpa::GemmF64Args gemm_nn(int M, int N, int64_t K, const double* A, int64_t lda, const double* B, int64_t ldb,
                         double* C, int64_t ldc) {
  rpa::GemmF64Args g{};
  g.M = M;
  g.N = N;
  g.K = K;
  g.A = A;
  g.a_m = 1;
  g.a_k = lda;
  g.B = B;
  g.b_k = 1;
  g.b_n = ldb;
  g.C = C;
  g.ldc = ldc;
  g.alpha = 1.0;
  g.beta = 0.0;
  g.batch = 1;
  return g;
}
rpa::GemmF64Args gemm_tn(int M, int N, int64_t K, const double* A, int64_t lda, const double* B, int64_t ldb,
                         double* C, int64_t ldc) {
  rpa::GemmF64Args g = gemm_nn(M, N, K, A, lda, B, ldb, C, ldc);
  g.a_m = lda;
  g.a_k = 1;
  return g;
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
    cudaGetLastError();
    return 0.f;
  }
  return ms;
}

int begin_call(rpa_b200_handle* h) {
  if (!h) return RPA_ERR_INVALID_ARG;
  h->last_error.clear();
  g_account = &h->account;
  h->pool_used = 0;
  h->split_ev.clear();
  h->tc_ev.clear();
  rpa::g_launches = 0;
  RPA_CUDA(h, cudaSetDevice(h->device));
  RPA_CUDA(h, cudaMemsetAsync(h->err_dev, 0, sizeof(int), h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[0], h->stream));
  return RPA_OK;
}

void finish_timings(rpa_b200_handle* h) {
  cudaEventSynchronize(h->ev[4]);
  h->timings[0] = elapsed(h->ev[0], h->ev[1]);
  h->timings[1] = elapsed(h->ev[1], h->ev[2]);
  h->timings[2] = elapsed(h->ev[2], h->ev[3]);
  h->timings[3] = elapsed(h->ev[3], h->ev[4]);
  double tc = 0.0, sp = 0.0;
  for (auto& p : h->tc_ev) tc += elapsed(p.first, p.second);
  for (auto& p : h->split_ev) sp += elapsed(p.first, p.second);
  h->timings[4] = tc;
  h->timings[5] = sp;
  h->launches = rpa::g_launches;
}

// Handler of the entry points' function-try-blocks: the status of the exception in flight, its
// text in last_error, and a stream capture the unwound call left open on the handle's stream ended
// and discarded, so that the next call on this handle starts clean.
int exception_status(rpa_b200_handle* h) noexcept {
  if (!h) return rpa::status_of_exception(nullptr);
  const int status = rpa::status_of_exception(&h->last_error);
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (h->stream && cudaStreamIsCapturing(h->stream, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(h->stream, &g);
    if (g) cudaGraphDestroy(g);
  }
  cudaGetLastError();
  return status;
}

}  // namespace

extern "C" {

int rpa_b200_create(rpa_b200_handle** handle, int64_t device, int64_t flags) try {
  (void)flags;
  if (!handle) return RPA_ERR_INVALID_ARG;
  *handle = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return RPA_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) return RPA_ERR_INVALID_ARG;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, (int)device) != cudaSuccess) return RPA_ERR_CUDA;
  if (prop.major != 10) return RPA_ERR_NO_DEVICE;  // sm_100 family only
  rpa_b200_handle* h = new rpa_b200_handle();
  h->device = (int)device;
  h->num_sms = prop.multiProcessorCount;
  if (cudaSetDevice(h->device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->aux[0], cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->aux[1], cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->aux[2], cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&h->err_dev, sizeof(int)) != cudaSuccess || cudaMalloc(&h->count_dev, sizeof(int)) != cudaSuccess) {
    rpa_b200_destroy(h);  // releases whatever was created (it skips null members)
    return RPA_ERR_CUDA;
  }
  h->stream = h->own_stream;
  if (const char* sc = std::getenv("RPA_B200_SEG_CHUNKS")) h->seg_chunks = std::atoi(sc);
  if (const char* se = std::getenv("RPA_B200_SYNC_EVERY")) h->sync_every = std::atoi(se);
  if (const char* at = std::getenv("RPA_B200_AUTOTUNE")) h->autotune = std::atoi(at) != 0;
  if (const char* bb = std::getenv("RPA_B200_BATCH_BYTES")) h->batch_bytes = (size_t)std::atoll(bb);
  if (const char* tp = std::getenv("RPA_B200_THC_PIECE_BYTES")) h->thc_piece_bytes = (size_t)std::max(1ll, std::atoll(tp));
  if (const char* sg = std::getenv("RPA_B200_SOSEX_SEG")) h->sosex_seg = std::max(1, std::atoi(sg));
  if (const char* rg = std::getenv("RPA_B200_RING_SEG")) h->ring_seg = std::max(1, std::atoi(rg));
  for (auto& e : h->ev) cudaEventCreate(&e);
  for (auto& e : h->fork_ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  if (const char* la = std::getenv("RPA_B200_LOOKAHEAD")) h->lookahead = std::atoi(la) != 0;
  h->ozaki_slices = rpa::ozaki_slices_default();
  {
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    for (auto& l : h->la) {
      if (cudaStreamCreateWithPriority(&l.crit, cudaStreamNonBlocking, greatest) != cudaSuccess ||
          cudaStreamCreateWithPriority(&l.rest, cudaStreamNonBlocking, least) != cudaSuccess) {
        rpa_b200_destroy(h);
        return RPA_ERR_CUDA;
      }
      for (auto& e : l.ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    }
  }
  cudaDriverEntryPointQueryResult q;
  void* fn = nullptr;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !fn) {
    rpa_b200_destroy(h);
    return RPA_ERR_CUDA;
  }
  h->encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  *handle = h;
  return RPA_OK;
} catch (...) {
  return rpa::status_of_exception(nullptr);
}

int rpa_b200_destroy(rpa_b200_handle* h) try {
  if (!h) return RPA_OK;
  g_account = &h->account;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->own_stream) cudaStreamSynchronize(h->own_stream);
  if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
  for (DevBuf* b : {&h->R, &h->D, &h->eps, &h->Xhi, &h->Xlo, &h->diag_part, &h->diag, &h->Pi, &h->Ldiag, &h->ddbuf,
                    &h->tZ, &h->tOm, &h->tIOm, &h->tP, &h->tS, &h->tV, &h->tT, &h->tTIT, &h->tVt, &h->tW, &h->tU,
                    &h->tRU, &h->tSmall, &h->tPerm, &h->bDesc, &h->bRes, &h->gY, &h->gD,
                    &h->xM, &h->eW, &h->eA, &h->eZ, &h->thZ, &h->thXa, &h->thXi, &h->thYX, &h->thR,
                    &h->jU, &h->jL, &h->jX, &h->jPno, &h->jWork,
                    &h->jPack, &h->jQS, &h->jS, &h->jD, &h->syncBuf,
                    &h->jT, &h->jM, &h->jV, &h->jMap, &h->jSK, &h->tune, &h->sxR, &h->sxU, &h->sxP,
                    &h->t2Z, &h->t2M, &h->t2Sync, &h->ozBuf[0], &h->ozBuf[1]})
    release(*b);
  for (auto e : h->bgraph.execs) cudaGraphExecDestroy(e);
  if (h->err_dev) cudaFree(h->err_dev);
  if (h->count_dev) cudaFree(h->count_dev);
  for (auto& e : h->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : h->pool) cudaEventDestroy(e);
  for (auto& g : h->chol_graphs) cudaGraphExecDestroy(g.exec);
  for (auto& e : h->fork_ev)
    if (e) cudaEventDestroy(e);
  for (auto& st : h->aux)
    if (st) {
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
  for (auto& l : h->la) {
    for (cudaStream_t st : {l.crit, l.rest})
      if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
      }
    for (auto& e : l.ev)
      if (e) cudaEventDestroy(e);
  }
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  g_account = nullptr;
  delete h;
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}

const char* rpa_b200_status_string(int status) {
  switch (status) {
    case RPA_OK: return "success";
    case RPA_ERR_INVALID_ARG: return "invalid argument";
    case RPA_ERR_NOT_SPD: return "1+Pi(u) is not positive definite";
    case RPA_ERR_NONFINITE: return "non-finite input or result";
    case RPA_ERR_OOM: return "out of memory";
    case RPA_ERR_CUDA: return "CUDA error";
    case RPA_ERR_TIMEOUT: return "device-side wait timed out";
    case RPA_ERR_NO_DEVICE: return "no sm_100 device";
    case RPA_ERR_NOT_CONVERGED: return "not converged";
    case RPA_ERR_TOO_LARGE: return "problem exceeds a size limit of the entry point";
    case RPA_ERR_INTERNAL: return "internal error";
    default: return "unknown status";
  }
}

const char* rpa_b200_last_error(const rpa_b200_handle* h) { return h ? h->last_error.c_str() : "null handle"; }

int rpa_b200_last_timings(const rpa_b200_handle* h, double* out, int64_t n) try {
  if (!h || !out) return RPA_ERR_INVALID_ARG;
  for (int64_t i = 0; i < n && i < 6; ++i) out[i] = h->timings[i];
  return RPA_OK;
} catch (...) {
  return rpa::status_of_exception(nullptr);
}

int64_t rpa_b200_last_launches(const rpa_b200_handle* h) { return h ? h->launches : -1; }

int rpa_b200_set_stream(rpa_b200_handle* h, void* stream) try {
  if (!h) return RPA_ERR_INVALID_ARG;
  h->stream = stream ? static_cast<cudaStream_t>(stream) : h->own_stream;
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}

int rpa_b200_tune_logdet(rpa_b200_handle* h, int64_t NQ, int64_t NMat, int64_t* Nb2, int64_t* Tile, double* Ms) try {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
  if (NQ < 1 || NQ > (1 << 20) || NMat < 1 || NMat > (1 << 20))
    return fail(h, RPA_ERR_INVALID_ARG, "invalid tuning case NQ=%lld NMat=%lld", (long long)NQ, (long long)NMat);
  const int n = (int)NQ, nmat = (int)NMat;
  RPA_CUDA(h, ensure(h->Pi, (size_t)nmat * n * n * 8));
  if ((s = tune_uniform(h, n, nmat, static_cast<double*>(h->Pi.p), Ms))) return s;
  const rpa::LogdetPlan p = plan_for(h, n);
  if (Nb2) *Nb2 = p.nb2;
  if (Tile) *Tile = 32 * p.tile_w;
  h->launches = rpa::g_launches;
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}

int rpa_b200_set_logdet_plan(rpa_b200_handle* h, int64_t NQ, int64_t Nb2, int64_t Tile) try {
  if (!h || NQ < 1) return RPA_ERR_INVALID_ARG;
  const rpa::LogdetPlan p{(int)Nb2, (int)(Tile / 32)};
  if ((Nb2 != 128 && Nb2 != 256 && Nb2 != 512) || (Tile != 64 && Tile != 128) || !rpa::valid_logdet_plan(p))
    return fail(h, RPA_ERR_INVALID_ARG, "invalid log-det plan Nb2=%lld Tile=%lld", (long long)Nb2, (long long)Tile);
  h->logdet_plans[plan_bucket((int)std::min<int64_t>(NQ, 1 << 30))] = p;
  ++h->plans_version;
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}

int rpa_b200_get_logdet_plan(const rpa_b200_handle* h, int64_t NQ, int64_t* Nb2, int64_t* Tile) try {
  if (!h || NQ < 1) return RPA_ERR_INVALID_ARG;
  const rpa::LogdetPlan p = plan_for(h, (int)std::min<int64_t>(NQ, 1 << 30));
  if (Nb2) *Nb2 = p.nb2;
  if (Tile) *Tile = 32 * p.tile_w;
  return RPA_OK;
} catch (...) {
  return rpa::status_of_exception(nullptr);
}

int rpa_b200_set_workspace_limit(rpa_b200_handle* h, int64_t Bytes) try {
  if (!h || Bytes < 0) return RPA_ERR_INVALID_ARG;
  h->account.limit = (size_t)Bytes;
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}

int rpa_b200_workspace_bytes(const rpa_b200_handle* h, int64_t* Used, int64_t* Limit) try {
  if (!h) return RPA_ERR_INVALID_ARG;
  if (Used) *Used = (int64_t)h->account.used;
  if (Limit) *Limit = (int64_t)h->account.limit;
  return RPA_OK;
} catch (...) {
  return rpa::status_of_exception(nullptr);
}

int rpa_b200_selftest_wait_timeout(rpa_b200_handle* h, double LimitMs) try {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
  if (!(LimitMs > 0.0) || LimitMs > rpa::kWaitLimitNs * 1e-6)
    return fail(h, RPA_ERR_INVALID_ARG, "LimitMs must be in (0, %g]", rpa::kWaitLimitNs * 1e-6);
  RPA_CUDA(h, rpa::launch_wait_timeout_selftest(h->err_dev, (unsigned long long)(LimitMs * 1e6), h->stream));
  return check_device_error(h);
} catch (...) {
  return exception_status(h);
}

int rpa_b200_set_autotune(rpa_b200_handle* h, int64_t on) try {
  if (!h) return RPA_ERR_INVALID_ARG;
  h->autotune = on != 0;
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}

int rpa_b200_pi(rpa_b200_handle* h, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* R, int64_t ldR,
                const double* OccEnergies, const double* VirtEnergies, int64_t NFreqs, const double* Freqs,
                double alpha, int64_t prec, double* PiU, int64_t ldPi) try {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
  if ((s = check_arrays(h, {R, OccEnergies, VirtEnergies, Freqs, PiU}))) return s;
  Validated v;
  if ((s = validate_common(h, NQ, NOcc, NVirt, R, ldR, OccEnergies, VirtEnergies, NFreqs, Freqs, alpha, prec, v)))
    return s;
  if (!PiU || ldPi < NQ) return fail(h, RPA_ERR_INVALID_ARG, "PiU is NULL or ldPi < NQ");
  const double* Rd;
  int64_t ldd;
  if ((s = stage_R(h, v, R, ldR, &Rd, &ldd))) return s;
  RPA_CUDA(h, cudaEventRecord(h->ev[1], h->stream));
  if ((s = build_pi(h, v, Rd, ldd, alpha, prec))) return s;
  double* Pi = static_cast<double*>(h->Pi.p);
  RPA_CUDA(h, rpa::launch_symmetrize(Pi, NQ, NQ * NQ, v.NQ, v.K, h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[2], h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[3], h->stream));
  const bool dev = is_device_ptr(PiU);
  const cudaMemcpyKind kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (ldPi == NQ)
    RPA_CUDA(h, cudaMemcpyAsync(PiU, Pi, (size_t)v.K * NQ * NQ * 8, kind, h->stream));
  else
    for (int k = 0; k < v.K; ++k)
      RPA_CUDA(h, cudaMemcpy2DAsync(PiU + (int64_t)k * ldPi * NQ, (size_t)ldPi * 8, Pi + (int64_t)k * NQ * NQ,
                                    (size_t)NQ * 8, (size_t)NQ * 8, (size_t)NQ, kind, h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[4], h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  if ((s = check_device_error(h))) return s;
  finish_timings(h);
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}

int rpa_b200_ec_from_pi(rpa_b200_handle* h, int64_t NQ, int64_t NFreqs, const double* PiU, int64_t ldPi,
                        const double* FreqWeights, double* Ec, double* Eu) try {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
  if ((s = check_arrays(h, {PiU, FreqWeights}))) return s;
  if (NQ < 1 || NQ > (1 << 20) || NFreqs < 1 || NFreqs > 64 || ldPi < NQ || !PiU || !FreqWeights || !Ec)
    return fail(h, RPA_ERR_INVALID_ARG, "invalid argument to rpa_b200_ec_from_pi");
  std::vector<double> w;
  if ((s = fetch_small(h, FreqWeights, NFreqs, w))) return s;
  const int n = (int)NQ, K = (int)NFreqs;
  RPA_CUDA(h, ensure(h->Pi, (size_t)K * n * n * 8));
  double* Pi = static_cast<double*>(h->Pi.p);
  if (is_device_ptr(PiU)) {
    RPA_CUDA(h, rpa::launch_copy_lower(PiU, ldPi, ldPi * NQ, Pi, n, (int64_t)n * n, n, K, h->stream));
  } else if (ldPi == NQ) {
    RPA_CUDA(h, cudaMemcpyAsync(Pi, PiU, (size_t)K * n * n * 8, cudaMemcpyHostToDevice, h->stream));
  } else {
    for (int k = 0; k < K; ++k)
      RPA_CUDA(h, cudaMemcpy2DAsync(Pi + (int64_t)k * n * n, (size_t)n * 8, PiU + (int64_t)k * ldPi * NQ,
                                    (size_t)ldPi * 8, (size_t)n * 8, (size_t)n, cudaMemcpyHostToDevice, h->stream));
  }
  RPA_CUDA(h, cudaMemsetAsync(h->count_dev, 0, sizeof(int), h->stream));
  // only the lower triangle is read (a device input copies nothing else; the workspace's upper half holds leftovers)
  RPA_CUDA(h, rpa::launch_count_nonfinite_lower(Pi, n, (int64_t)n * n, n, K, h->count_dev, h->stream));
  int cnt = 0;
  RPA_CUDA(h, cudaMemcpyAsync(&cnt, h->count_dev, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  if (cnt) return fail(h, RPA_ERR_NONFINITE, "%d non-finite entries in Pi(u)", cnt);
  RPA_CUDA(h, cudaEventRecord(h->ev[1], h->stream));
  if ((s = energy_from_workspace(h, n, K, w, Ec, Eu))) return s;
  RPA_CUDA(h, cudaEventRecord(h->ev[4], h->stream));
  finish_timings(h);
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}

int rpa_b200_ec(rpa_b200_handle* h, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* R, int64_t ldR,
                const double* OccEnergies, const double* VirtEnergies, int64_t NFreqs, const double* Freqs,
                const double* FreqWeights, double alpha, int64_t prec, double* Ec, double* Eu) try {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
  if ((s = check_arrays(h, {R, OccEnergies, VirtEnergies, Freqs, FreqWeights}))) return s;
  Validated v;
  if ((s = validate_common(h, NQ, NOcc, NVirt, R, ldR, OccEnergies, VirtEnergies, NFreqs, Freqs, alpha, prec, v)))
    return s;
  if (!FreqWeights || !Ec) return fail(h, RPA_ERR_INVALID_ARG, "FreqWeights or Ec is NULL");
  if ((s = fetch_small(h, FreqWeights, NFreqs, v.weights))) return s;
  if (prec == RPA_PREC_SPLIT_BF16 && !is_device_ptr(R)) {
    // host R: staging overlapped with the Pi build, piece by piece
    if ((s = stage_eps(h, v))) return s;
    RPA_CUDA(h, cudaEventRecord(h->ev[1], h->stream));
    s = build_pi_pipelined(h, v, R, ldR, alpha);
    if (s == RPA_OK) {
      int cnt = 0;
      RPA_CUDA(h, cudaMemcpyAsync(&cnt, h->count_dev, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
      const int se = energy_from_workspace(h, v.NQ, v.K, v.weights, Ec, Eu);
      RPA_CUDA(h, cudaStreamSynchronize(h->stream));
      if (cnt) return fail(h, RPA_ERR_NONFINITE, "%d non-finite entries in the Cholesky vectors", cnt);
      if (se) return se;
      RPA_CUDA(h, cudaEventRecord(h->ev[4], h->stream));
      finish_timings(h);
      return RPA_OK;
    }
    if (s != 1) return s;  // 1: frequencies need several groups, stage R whole instead
  }
  const double* Rd;
  int64_t ldd;
  if ((s = stage_R(h, v, R, ldR, &Rd, &ldd))) return s;
  RPA_CUDA(h, cudaEventRecord(h->ev[1], h->stream));
  if ((s = build_pi(h, v, Rd, ldd, alpha, prec))) return s;
  if ((s = energy_from_workspace(h, v.NQ, v.K, v.weights, Ec, Eu))) return s;
  RPA_CUDA(h, cudaEventRecord(h->ev[4], h->stream));
  finish_timings(h);
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}


int rpa_b200_dring_t2(rpa_b200_handle* h, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* R, int64_t ldR,
                      const double* OccEnergies, const double* VirtEnergies, int64_t NFreqs, const double* Freqs,
                      const double* FreqWeights, double alpha, int64_t prec, int64_t GuessNVecs, const double* Omega,
                      uint64_t seed, double SmallEigenvalsCutoff, double CutoffThresh, int64_t CutoffType,
                      double* CommonThresh, int64_t MaxNVecsT2, double* A, double* U, int64_t ldU,
                      int64_t* NVecsT2, double* EigRPA, double* Ec) try {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
  if ((s = check_arrays(h, {R, OccEnergies, VirtEnergies, Freqs, FreqWeights, Omega, A, U}))) return s;
  Validated v;
  if ((s = validate_common(h, NQ, NOcc, NVirt, R, ldR, OccEnergies, VirtEnergies, NFreqs, Freqs, alpha, prec, v)))
    return s;
  if (!FreqWeights || !CommonThresh || !A || !U || !NVecsT2 || !EigRPA || MaxNVecsT2 < 1 || GuessNVecs < 1 ||
      ldU < NOcc * NVirt)
    return fail(h, RPA_ERR_INVALID_ARG, "invalid T2 output arguments");
  if (CutoffType < 0 || CutoffType > 3) return fail(h, RPA_ERR_INVALID_ARG, "unknown T2 cutoff type");
  if ((s = fetch_small(h, FreqWeights, NFreqs, v.weights))) return s;
  const double* Rd;
  int64_t ldd;
  if ((s = stage_R(h, v, R, ldR, &Rd, &ldd))) return s;
  RPA_CUDA(h, cudaEventRecord(h->ev[1], h->stream));
  if ((s = build_pi(h, v, Rd, ldd, alpha, prec))) return s;
  double ec = 0.0;
  if ((s = energy_from_workspace(h, v.NQ, v.K, v.weights, &ec, nullptr))) return s;  // leaves L_k in h->Pi
  if (Ec) *Ec = ec;

  T2Ctx c;
  c.NQ = v.NQ;
  c.K = v.K;
  c.nov = v.nov;
  c.R = Rd;
  c.ldR = ldd;
  c.alpha = alpha;
  for (int k = 0; k < v.K; ++k) {
    c.u2.push_back(v.freqs[k] * v.freqs[k]);
    c.w.push_back(v.weights[k]);
  }
  const int G = (int)GuessNVecs;
  const int64_t nov = v.nov;
  size_t freeB = 0, totalB = 0;
  RPA_CUDA(h, cudaMemGetInfo(&freeB, &totalB));
  const size_t zAll = (size_t)v.K * v.NQ * nov * 8;
  const size_t fixed = (size_t)nov * G * 8 * 3 + (size_t)G * G * 8 * 2;
  c.z_resident = zAll + fixed < (size_t)(0.8 * (double)(freeB + h->tZ.bytes));
  c.zk = c.z_resident ? v.K : std::max(1, (int)std::min<size_t>(v.K, (size_t)(0.4 * freeB) / ((size_t)v.NQ * nov * 8)));
  RPA_CUDA(h, ensure(h->tZ, (size_t)c.zk * v.NQ * nov * 8 * (c.z_resident ? 1 : 1)));
  if (c.z_resident) RPA_CUDA(h, ensure(h->tZ, zAll));
  RPA_CUDA(h, ensure(h->tP, (size_t)c.zk * v.NQ * G * 8));
  RPA_CUDA(h, ensure(h->tOm, (size_t)nov * G * 8));
  RPA_CUDA(h, ensure(h->tIOm, (size_t)nov * G * 8));
  RPA_CUDA(h, ensure(h->tS, (size_t)G * G * 8));
  RPA_CUDA(h, ensure(h->tV, (size_t)G * G * 8));
  RPA_CUDA(h, ensure(h->tSmall, (size_t)std::max<int64_t>(G, 64) * 8 + 64));
  RPA_CUDA(h, ensure(h->tPerm, (size_t)G * sizeof(int)));
  if (c.z_resident)
    for (int g0 = 0; g0 < v.K; g0 += c.zk)
      if ((s = build_z_group(h, c, g0, std::min(c.zk, v.K - g0), static_cast<double*>(h->tZ.p)))) return s;
  if (prec == RPA_PREC_SPLIT_BF16 && c.z_resident)
    if ((s = prepare_split_z(h, c))) return s;

  // guess vectors (rpa_CC_Doubles.f90:746-763): given, or uniform [-1/2, 1/2) from the seed
  double* Om = static_cast<double*>(h->tOm.p);
  double* IOm = static_cast<double*>(h->tIOm.p);
  if (Omega) {
    RPA_CUDA(h, cudaMemcpyAsync(Om, Omega, (size_t)nov * G * 8, cudaMemcpyDefault, h->stream));
    if ((s = screen_result(h, Om, nov, nov, G, "the given guess vectors"))) return s;
  } else {
    RPA_CUDA(h, rpa::launch_fill_uniform(Om, nov, G, nov, seed, h->stream));
  }
  if ((s = normalize_columns(h, Om, nov, G))) return s;
  if ((s = apply_I(h, c, Om, G, IOm))) return s;
  if ((s = normalize_columns(h, IOm, nov, G))) return s;
  // S = IOm^T IOm, eigenvalues above the linear-dependency cutoff (771-795)
  double* S = static_cast<double*>(h->tS.p);
  double* Vs = static_cast<double*>(h->tV.p);
  RPA_CUDA(h, rpa::launch_gemm_f64(gemm_tn(G, G, nov, IOm, nov, IOm, nov, S, G), h->stream));
  RPA_CUDA(h, rpa::launch_symmetrize_avg(S, G, G, h->stream));
  std::vector<double> sval;
  std::vector<int> sord;
  if ((s = sym_eig(h, S, Vs, G, sval, sord))) return s;
  int NT = 0;
  for (int i = G - 1; i >= 0; --i) {
    if (sval[sord[i]] > SmallEigenvalsCutoff) ++NT;
    else break;
  }
  if (NT == 0) return fail(h, RPA_ERR_NOT_CONVERGED, "no T2 guess direction above the linear-dependency cutoff");
  std::vector<int> wcols(NT);
  std::vector<double> wscale(NT);
  for (int j = 0; j < NT; ++j) {
    wcols[j] = sord[G - NT + j];
    wscale[j] = 1.0 / std::sqrt(sval[wcols[j]]);
  }
  RPA_CUDA(h, ensure(h->tW, (size_t)G * NT * 8));
  RPA_CUDA(h, ensure(h->tT, (size_t)nov * NT * 8));
  double* W = static_cast<double*>(h->tW.p);
  double* T = static_cast<double*>(h->tT.p);
  if ((s = gather(h, Vs, G, W, wcols, &wscale))) return s;
  RPA_CUDA(h, rpa::launch_gemm_f64(gemm_nn((int)nov, NT, G, IOm, nov, W, G, T, nov), h->stream));
  // Rayleigh-Ritz: TIT = T^T I T (rpa_CC_MIM_v5, 425-488), eigenpairs (797-808)
  double* IT = Om;  // guess vectors no longer needed
  if ((s = apply_I(h, c, T, NT, IT))) return s;
  RPA_CUDA(h, ensure(h->tTIT, (size_t)NT * NT * 8));
  RPA_CUDA(h, ensure(h->tVt, (size_t)NT * NT * 8));
  double* TIT = static_cast<double*>(h->tTIT.p);
  double* Vt = static_cast<double*>(h->tVt.p);
  RPA_CUDA(h, rpa::launch_gemm_f64(gemm_tn(NT, NT, nov, T, nov, IT, nov, TIT, NT), h->stream));
  RPA_CUDA(h, rpa::launch_symmetrize_avg(TIT, NT, NT, h->stream));
  std::vector<double> aval;
  std::vector<int> aord;
  if ((s = sym_eig(h, TIT, Vt, NT, aval, aord))) return s;
  std::vector<double> Aall(NT);
  for (int i = 0; i < NT; ++i) {
    const double a = aval[aord[i]];
    Aall[i] = 0.5 * (a / (a + 1.0));
  }
  // eigenvalue cutoff (rpa_THC_CC_T2, 855-945); supersystem when *CommonThresh < 0
  double K = 0.0;
  if (*CommonThresh < 0.0) {
    switch (CutoffType) {
      case 0: K = CutoffThresh; break;
      case 1: {
        double mx = 0.0;
        for (double a : Aall) mx = std::max(mx, std::fabs(a));
        K = CutoffThresh * mx;
        break;
      }
      case 2: K = CutoffThresh / (double)(NOcc * 2); break;
      case 3: {
        K = 0.0;
        for (int i = 0; i + 1 < NT; ++i) {
          double sum = 0.0;
          for (int j = i + 1; j < NT; ++j) sum += Aall[j];
          if (std::fabs(sum) < CutoffThresh) {
            K = std::fabs(Aall[i + 1]);
            break;
          }
        }
        break;
      }
    }
  } else {
    K = *CommonThresh;
  }
  int keep = 0;
  for (int i = 0; i < NT; ++i) {
    if (std::fabs(Aall[i]) > K) keep = i + 1;
    else break;
  }
  if (keep == 0) return fail(h, RPA_ERR_NOT_CONVERGED, "Invalid T2CutoffThresh: no eigenvectors left after cutoff");
  if (keep > MaxNVecsT2) return fail(h, RPA_ERR_INVALID_ARG, "%d T2 eigenvectors exceed MaxNVecsT2", keep);
  std::vector<int> tcols(aord.begin(), aord.begin() + keep);
  if ((s = gather(h, Vt, NT, W, tcols, nullptr))) return s;  // W reused: NT x keep
  RPA_CUDA(h, ensure(h->tU, (size_t)nov * keep * 8));
  double* Ud = static_cast<double*>(h->tU.p);
  RPA_CUDA(h, rpa::launch_gemm_f64(gemm_nn((int)nov, keep, NT, T, nov, W, NT, Ud, nov), h->stream));
  // EigRPA(mu) = 2 A_mu |R U_mu|^2 (rpa_T2_EigRPA, 987-1009)
  RPA_CUDA(h, ensure(h->tRU, (size_t)v.NQ * keep * 8));
  double* RU = static_cast<double*>(h->tRU.p);
  RPA_CUDA(h, rpa::launch_gemm_f64(gemm_nn(v.NQ, keep, nov, Rd, ldd, Ud, nov, RU, v.NQ), h->stream));
  double* nrm = static_cast<double*>(h->tSmall.p);
  RPA_CUDA(h, rpa::launch_col_sqnorm(RU, v.NQ, keep, v.NQ, nrm, h->stream));
  std::vector<double> n2(keep);
  RPA_CUDA(h, cudaMemcpyAsync(n2.data(), nrm, (size_t)keep * 8, cudaMemcpyDeviceToHost, h->stream));
  const cudaMemcpyKind kind = is_device_ptr(U) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  RPA_CUDA(h, cudaMemcpy2DAsync(U, (size_t)ldU * 8, Ud, (size_t)nov * 8, (size_t)nov * 8, (size_t)keep, kind,
                                h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[4], h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  if ((s = check_device_error(h))) return s;
  for (int i = 0; i < keep; ++i) {
    A[i] = Aall[i];
    EigRPA[i] = 2.0 * Aall[i] * n2[i];
  }
  *NVecsT2 = keep;
  if (*CommonThresh < 0.0) *CommonThresh = K;
  finish_timings(h);
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}

// Split-BF16 pair contraction on the tensor cores: *out = sum_{i>=j} (2 - delta_ij) sum_{Q,mu} B_mu
// W_ij W_ji with W_ij = R_i U_j^T and W_ji = R_j U2_i^T (U2 null: U).  R, U (and U2) are split into
// bf16 hi/lo rows once per call; the unit partials are summed in a fixed order (deterministic).
static int sosex_split(rpa_b200_handle* h, const double* R, int64_t ldR, int NQ, int no, int nv, const double* U,
                int64_t ldU, const double* U2, int64_t ldU2, int NT, const double* Bd, double* out) {
  const int nvp = rpa::sosex_tc_nvp(nv);
  const size_t P = (size_t)no * nvp;
  const size_t rb = (size_t)NQ * P * 2, ub = (size_t)NT * P * 2;  // bytes of one bf16 part
  RPA_CUDA(h, ensure(h->sxR, 2 * rb + 256));
  RPA_CUDA(h, ensure(h->sxU, (U2 ? 4 : 2) * ub + 256));
  auto* Rh = static_cast<__nv_bfloat16*>(h->sxR.p);
  auto* Rl = Rh + (size_t)NQ * P;
  auto* Uh = static_cast<__nv_bfloat16*>(h->sxU.p);
  auto* Ul = Uh + (size_t)NT * P;
  auto* U2h = U2 ? Ul + (size_t)NT * P : Uh;
  auto* U2l = U2 ? U2h + (size_t)NT * P : Ul;
  RPA_CUDA(h, rpa::launch_split_rows(R, ldR, NQ, no, nv, Rh, Rl, h->stream));
  RPA_CUDA(h, rpa::launch_split_cols(U, ldU, NT, no, nv, Uh, Ul, h->stream));
  if (U2) RPA_CUDA(h, rpa::launch_split_cols(U2, ldU2, NT, no, nv, U2h, U2l, h->stream));
  CUtensorMap maps[6];
  int s;
  if ((s = encode_map(h, &maps[0], Rh, (int64_t)P, NQ, 1, (int64_t)P, 128))) return s;
  if ((s = encode_map(h, &maps[1], Rl, (int64_t)P, NQ, 1, (int64_t)P, 128))) return s;
  if ((s = encode_map(h, &maps[2], Uh, (int64_t)P, NT, 1, (int64_t)P, 128))) return s;
  if ((s = encode_map(h, &maps[3], Ul, (int64_t)P, NT, 1, (int64_t)P, 128))) return s;
  if ((s = encode_map(h, &maps[4], U2h, (int64_t)P, NT, 1, (int64_t)P, 128))) return s;
  if ((s = encode_map(h, &maps[5], U2l, (int64_t)P, NT, 1, (int64_t)P, 128))) return s;
  rpa::SosexTcArgs a{};
  a.NQ = NQ;
  a.no = no;
  a.nvp = nvp;
  a.NT = NT;
  a.nqt = (NQ + 127) / 128;
  a.nmt = (NT + 127) / 128;
  const int64_t units = rpa::sosex_tc_units(NQ, no, NT);
  if (units > (int64_t)INT32_MAX) return fail(h, RPA_ERR_TOO_LARGE, "exchange contraction too large (%lld units)",
                                              (long long)units);
  a.nunits = (int)units;
  a.same = U2 ? 0 : 1;
  a.seg_chunks = h->sosex_seg;
  a.Bmu = Bd;
  a.err = h->err_dev;
  const int64_t np = rpa::sosex_tc_partials(NQ, no, NT);
  const int64_t chunk = 4096;
  const int64_t nsum = (np + chunk - 1) / chunk;
  RPA_CUDA(h, ensure(h->sxP, (size_t)(np + nsum) * 8 + 256));
  a.partial = static_cast<double*>(h->sxP.p);
  double* sums = a.partial + np;
  RPA_CUDA(h, rpa::launch_sosex_split_bf16(maps, a, h->num_sms, h->stream));
  int64_t nout = 0;
  RPA_CUDA(h, rpa::launch_chunk_sum(a.partial, np, chunk, sums, &nout, h->stream));
  std::vector<double> hs((size_t)nout);
  RPA_CUDA(h, cudaMemcpyAsync(hs.data(), sums, (size_t)nout * 8, cudaMemcpyDeviceToHost, h->stream));
  if ((s = check_device_error(h))) return s;  // also synchronises the stream
  dd acc{0.0, 0.0};
  for (double x : hs) acc = rpa::dd_add(acc, x);
  *out = acc.hi + acc.lo;
  return RPA_OK;
}

int rpa_b200_exchange_sosex(rpa_b200_handle* h, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* R,
                            int64_t ldR, int64_t NVecsT2, const double* U, int64_t ldU, const double* A, double Alpha,
                            int64_t S2Operator, int64_t Prec, double* Ex) try {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
  if ((s = check_arrays(h, {R, U, A}))) return s;
  const int64_t nov = NOcc * NVirt;
  if (NQ < 1 || NOcc < 1 || NVirt < 1 || NVecsT2 < 1 || ldR < NQ || ldU < nov || !R || !U || !A || !Ex ||
      (Prec != RPA_PREC_FP64 && Prec != RPA_PREC_SPLIT_BF16))
    return fail(h, RPA_ERR_INVALID_ARG, "invalid argument to rpa_b200_exchange_sosex");
  const int NT = (int)NVecsT2;
  std::vector<double> Ah;
  if ((s = fetch_small(h, A, NT, Ah))) return s;
  std::vector<double> B(NT);
  for (int m = 0; m < NT; ++m) {
    B[m] = S2Operator ? Ah[m] / (1.0 - 4.0 * Ah[m] * Ah[m]) : Ah[m];
    if (!std::isfinite(B[m])) return fail(h, RPA_ERR_NONFINITE, "non-finite T2 eigenvalue");
  }
  // stage R and U on the device
  const double* Rd = R;
  int64_t ldr = ldR;
  if (!is_device_ptr(R)) {
    RPA_CUDA(h, ensure(h->R, (size_t)NQ * nov * 8));
    RPA_CUDA(h, cudaMemcpy2DAsync(h->R.p, (size_t)NQ * 8, R, (size_t)ldR * 8, (size_t)NQ * 8, (size_t)nov,
                                  cudaMemcpyHostToDevice, h->stream));
    Rd = static_cast<const double*>(h->R.p);
    ldr = NQ;
  }
  const double* Ud = U;
  int64_t ldu = ldU;
  if (!is_device_ptr(U)) {
    RPA_CUDA(h, ensure(h->tU, (size_t)nov * NT * 8));
    RPA_CUDA(h, cudaMemcpy2DAsync(h->tU.p, (size_t)nov * 8, U, (size_t)ldU * 8, (size_t)nov * 8, (size_t)NT,
                                  cudaMemcpyHostToDevice, h->stream));
    Ud = static_cast<const double*>(h->tU.p);
    ldu = nov;
  }
  const int64_t np = rpa::sosex_partials((int)NQ, (int)NOcc, NT);
  RPA_CUDA(h, ensure(h->tSmall, (size_t)(NT + np) * 8));
  double* Bd = static_cast<double*>(h->tSmall.p);
  double* part = Bd + NT;
  RPA_CUDA(h, cudaMemcpyAsync(Bd, B.data(), (size_t)NT * 8, cudaMemcpyHostToDevice, h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[1], h->stream));
  if (Prec == RPA_PREC_SPLIT_BF16) {
    double sum = 0.0;
    if ((s = sosex_split(h, Rd, ldr, (int)NQ, (int)NOcc, (int)NVirt, Ud, ldu, nullptr, 0, NT, Bd, &sum))) return s;
    RPA_CUDA(h, cudaEventRecord(h->ev[2], h->stream));
    RPA_CUDA(h, cudaEventRecord(h->ev[3], h->stream));
    RPA_CUDA(h, cudaEventRecord(h->ev[4], h->stream));
    if ((s = finite_or_fail(h, {sum}, "exchange energy"))) return s;
    *Ex = -Alpha * sum;
    finish_timings(h);
    return RPA_OK;
  }
  int64_t npart = 0;
  RPA_CUDA(h, rpa::launch_sosex(Rd, ldr, (int)NQ, (int)NOcc, (int)NVirt, Ud, ldu, nullptr, 0, NT, Bd, part, &npart,
                                h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[2], h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[3], h->stream));
  std::vector<double> hp((size_t)npart);
  RPA_CUDA(h, cudaMemcpyAsync(hp.data(), part, (size_t)npart * 8, cudaMemcpyDeviceToHost, h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[4], h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  dd acc{0.0, 0.0};
  for (double x : hp) acc = rpa::dd_add(acc, x);
  if ((s = finite_or_fail(h, {acc.hi}, "exchange energy"))) return s;
  *Ex = -Alpha * (acc.hi + acc.lo);
  finish_timings(h);
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}

// MBPT3 exchange (rpa_CC_Exchange_MBPT3_1, src/rpa/rpa_CC_Exchange.f90:232-272, with rpa_CC_Ukl :177,
// rpa_CC_Dkl and rpa_CC_TrXK :275).  The reference solves B^T X + X B = A by a real Schur form and
// DTRSYL (real_Lyapunov, src/linear-algebra/real_linalg.f90:125-171).  Here the operator is split
// into its symmetric part S = (B + B^T)/2, inverted exactly through S = Q diag(mu) Q^T
// ((S Y + Y S)_mn = mu_m + mu_n in the eigenbasis), and the antisymmetric part 2 U_mn (A_n - A_m),
// which is small because |A| << 1; the residual-correction iteration
//   X <- X + Q [(Q^T (A - B^T X - X B) Q)_mn / (mu_m + mu_n)] Q^T
// contracts by about three orders of magnitude per step.  All matrix products are FP64 DMMA GEMMs.
int rpa_b200_exchange_mbpt3(rpa_b200_handle* h, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* R,
                            int64_t ldR, const double* OccEnergies, const double* VirtEnergies, int64_t NVecsT2,
                            const double* U, int64_t ldU, const double* A, int64_t Prec, double* Ex, double* X,
                            int64_t ldX) try {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
  if ((s = check_arrays(h, {R, OccEnergies, VirtEnergies, U, A, X}))) return s;
  const int64_t nov = NOcc * NVirt;
  if (NQ < 1 || NOcc < 1 || NVirt < 1 || NVecsT2 < 1 || ldR < NQ || ldU < nov || !R || !U || !A || !Ex ||
      !OccEnergies || !VirtEnergies || (X && ldX < NVecsT2) || (Prec != RPA_PREC_FP64 && Prec != RPA_PREC_SPLIT_BF16))
    return fail(h, RPA_ERR_INVALID_ARG, "invalid argument to rpa_b200_exchange_mbpt3");
  if (NQ > INT32_MAX || nov > INT32_MAX || NVecsT2 > 65535)
    return fail(h, RPA_ERR_TOO_LARGE, "rpa_b200_exchange_mbpt3: dimensions too large");
  const int NT = (int)NVecsT2;
  std::vector<double> Ah, eo, ev;
  if ((s = fetch_small(h, A, NT, Ah)) || (s = fetch_small(h, OccEnergies, NOcc, eo)) ||
      (s = fetch_small(h, VirtEnergies, NVirt, ev)))
    return s;
  std::vector<double> Dh((size_t)nov);
  for (int64_t i = 0; i < NOcc; ++i)
    for (int64_t a = 0; a < NVirt; ++a) Dh[(size_t)(a + NVirt * i)] = ev[a] - eo[i];
  for (double x : Ah)
    if (!std::isfinite(x)) return fail(h, RPA_ERR_NONFINITE, "non-finite T2 eigenvalue");
  for (double x : Dh)
    if (!std::isfinite(x)) return fail(h, RPA_ERR_NONFINITE, "non-finite orbital energy");

  const double* Rd = R;
  int64_t ldr = ldR;
  if (!is_device_ptr(R)) {
    RPA_CUDA(h, ensure(h->R, (size_t)NQ * nov * 8));
    RPA_CUDA(h, cudaMemcpy2DAsync(h->R.p, (size_t)NQ * 8, R, (size_t)ldR * 8, (size_t)NQ * 8, (size_t)nov,
                                  cudaMemcpyHostToDevice, h->stream));
    Rd = static_cast<const double*>(h->R.p);
    ldr = NQ;
  }
  const double* Ud = U;
  int64_t ldu = ldU;
  if (!is_device_ptr(U)) {
    RPA_CUDA(h, ensure(h->tU, (size_t)nov * NT * 8));
    RPA_CUDA(h, cudaMemcpy2DAsync(h->tU.p, (size_t)nov * 8, U, (size_t)ldU * 8, (size_t)nov * 8, (size_t)NT,
                                  cudaMemcpyHostToDevice, h->stream));
    Ud = static_cast<const double*>(h->tU.p);
    ldu = nov;
  }
  // workspace: 8 NT x NT matrices, R U (NQ x NT), U X (nov x NT), D, A, mu, partials
  const size_t nn = (size_t)NT * NT;
  const int64_t np = rpa::sosex_partials((int)NQ, (int)NOcc, NT);
  const size_t words = 8 * nn + (size_t)NQ * NT + (size_t)nov * NT + (size_t)nov + 3 * (size_t)NT + (size_t)np + 8;
  RPA_CUDA(h, ensure(h->xM, words * 8));
  RPA_CUDA(h, ensure(h->tSmall, (size_t)std::max<int64_t>(NT, 256) * 8 + 64));
  RPA_CUDA(h, ensure(h->tPerm, (size_t)NT * sizeof(int)));
  double* w = static_cast<double*>(h->xM.p);
  double* Ukl = w;
  double* Dkl = Ukl + nn;
  double* Am = Dkl + nn;
  double* Bm = Am + nn;
  double* Sm = Bm + nn;  // symmetric part; diagonalised in place
  double* Q = Sm + nn;
  double* Xd = Q + nn;
  double* Res = Xd + nn;
  double* RU = Res + nn;
  double* UX = RU + (size_t)NQ * NT;
  double* Dd = UX + (size_t)nov * NT;
  double* Ad = Dd + nov;
  double* mud = Ad + NT;
  double* ones = mud + NT;
  double* part = ones + NT;
  int* bad = h->count_dev;
  RPA_CUDA(h, cudaMemcpyAsync(Dd, Dh.data(), (size_t)nov * 8, cudaMemcpyHostToDevice, h->stream));
  RPA_CUDA(h, cudaMemcpyAsync(Ad, Ah.data(), (size_t)NT * 8, cudaMemcpyHostToDevice, h->stream));
  {
    std::vector<double> one((size_t)NT, 1.0);
    RPA_CUDA(h, cudaMemcpyAsync(ones, one.data(), (size_t)NT * 8, cudaMemcpyHostToDevice, h->stream));
    RPA_CUDA(h, cudaStreamSynchronize(h->stream));  // host vectors must outlive their copies
  }
  RPA_CUDA(h, cudaEventRecord(h->ev[1], h->stream));

  // Ukl = (R U)^T (R U), Dkl = U^T diag(D) U, then the A, B and S matrices
  RPA_CUDA(h, rpa::launch_gemm_f64(gemm_nn((int)NQ, NT, nov, Rd, ldr, Ud, ldu, RU, NQ), h->stream));
  RPA_CUDA(h, rpa::launch_gemm_f64(gemm_tn(NT, NT, NQ, RU, NQ, RU, NQ, Ukl, NT), h->stream));
  {
    rpa::GemmF64Args g = gemm_tn(NT, NT, nov, Ud, ldu, Ud, ldu, Dkl, NT);
    g.kscale = Dd;
    RPA_CUDA(h, rpa::launch_gemm_f64(g, h->stream));
  }
  RPA_CUDA(h, rpa::launch_mbpt3_build(Ukl, Dkl, Ad, NT, Am, Bm, Sm, h->stream));
  std::vector<double> mu;
  std::vector<int> order;
  if ((s = sym_eig(h, Sm, Q, NT, mu, order))) return s;
  RPA_CUDA(h, cudaMemcpyAsync(mud, mu.data(), (size_t)NT * 8, cudaMemcpyHostToDevice, h->stream));
  RPA_CUDA(h, cudaMemsetAsync(bad, 0, sizeof(int), h->stream));

  // residual-correction iteration, X_0 = 0
  double* red = static_cast<double*>(h->tSmall.p);
  RPA_CUDA(h, cudaMemsetAsync(Xd, 0, nn * 8, h->stream));
  auto sqnorm = [&](const double* M, double& out) -> int {
    double od[2];
    RPA_CUDA(h, rpa::launch_offdiag(M, NT, NT, red, h->stream));
    RPA_CUDA(h, cudaMemcpyAsync(od, red, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    RPA_CUDA(h, cudaStreamSynchronize(h->stream));
    out = od[0] + od[1];
    return RPA_OK;
  };
  double a2 = 0.0;
  if ((s = sqnorm(Am, a2))) return s;
  bool converged = (a2 == 0.0);
  double r2 = a2;
  for (int it = 0; it < 60 && !converged; ++it) {
    // Res = A - B^T X - X B
    RPA_CUDA(h, cudaMemcpyAsync(Res, Am, nn * 8, cudaMemcpyDeviceToDevice, h->stream));
    if (it > 0) {
      rpa::GemmF64Args g1 = gemm_tn(NT, NT, NT, Bm, NT, Xd, NT, Res, NT);
      g1.alpha = -1.0;
      g1.beta = 1.0;
      RPA_CUDA(h, rpa::launch_gemm_f64(g1, h->stream));
      rpa::GemmF64Args g2 = gemm_nn(NT, NT, NT, Xd, NT, Bm, NT, Res, NT);
      g2.alpha = -1.0;
      g2.beta = 1.0;
      RPA_CUDA(h, rpa::launch_gemm_f64(g2, h->stream));
      if ((s = sqnorm(Res, r2))) return s;
      if (!std::isfinite(r2) || r2 > 1e4 * a2)
        return fail(h, RPA_ERR_NOT_CONVERGED, "MBPT3 Lyapunov iteration diverged (|res|/|A| = %.3e)",
                    std::sqrt(r2 / a2));
      if (r2 <= 1e-26 * a2) {
        converged = true;
        break;
      }
    }
    // Y = Q^T Res Q / (mu_m + mu_n);  X += Q Y Q^T   (Sm and Ukl serve as scratch)
    RPA_CUDA(h, rpa::launch_gemm_f64(gemm_tn(NT, NT, NT, Q, NT, Res, NT, Sm, NT), h->stream));
    RPA_CUDA(h, rpa::launch_gemm_f64(gemm_nn(NT, NT, NT, Sm, NT, Q, NT, Ukl, NT), h->stream));
    RPA_CUDA(h, rpa::launch_lyap_scale(Ukl, mud, NT, bad, h->stream));
    RPA_CUDA(h, rpa::launch_gemm_f64(gemm_nn(NT, NT, NT, Q, NT, Ukl, NT, Sm, NT), h->stream));
    rpa::GemmF64Args g3 = gemm_nn(NT, NT, NT, Sm, NT, Q, NT, Xd, NT);
    g3.b_k = NT;  // Q^T
    g3.b_n = 1;
    g3.beta = 1.0;
    RPA_CUDA(h, rpa::launch_gemm_f64(g3, h->stream));
    if (it == 0) {
      int nbad = 0;
      RPA_CUDA(h, cudaMemcpyAsync(&nbad, bad, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
      RPA_CUDA(h, cudaStreamSynchronize(h->stream));
      if (nbad)
        return fail(h, RPA_ERR_NOT_CONVERGED,
                    "MBPT3 Lyapunov solve: symmetric part of B is not positive definite (%d pairs)", nbad);
    }
  }
  if (!converged)
    return fail(h, RPA_ERR_NOT_CONVERGED, "MBPT3 Lyapunov iteration did not converge (|res|/|A| = %.3e)",
                std::sqrt(r2 / a2));

  // Tr(XK): W_ij from U, W_ji from U X
  RPA_CUDA(h, rpa::launch_gemm_f64(gemm_nn((int)nov, NT, NT, Ud, ldu, Xd, NT, UX, nov), h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[2], h->stream));
  int64_t npart = 0;
  double split_sum = 0.0;
  if (Prec == RPA_PREC_SPLIT_BF16) {
    if ((s = sosex_split(h, Rd, ldr, (int)NQ, (int)NOcc, (int)NVirt, Ud, ldu, UX, nov, NT, ones, &split_sum)))
      return s;
  } else {
    RPA_CUDA(h, rpa::launch_sosex(Rd, ldr, (int)NQ, (int)NOcc, (int)NVirt, Ud, ldu, UX, nov, NT, ones, part, &npart,
                                  h->stream));
  }
  RPA_CUDA(h, cudaEventRecord(h->ev[3], h->stream));
  std::vector<double> hp((size_t)npart);
  if (npart) RPA_CUDA(h, cudaMemcpyAsync(hp.data(), part, (size_t)npart * 8, cudaMemcpyDeviceToHost, h->stream));
  if (X) {
    if (is_device_ptr(X))
      RPA_CUDA(h, cudaMemcpy2DAsync(X, (size_t)ldX * 8, Xd, (size_t)NT * 8, (size_t)NT * 8, (size_t)NT,
                                    cudaMemcpyDeviceToDevice, h->stream));
    else
      RPA_CUDA(h, cudaMemcpy2DAsync(X, (size_t)ldX * 8, Xd, (size_t)NT * 8, (size_t)NT * 8, (size_t)NT,
                                    cudaMemcpyDeviceToHost, h->stream));
  }
  RPA_CUDA(h, cudaEventRecord(h->ev[4], h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  dd acc{split_sum, 0.0};
  for (double x : hp) acc = rpa::dd_add(acc, x);
  if ((s = finite_or_fail(h, {acc.hi}, "MBPT3 exchange energy"))) return s;
  *Ex = -(acc.hi + acc.lo);
  finish_timings(h);
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}

// Replaces real_EVD (src/linear-algebra/real_linalg.f90:1501-1559, LAPACK dsyevd) with
// ComputeEigenvecs = .true.: eigenvalues ascending, A overwritten by the eigenvectors.
int rpa_b200_syevd(rpa_b200_handle* h, int64_t N, double* A, int64_t ldA, double* Eigenvals) try {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
  if ((s = check_arrays(h, {A, Eigenvals}))) return s;
  if (N < 1 || ldA < N || !A || !Eigenvals) return fail(h, RPA_ERR_INVALID_ARG, "invalid argument to rpa_b200_syevd");
  if (N > 46340) return fail(h, RPA_ERR_TOO_LARGE, "rpa_b200_syevd: N too large");
  const int n = (int)N;
  const size_t nn = (size_t)n * n;
  RPA_CUDA(h, ensure(h->eA, nn * 8));
  RPA_CUDA(h, ensure(h->eZ, nn * 8));
  double* Ad = static_cast<double*>(h->eA.p);
  double* Zd = static_cast<double*>(h->eZ.p);
  const bool dev = is_device_ptr(A);
  RPA_CUDA(h, cudaMemcpy2DAsync(Ad, (size_t)n * 8, A, (size_t)ldA * 8, (size_t)n * 8, (size_t)n,
                                dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, h->stream));
  RPA_CUDA(h, cudaMemsetAsync(h->count_dev, 0, sizeof(int), h->stream));
  RPA_CUDA(h, rpa::launch_count_nonfinite(Ad, (int64_t)nn, h->count_dev, h->stream));
  int cnt = 0;
  RPA_CUDA(h, cudaMemcpyAsync(&cnt, h->count_dev, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  if (cnt) return fail(h, RPA_ERR_NONFINITE, "%d non-finite entries in A", cnt);
  RPA_CUDA(h, cudaEventRecord(h->ev[1], h->stream));
  std::vector<double> ev;
  std::vector<int> order;
  if ((s = sym_eig(h, Ad, Zd, n, ev, order))) return s;
  RPA_CUDA(h, ensure(h->tPerm, (size_t)n * sizeof(int)));
  if ((s = gather(h, Zd, n, Ad, order, nullptr))) return s;  // columns in ascending order
  RPA_CUDA(h, cudaEventRecord(h->ev[2], h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[3], h->stream));
  RPA_CUDA(h, cudaMemcpy2DAsync(A, (size_t)ldA * 8, Ad, (size_t)n * 8, (size_t)n * 8, (size_t)n,
                                dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, h->stream));
  std::vector<double> sorted(n);
  for (int i = 0; i < n; ++i) sorted[i] = ev[order[i]];
  RPA_CUDA(h, cudaMemcpyAsync(Eigenvals, sorted.data(), (size_t)n * 8,
                              is_device_ptr(Eigenvals) ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost, h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[4], h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  finish_timings(h);
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}

// Basis of the effective dielectric matrix from Pi at the lowest frequency: rpa_G
// (src/rpa/rpa.f90:31-173).  EIGEN: eigenvectors of Pi by descending eigenvalue; RANDOM: two
// subspace iterations G <- qr(Pi G), the QR by CholeskyQR2 (the same Gram-Schmidt Q as Householder
// QR up to column signs), trace weights diag(G^T Pi G); FULL: G = I.  NVecs is chosen by the
// reference's tail scan of the trace weights against TargetError.
int rpa_b200_piu_basis(rpa_b200_handle* h, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* R, int64_t ldR,
                       const double* OccEnergies, const double* VirtEnergies, double LowestFreq, double alpha,
                       int64_t prec, int64_t BasisType, double TargetError, const double* Guess, int64_t ldGuess,
                       uint64_t seed, double* G, int64_t ldG, int64_t* NVecs, double* TraceError,
                       double* ExactTrace) try {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
  if ((s = check_arrays(h, {R, OccEnergies, VirtEnergies, Guess, G}))) return s;
  if (BasisType < 1 || BasisType > 3) return fail(h, RPA_ERR_INVALID_ARG, "invalid basis type %lld", (long long)BasisType);
  if (!G || ldG < NQ || !NVecs || !(TargetError >= 0.0) || (Guess && ldGuess < NQ))
    return fail(h, RPA_ERR_INVALID_ARG, "invalid argument to rpa_b200_piu_basis");
  if (NQ > 46340) return fail(h, RPA_ERR_TOO_LARGE, "rpa_b200_piu_basis: NQ too large");
  Validated v;
  if ((s = validate_common(h, NQ, NOcc, NVirt, R, ldR, OccEnergies, VirtEnergies, 1, &LowestFreq, alpha, prec, v)))
    return s;
  const int n = (int)NQ;
  const size_t nn = (size_t)n * n;
  const double* Rd;
  int64_t ldd;
  if ((s = stage_R(h, v, R, ldR, &Rd, &ldd))) return s;
  RPA_CUDA(h, cudaEventRecord(h->ev[1], h->stream));
  if ((s = build_pi(h, v, Rd, ldd, alpha, prec))) return s;
  double* Pi = static_cast<double*>(h->Pi.p);
  RPA_CUDA(h, rpa::launch_symmetrize(Pi, n, (int64_t)nn, n, 1, h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[2], h->stream));
  std::vector<double> dg(n);
  RPA_CUDA(h, cudaMemcpy2DAsync(dg.data(), 8, Pi, (size_t)(n + 1) * 8, 8, (size_t)n, cudaMemcpyDeviceToHost,
                                h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  if ((s = check_device_error(h))) return s;
  dd exact{0.0, 0.0};
  for (double x : dg) exact = rpa::dd_add(exact, x);
  if (ExactTrace) *ExactTrace = exact.hi + exact.lo;
  RPA_CUDA(h, ensure(h->eA, nn * 8));
  RPA_CUDA(h, ensure(h->eZ, nn * 8));
  double* Gd = static_cast<double*>(h->eA.p);  // the full basis, column-major n x n
  std::vector<double> rwr(n);
  if (BasisType == 3) {  // full Cholesky space
    std::vector<double> eye(nn, 0.0);
    for (int i = 0; i < n; ++i) eye[(size_t)i * (n + 1)] = 1.0;
    RPA_CUDA(h, cudaMemcpyAsync(Gd, eye.data(), nn * 8, cudaMemcpyHostToDevice, h->stream));
    RPA_CUDA(h, cudaStreamSynchronize(h->stream));
    *NVecs = n;
    if (TraceError) *TraceError = 0.0;
  } else {
    if (BasisType == 2) {  // eigenvectors, descending eigenvalues
      double* Zd = static_cast<double*>(h->eZ.p);
      RPA_CUDA(h, cudaMemcpyAsync(Zd, Pi, nn * 8, cudaMemcpyDeviceToDevice, h->stream));
      std::vector<double> ev;
      std::vector<int> order;
      RPA_CUDA(h, ensure(h->tPerm, (size_t)n * sizeof(int)));
      RPA_CUDA(h, ensure(h->tSmall, (size_t)std::max(n, 64) * 8 + 64));
      // sym_eig destroys its input: diagonalise the copy in Zd, eigenvectors into Gd, then reorder
      if ((s = sym_eig(h, Zd, Gd, n, ev, order))) return s;
      std::vector<int> desc(order.rbegin(), order.rend());
      if ((s = gather(h, Gd, n, Zd, desc, nullptr))) return s;
      RPA_CUDA(h, cudaMemcpyAsync(Gd, Zd, nn * 8, cudaMemcpyDeviceToDevice, h->stream));
      for (int i = 0; i < n; ++i) rwr[i] = ev[desc[i]];
    } else {  // random subspace
      double* Yt = static_cast<double*>(h->eZ.p);  // holds Q^T
      RPA_CUDA(h, ensure(h->tS, nn * 8));
      RPA_CUDA(h, ensure(h->Ldiag, (size_t)n * 8));
      RPA_CUDA(h, ensure(h->tSmall, (size_t)std::max(n, 256) * 8 + 64));
      double* S = static_cast<double*>(h->tS.p);
      double* Q0 = Gd;
      if (Guess) {
        RPA_CUDA(h, cudaMemcpy2DAsync(Q0, (size_t)n * 8, Guess, (size_t)ldGuess * 8, (size_t)n * 8, (size_t)n,
                                      is_device_ptr(Guess) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                      h->stream));
      } else {
        RPA_CUDA(h, rpa::launch_fill_uniform(Q0, n, n, n, seed, h->stream));
      }
      // Yt = (Pi G0)^T = G0^T Pi
      RPA_CUDA(h, rpa::launch_gemm_f64(gemm_tn(n, n, n, Q0, n, Pi, n, Yt, n), h->stream));
      for (int it = 0; it < 2; ++it) {
        if (it > 0)  // Yt <- Q^T Pi  (Y = Pi Q)
          RPA_CUDA(h, rpa::launch_gemm_f64(gemm_nn(n, n, n, Gd, n, Pi, n, Yt, n), h->stream));
        // shifted CholeskyQR3 on the columns of Y = Yt^T (Fukaya, Kannan, Nakatsukasa, Zhang,
        // Yamamoto, SIAM J. Sci. Comput. 42 (2020) A477): the first pass factors Y^T Y +
        // 11 (n^2 + n(n+1)) u ||Y||_F^2 I, which succeeds for numerically rank-deficient Y; two
        // plain passes then make Q orthonormal.  The composite R is upper triangular, so Q is the
        // Gram-Schmidt Q of Householder QR up to column signs.
        for (int pass = 0; pass < 3; ++pass) {
          rpa::GemmF64Args g = gemm_nn(n, n, n, Yt, n, Yt, n, S, n);  // S = Yt Yt^T
          g.b_k = n;
          g.b_n = 1;
          RPA_CUDA(h, rpa::launch_gemm_f64(g, h->stream));
          if (pass == 0) {
            double* red = static_cast<double*>(h->tSmall.p);
            RPA_CUDA(h, rpa::launch_offdiag(Yt, n, n, red, h->stream));  // red[0] + red[1] = ||Y||_F^2
            const double shift = 11.0 * (2.0 * (double)n * n + (double)n) * 1.1102230246251565e-16;
            RPA_CUDA(h, rpa::launch_add_diag_scaled(S, n, n, shift, red, h->stream));
            RPA_CUDA(h, rpa::launch_add_diag_scaled(S, n, n, shift, red + 1, h->stream));
          }
          if ((s = cholesky(h, S, n, (int64_t)nn, n, 1, static_cast<double*>(h->Ldiag.p)))) return s;
          RPA_CUDA(h, rpa::launch_trsm_lower_left(S, n, (int64_t)nn, Yt, n, (int64_t)nn, n, n, 1, h->stream));
        }
        // the last pass factors the Gram matrix of an (almost) orthonormal Q: its pivots are ~1
        // unless the columns of Pi G were numerically dependent
        std::vector<double> piv(n);
        RPA_CUDA(h, cudaMemcpyAsync(piv.data(), h->Ldiag.p, (size_t)n * 8, cudaMemcpyDeviceToHost, h->stream));
        RPA_CUDA(h, cudaStreamSynchronize(h->stream));
        const auto mm = std::minmax_element(piv.begin(), piv.end());
        if (check_device_error(h) != RPA_OK || !(*mm.first > 0.5) || !(*mm.second < 2.0))
          return fail(h, RPA_ERR_NOT_SPD, "random Pi basis: Pi G is numerically rank deficient (CholeskyQR)");
        RPA_CUDA(h, cudaMemcpyAsync(Gd, Yt, nn * 8, cudaMemcpyDeviceToDevice, h->stream));  // Gd <- Q^T
      }
      // trace weights diag(Q^T Pi Q): T = Q^T Pi, rwr_p = sum_k T(p,k) Q^T(p,k)
      RPA_CUDA(h, rpa::launch_gemm_f64(gemm_nn(n, n, n, Yt, n, Pi, n, S, n), h->stream));
      std::vector<double> Th(nn), Qh(nn);
      RPA_CUDA(h, cudaMemcpyAsync(Th.data(), S, nn * 8, cudaMemcpyDeviceToHost, h->stream));
      RPA_CUDA(h, cudaMemcpyAsync(Qh.data(), Yt, nn * 8, cudaMemcpyDeviceToHost, h->stream));
      RPA_CUDA(h, rpa::launch_transpose(Yt, n, n, n, Gd, n, h->stream));  // G = Q
      RPA_CUDA(h, cudaStreamSynchronize(h->stream));
      for (int p = 0; p < n; ++p) {
        dd acc{0.0, 0.0};
        for (int k = 0; k < n; ++k) acc = rpa::dd_add(acc, Th[(size_t)p + (size_t)n * k] * Qh[(size_t)p + (size_t)n * k]);
        rwr[p] = acc.hi + acc.lo;
      }
    }
    // the reference's tail scan: drop RWR(p,p) from the end while the sum stays below the target
    int nv = n;
    dd abs_err{0.0, 0.0};
    for (int p = n - 1; p >= 0; --p) {
      const dd next = rpa::dd_add(abs_err, rwr[p]);
      if (next.hi + next.lo < TargetError) {
        abs_err = next;
        nv = p + 1;
      } else {
        break;
      }
    }
    *NVecs = nv;
    if (TraceError) *TraceError = abs_err.hi + abs_err.lo;
  }
  RPA_CUDA(h, cudaEventRecord(h->ev[3], h->stream));
  RPA_CUDA(h, cudaMemcpy2DAsync(G, (size_t)ldG * 8, Gd, (size_t)n * 8, (size_t)n * 8, (size_t)*NVecs,
                                is_device_ptr(G) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[4], h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  finish_timings(h);
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}

// R' = G^T R (NVecs x nov): the Cholesky vectors in the compressed Pi basis (the Cholesky-path
// counterpart of THC_ZgkPiU = Zgk G(:, 1:NVecsPiU), src/rpa/rpa.f90:2318-2320).
int rpa_b200_project_basis(rpa_b200_handle* h, int64_t NQ, int64_t NVecs, int64_t nov, const double* G, int64_t ldG,
                           const double* R, int64_t ldR, double* Rp, int64_t ldRp) try {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
  if ((s = check_arrays(h, {G, R, Rp}))) return s;
  if (NQ < 1 || NVecs < 1 || NVecs > NQ || nov < 1 || !G || !R || !Rp || ldG < NQ || ldR < NQ || ldRp < NVecs)
    return fail(h, RPA_ERR_INVALID_ARG, "invalid argument to rpa_b200_project_basis");
  if (NQ > INT32_MAX || nov > INT32_MAX) return fail(h, RPA_ERR_TOO_LARGE, "rpa_b200_project_basis: too large");
  const double* Gd = G;
  int64_t ldg = ldG;
  if (!is_device_ptr(G)) {
    RPA_CUDA(h, ensure(h->eA, (size_t)NQ * NVecs * 8));
    RPA_CUDA(h, cudaMemcpy2DAsync(h->eA.p, (size_t)NQ * 8, G, (size_t)ldG * 8, (size_t)NQ * 8, (size_t)NVecs,
                                  cudaMemcpyHostToDevice, h->stream));
    Gd = static_cast<const double*>(h->eA.p);
    ldg = NQ;
  }
  const double* Rd = R;
  int64_t ldr = ldR;
  if (!is_device_ptr(R)) {
    RPA_CUDA(h, ensure(h->R, (size_t)NQ * nov * 8));
    RPA_CUDA(h, cudaMemcpy2DAsync(h->R.p, (size_t)NQ * 8, R, (size_t)ldR * 8, (size_t)NQ * 8, (size_t)nov,
                                  cudaMemcpyHostToDevice, h->stream));
    Rd = static_cast<const double*>(h->R.p);
    ldr = NQ;
  }
  const bool dev_out = is_device_ptr(Rp);
  double* out = Rp;
  int64_t ldo = ldRp;
  if (!dev_out) {
    RPA_CUDA(h, ensure(h->eZ, (size_t)NVecs * nov * 8));
    out = static_cast<double*>(h->eZ.p);
    ldo = NVecs;
  }
  RPA_CUDA(h, cudaEventRecord(h->ev[1], h->stream));
  RPA_CUDA(h, rpa::launch_gemm_f64(gemm_tn((int)NVecs, (int)nov, NQ, Gd, ldg, Rd, ldr, out, ldo), h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[2], h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[3], h->stream));
  if ((s = screen_result(h, out, ldo, NVecs, nov, "the projected Cholesky vectors"))) return s;
  if (!dev_out)
    RPA_CUDA(h, cudaMemcpy2DAsync(Rp, (size_t)ldRp * 8, out, (size_t)NVecs * 8, (size_t)NVecs * 8, (size_t)nov,
                                  cudaMemcpyDeviceToHost, h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[4], h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  finish_timings(h);
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}

// Device copy of a column-major (rows x cols) input, or the input itself when it is already on
// the device; ld receives the leading dimension of the returned pointer.
static int stage_matrix(rpa_b200_handle* h, DevBuf& buf, const double* A, int64_t lda, int64_t rows, int64_t cols,
                 const double** out, int64_t* ld) {
  if (is_device_ptr(A)) {
    *out = A;
    *ld = lda;
    return RPA_OK;
  }
  RPA_CUDA(h, ensure(buf, (size_t)rows * cols * 8));
  RPA_CUDA(h, cudaMemcpy2DAsync(buf.p, (size_t)rows * 8, A, (size_t)lda * 8, (size_t)rows * 8, (size_t)cols,
                                cudaMemcpyHostToDevice, h->stream));
  *out = static_cast<const double*>(buf.p);
  *ld = rows;
  return RPA_OK;
}

// R = Z^T (Xa * Xi) into Rout (device, NQ x nov, ld ldR): Khatri-Rao blocks of whole occupied
// orbitals (<= ~1 GB each) and one FP64 DMMA GEMM per block.
static int form_thc_r(rpa_b200_handle* h, int64_t NGrid, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* Zd, int64_t ldz,
               const double* Xad, int64_t ldxa, const double* Xid, int64_t ldxi, double* Rout, int64_t ldR) {
  const int64_t per_occ = NGrid * NVirt;
  int64_t ib = std::max<int64_t>(1, std::min<int64_t>(NOcc, (int64_t)(1ll << 27) / std::max<int64_t>(per_occ, 1)));
  RPA_CUDA(h, ensure(h->thYX, (size_t)per_occ * ib * 8));
  double* YX = static_cast<double*>(h->thYX.p);
  for (int64_t i0 = 0; i0 < NOcc; i0 += ib) {
    const int64_t ni = std::min(ib, NOcc - i0);
    RPA_CUDA(h, rpa::launch_khatri_rao(Xad, ldxa, Xid, ldxi, (int)NGrid, (int)NVirt, (int)i0, (int)ni, YX, h->stream));
    RPA_CUDA(h, rpa::launch_gemm_f64(gemm_tn((int)NQ, (int)(NVirt * ni), NGrid, Zd, ldz, YX, NGrid,
                                             Rout + ldR * (i0 * NVirt), ldR),
                                     h->stream));
  }
  return RPA_OK;
}

static int check_thc_args(rpa_b200_handle* h, int64_t NGrid, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* Zgk,
                   int64_t ldZ, const double* Xga, int64_t ldXa, const double* Xgi, int64_t ldXi) {
  if (NGrid < 1 || NQ < 1 || NOcc < 1 || NVirt < 1 || !Zgk || !Xga || !Xgi || ldZ < NGrid || ldXa < NGrid ||
      ldXi < NGrid)
    return fail(h, RPA_ERR_INVALID_ARG, "invalid THC factor dimensions");
  if (NGrid > INT32_MAX || NQ > INT32_MAX || NOcc > INT32_MAX / NVirt)
    return fail(h, RPA_ERR_TOO_LARGE, "THC dimensions too large");
  return RPA_OK;
}

// Cholesky vectors from THC factors, R(k, ai) = sum_g Z(g, k) Xa(g, a) Xi(g, i), ai = a + NVirt i:
// rpa_THC_Rkab / rpa_THC_Rkai (src/rpa/rpa_THC.f90:374-426).
int rpa_b200_thc_r(rpa_b200_handle* h, int64_t NGrid, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* Zgk,
                   int64_t ldZ, const double* Xga, int64_t ldXa, const double* Xgi, int64_t ldXi, double* R,
                   int64_t ldR) try {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
  if ((s = check_arrays(h, {Zgk, Xga, Xgi, R}))) return s;
  if ((s = check_thc_args(h, NGrid, NQ, NOcc, NVirt, Zgk, ldZ, Xga, ldXa, Xgi, ldXi))) return s;
  if (!R || ldR < NQ) return fail(h, RPA_ERR_INVALID_ARG, "R is NULL or ldR < NQ");
  const int64_t nov = NOcc * NVirt;
  const double *Zd, *Xad, *Xid;
  int64_t ldz, ldxa, ldxi;
  if ((s = stage_matrix(h, h->thZ, Zgk, ldZ, NGrid, NQ, &Zd, &ldz))) return s;
  if ((s = stage_matrix(h, h->thXa, Xga, ldXa, NGrid, NVirt, &Xad, &ldxa))) return s;
  if ((s = stage_matrix(h, h->thXi, Xgi, ldXi, NGrid, NOcc, &Xid, &ldxi))) return s;
  const bool dev = is_device_ptr(R);
  double* Rd = R;
  int64_t ldr = ldR;
  if (!dev) {
    RPA_CUDA(h, ensure(h->thR, (size_t)NQ * nov * 8));
    Rd = static_cast<double*>(h->thR.p);
    ldr = NQ;
  }
  RPA_CUDA(h, cudaEventRecord(h->ev[1], h->stream));
  if ((s = form_thc_r(h, NGrid, NQ, NOcc, NVirt, Zd, ldz, Xad, ldxa, Xid, ldxi, Rd, ldr))) return s;
  RPA_CUDA(h, cudaEventRecord(h->ev[2], h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[3], h->stream));
  if ((s = screen_result(h, Rd, ldr, NQ, nov, "the formed Cholesky vectors"))) return s;
  if (!dev)
    RPA_CUDA(h, cudaMemcpy2DAsync(R, (size_t)ldR * 8, Rd, (size_t)NQ * 8, (size_t)NQ * 8, (size_t)nov,
                                  cudaMemcpyDeviceToHost, h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[4], h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  finish_timings(h);
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}

// Split-BF16 Pi build straight from THC factors, the way rpa_THC_PiU_BlockAlgo forms and
// contracts R block by block (src/rpa/rpa_THC.f90:285-340, 374-403): the ai columns are taken in
// pieces; for each piece the Khatri-Rao block YX = Xa * Xi of its columns, one FP64 DMMA GEMM
// R_piece = Z^T YX, the scale/split pass into piece-sized bf16 operands and the tensor-core SYRK
// adding the piece into Pi (FP64).  Neither the whole R nor the whole split operands are held:
// the device holds one piece of each (the piece width is sized to h->thc_piece_bytes).  The exact
// diagonal is summed over the pieces and written by the last piece's SYRK.
int build_pi_thc(rpa_b200_handle* h, const Validated& v, int64_t NGrid, const double* Zd, int64_t ldz,
                 const double* Xad, int64_t ldxa, const double* Xid, int64_t ldxi, double alpha) {
  const int NQ = v.NQ, K = v.K;
  const int64_t nov = v.nov;
  const size_t per_col = (size_t)NQ * 8 + (size_t)NGrid * 8 + (size_t)4 * K * NQ;  // R, YX, hi + lo
  int64_t w = (int64_t)(h->thc_piece_bytes / per_col) / 128 * 128;
  w = std::max<int64_t>(128, std::min<int64_t>(w, (nov + 127) / 128 * 128));
  const int64_t pitch = w;  // a multiple of 8 bf16 (16 bytes)
  RPA_CUDA(h, ensure(h->thR, (size_t)NQ * w * 8));
  RPA_CUDA(h, ensure(h->thYX, (size_t)NGrid * w * 8));
  RPA_CUDA(h, ensure(h->Xhi, (size_t)K * NQ * pitch * 2));
  RPA_CUDA(h, ensure(h->Xlo, (size_t)K * NQ * pitch * 2));
  RPA_CUDA(h, ensure(h->Pi, (size_t)K * NQ * NQ * 8));
  RPA_CUDA(h, ensure(h->diag, (size_t)2 * K * NQ * 8));
  double* Rp = static_cast<double*>(h->thR.p);
  double* YX = static_cast<double*>(h->thYX.p);
  double* Pi = static_cast<double*>(h->Pi.p);
  double* dsum = static_cast<double*>(h->diag.p);        // exact diagonal summed over the pieces
  double* dpiece = dsum + (size_t)K * NQ;                 // this piece's exact diagonal
  const double* D = static_cast<const double*>(h->D.p);
  rpa::FreqGroup fg{};
  fg.n = K;
  for (int k = 0; k < K; ++k) fg.u2[k] = v.freqs[k] * v.freqs[k];
  RPA_CUDA(h, cudaMemsetAsync(h->count_dev, 0, sizeof(int), h->stream));
  int s;
  for (int64_t a0 = 0; a0 < nov; a0 += w) {
    const int64_t wp = std::min(w, nov - a0);
    const bool first = a0 == 0, last = a0 + wp == nov;
    cudaEvent_t e0 = pool_event(h), e1 = pool_event(h), e2 = pool_event(h);
    RPA_CUDA(h, rpa::launch_khatri_rao_cols(Xad, ldxa, Xid, ldxi, (int)NGrid, (int)v.nv, a0, wp, YX, h->stream));
    RPA_CUDA(h, rpa::launch_gemm_f64(gemm_tn(NQ, (int)wp, NGrid, Zd, ldz, YX, NGrid, Rp, NQ), h->stream));
    RPA_CUDA(h, rpa::launch_count_nonfinite(Rp, (int64_t)NQ * wp, h->count_dev, h->stream));
    const rpa::SplitPlan plan = rpa::plan_scale_split(NQ, wp, h->num_sms);
    RPA_CUDA(h, ensure(h->diag_part, (size_t)plan.nsplit * K * NQ * 8));
    CUtensorMap sHi, sLo, mAh, mAl, mBh, mBl;
    if ((s = encode_store_maps(h, &sHi, &sLo, h->Xhi.p, h->Xlo.p, wp, NQ, K, pitch)) != RPA_OK) return s;
    if ((s = encode_map(h, &mAh, h->Xhi.p, wp, NQ, K, pitch, rpa::kSyrkTcTM)) != RPA_OK) return s;
    if ((s = encode_map(h, &mAl, h->Xlo.p, wp, NQ, K, pitch, rpa::kSyrkTcTM)) != RPA_OK) return s;
    if ((s = encode_map(h, &mBh, h->Xhi.p, wp, NQ, K, pitch, rpa::kSyrkTcTN)) != RPA_OK) return s;
    if ((s = encode_map(h, &mBl, h->Xlo.p, wp, NQ, K, pitch, rpa::kSyrkTcTN)) != RPA_OK) return s;
    RPA_CUDA(h, cudaEventRecord(e0, h->stream));
    RPA_CUDA(h, rpa::launch_scale_split(Rp, NQ, NQ, wp, D + a0, fg, alpha, &sHi, &sLo,
                                        static_cast<double*>(h->diag_part.p), dpiece, plan, h->err_dev, h->stream));
    RPA_CUDA(h, rpa::launch_add_into(dsum, dpiece, (int64_t)K * NQ, first, h->stream));
    RPA_CUDA(h, cudaEventRecord(e1, h->stream));
    h->split_ev.push_back({e0, e1});
    rpa::SyrkTcArgs a{};
    a.NQ = NQ;
    a.nov = wp;
    a.kg = K;
    a.Pi = Pi;
    a.ldPi = NQ;
    a.piStride = (int64_t)NQ * NQ;
    a.diag = last ? dsum : nullptr;
    a.err = h->err_dev;
    a.seg_chunks = h->seg_chunks;
    a.chunk0 = 0;
    a.nov_part = wp;
    a.accumulate = first ? 0 : 1;
    if ((s = prepare_sync(h, NQ, K, wp, &a.sync)) != RPA_OK) return s;
    a.sync_every = h->sync_every;
    a.sync_lag = 2;
    RPA_CUDA(h, rpa::launch_syrk_split_bf16(&mAh, &mAl, &mBh, &mBl, a, h->num_sms, h->stream));
    RPA_CUDA(h, cudaEventRecord(e2, h->stream));
    h->tc_ev.push_back({e1, e2});
  }
  int cnt = 0;
  RPA_CUDA(h, cudaMemcpyAsync(&cnt, h->count_dev, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  if (cnt) return fail(h, RPA_ERR_NONFINITE, "%d non-finite entries in the Cholesky vectors formed from the THC factors",
                       cnt);
  return RPA_OK;
}

// RPA energy from THC factors (the FullRkai branch of rpa_THC_PiU, src/rpa/rpa_THC.f90:215-329).
// Split precision with up to 16 frequencies: R is formed and contracted piece by piece
// (build_pi_thc).  Otherwise (FP64 form, or more frequencies than one split group) R is formed
// whole on the device and handed to the energy path; it never leaves the GPU.
int rpa_b200_ec_thc(rpa_b200_handle* h, int64_t NGrid, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* Zgk,
                    int64_t ldZ, const double* Xga, int64_t ldXa, const double* Xgi, int64_t ldXi,
                    const double* OccEnergies, const double* VirtEnergies, int64_t NFreqs, const double* Freqs,
                    const double* FreqWeights, double alpha, int64_t prec, double* Ec, double* Eu) try {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
  if ((s = check_arrays(h, {Zgk, Xga, Xgi, OccEnergies, VirtEnergies, Freqs, FreqWeights}))) return s;
  if ((s = check_thc_args(h, NGrid, NQ, NOcc, NVirt, Zgk, ldZ, Xga, ldXa, Xgi, ldXi))) return s;
  const int64_t nov = NOcc * NVirt;
  const double *Zd, *Xad, *Xid;
  int64_t ldz, ldxa, ldxi;
  if ((s = stage_matrix(h, h->thZ, Zgk, ldZ, NGrid, NQ, &Zd, &ldz))) return s;
  if ((s = stage_matrix(h, h->thXa, Xga, ldXa, NGrid, NVirt, &Xad, &ldxa))) return s;
  if ((s = stage_matrix(h, h->thXi, Xgi, ldXi, NGrid, NOcc, &Xid, &ldxi))) return s;
  if (prec == RPA_PREC_SPLIT_BF16 && NFreqs >= 1 && NFreqs <= rpa::kMaxKgLaunch) {
    Validated v;
    // R itself is formed below: the factor Z stands in for the R argument of the common checks
    if ((s = validate_common(h, NQ, NOcc, NVirt, Zd, NQ, OccEnergies, VirtEnergies, NFreqs, Freqs, alpha, prec, v)))
      return s;
    if (!FreqWeights || !Ec) return fail(h, RPA_ERR_INVALID_ARG, "FreqWeights or Ec is NULL");
    if ((s = fetch_small(h, FreqWeights, NFreqs, v.weights))) return s;
    if ((s = stage_eps(h, v))) return s;
    RPA_CUDA(h, cudaEventRecord(h->ev[1], h->stream));
    if ((s = build_pi_thc(h, v, NGrid, Zd, ldz, Xad, ldxa, Xid, ldxi, alpha))) return s;
    if ((s = energy_from_workspace(h, v.NQ, v.K, v.weights, Ec, Eu))) return s;
    RPA_CUDA(h, cudaEventRecord(h->ev[4], h->stream));
    finish_timings(h);
    return RPA_OK;
  }
  RPA_CUDA(h, ensure(h->thR, (size_t)NQ * nov * 8));
  double* Rd = static_cast<double*>(h->thR.p);
  if ((s = form_thc_r(h, NGrid, NQ, NOcc, NVirt, Zd, ldz, Xad, ldxa, Xid, ldxi, Rd, NQ))) return s;
  return rpa_b200_ec(h, NQ, NOcc, NVirt, Rd, NQ, OccEnergies, VirtEnergies, NFreqs, Freqs, FreqWeights, alpha, prec,
                     Ec, Eu);
} catch (...) {
  return exception_status(h);
}

// Device buffer grown to `bytes` keeping its first `used` bytes.
static int grow_keep(rpa_b200_handle* h, DevBuf& b, size_t bytes, size_t used) {
  if (b.p && b.bytes >= bytes) return RPA_OK;
  const size_t nb = std::max(bytes, b.bytes * 2);
  void* p = nullptr;
  RPA_CUDA(h, dev_alloc(&p, nb));
  if (b.p && used) RPA_CUDA(h, cudaMemcpyAsync(p, b.p, used, cudaMemcpyDeviceToDevice, h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  dev_free(b.p, b.bytes);
  b.p = p;
  b.bytes = nb;
  return RPA_OK;
}

// C = alpha A op(B) (+ beta C) with A (M x K) column-major and B given as (K x N) column-major
// (bt = false) or as (N x K) column-major, i.e. B^T (bt = true).
static rpa::GemmF64Args gemm_g(int M, int N, int64_t K, const double* A, int64_t lda, bool at, const double* B,
                        int64_t ldb, bool bt, double* C, int64_t ldc, double alpha = 1.0, double beta = 0.0) {
  rpa::GemmF64Args g = gemm_nn(M, N, K, A, lda, B, ldb, C, ldc);
  if (at) {
    g.a_m = lda;
    g.a_k = 1;
  }
  if (bt) {
    g.b_k = ldb;
    g.b_n = 1;
  }
  g.alpha = alpha;
  g.beta = beta;
  return g;
}

// Particle-hole corrections to direct RPA with pair-natural orbitals on THC factors:
// rpa_JCTC2024_Corrections and its helpers (src/rpa/rpa_JCTC2024.f90:24-703).  PNOs of each pair
// i >= j: T_ij = U_i diag(A) U_j^T, SVD through the eigen-decomposition of T T^T (U, s^2) and
// s V = T^T U for the singular values above CutoffThreshPNO.  Every product is an FP64 tensor-core
// GEMM (the Hadamard products with the THC orbital factors are folded into their k- and row-scales);
// every trace is a deterministic partial-sum reduction collected once at the end.
int rpa_b200_jctc2024(rpa_b200_handle* h, int64_t NGrid, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* Zgk,
                      int64_t ldZ, const double* Xgi, int64_t ldXi, const double* Yga, int64_t ldYa, int64_t NVecsT2,
                      const double* U, int64_t ldU, const double* Am, const double* Lik, int64_t ldL,
                      double CutoffThreshPNO, int64_t BoysScreening, double CutoffThreshVabij, double* Energies,
                      int64_t* PNOStats) try {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
  if ((s = check_arrays(h, {Zgk, Xgi, Yga, U, Am, Lik}))) return s;
  if (NGrid < 1 || NQ < 1 || NOcc < 1 || NVirt < 1 || NVecsT2 < 1 || !Zgk || !Xgi || !Yga || !U || !Am ||
      !Energies || ldZ < NGrid || ldXi < NGrid || ldYa < NGrid || ldU < NOcc * NVirt || (Lik && ldL < NOcc) ||
      !(CutoffThreshPNO >= 0.0))
    return fail(h, RPA_ERR_INVALID_ARG, "invalid argument to rpa_b200_jctc2024");
  if (NGrid > INT32_MAX || NQ > INT32_MAX || NOcc * NVirt > INT32_MAX || NVecsT2 > INT32_MAX || NVirt > 46340)
    return fail(h, RPA_ERR_TOO_LARGE, "rpa_b200_jctc2024: dimensions too large");
  const int ng = (int)NGrid, nq = (int)NQ, no = (int)NOcc, nv = (int)NVirt, nt = (int)NVecsT2;
  const int64_t nov = NOcc * NVirt;
  const double *Zd, *Yd, *Xd0, *Ud0, *Ld = nullptr;
  int64_t ldz, ldy, ldx0, ldu0, ldl = 0;
  if ((s = stage_matrix(h, h->thZ, Zgk, ldZ, NGrid, NQ, &Zd, &ldz))) return s;
  if ((s = stage_matrix(h, h->thXa, Yga, ldYa, NGrid, NVirt, &Yd, &ldy))) return s;
  if ((s = stage_matrix(h, h->thXi, Xgi, ldXi, NGrid, NOcc, &Xd0, &ldx0))) return s;
  if ((s = stage_matrix(h, h->tU, U, ldU, nov, NVecsT2, &Ud0, &ldu0))) return s;
  if (Lik && (s = stage_matrix(h, h->jL, Lik, ldL, NOcc, NOcc, &Ld, &ldl))) return s;
  std::vector<double> Ah;
  if ((s = fetch_small(h, Am, NVecsT2, Ah))) return s;
  // scratch: A, localised X and U, T, M, eigenvectors, products, partial sums
  const int64_t npairs = (int64_t)no * (no + 1) / 2;
  const int64_t nslot = 5 * npairs;  // S1a, S1b, S2ghij, S2bcd, Vijij per pair
  RPA_CUDA(h, ensure(h->jX, (size_t)ng * no * 8));
  RPA_CUDA(h, ensure(h->jU, (size_t)nov * nt * 8));
  const size_t nvv = (size_t)nv * nv;
  const size_t wwords = (size_t)nt + 3 * nvv + (size_t)nq * nv + 2 * (size_t)ng * nv + (size_t)nq + (size_t)ng +
                        2 * nvv + 4 * nvv + 2 * nvv + 2 * (size_t)ng * nv + (size_t)nslot * rpa::kDotPartials + 64;
  RPA_CUDA(h, ensure(h->jWork, wwords * 8));
  double* w = static_cast<double*>(h->jWork.p);
  double* Ad = w;
  double* Tm = Ad + nt;            // T_ij (nv x nv)
  double* Mm = Tm + nvv;           // T T^T
  double* Vm = Mm + nvv;           // its eigenvectors
  double* ZYXk = Vm + nvv;         // NQ x nv
  double* ZYXg = ZYXk + (size_t)nq * nv;  // NGrid x nv
  double* Wg = ZYXg + (size_t)ng * nv;    // NGrid x nv
  double* zk = Wg + (size_t)ng * nv;      // NQ
  double* zg = zk + nq;                   // NGrid
  double* Gg = zg + ng;                   // G for 2g..2j (nv x nv)
  double* Gb = Gg + nvv;                  // G for 2b..2d
  double* Sm = Gb + nvv;                  // 4 S blocks (<= nv x nv each)
  double* QS = Sm + 4 * nvv;              // nv x 2 Nkj
  double* Wx = QS + 2 * nvv;              // NGrid x N
  double* Wy = Wx + (size_t)ng * nv;
  double* part = Wy + (size_t)ng * nv;
  RPA_CUDA(h, cudaMemcpyAsync(Ad, Ah.data(), (size_t)nt * 8, cudaMemcpyHostToDevice, h->stream));
  RPA_CUDA(h, cudaMemsetAsync(part, 0, (size_t)nslot * rpa::kDotPartials * 8, h->stream));
  double* Xd = static_cast<double*>(h->jX.p);
  double* Ud = static_cast<double*>(h->jU.p);
  const int64_t ldx = ng, ldu = nov;
  RPA_CUDA(h, cudaEventRecord(h->ev[1], h->stream));
  // occupied localisation: X <- X L, U(:, :, mu) <- U(:, :, mu) L
  if (Ld) {
    RPA_CUDA(h, rpa::launch_gemm_f64(gemm_g(ng, no, no, Xd0, ldx0, false, Ld, ldl, false, Xd, ldx), h->stream));
    rpa::GemmF64Args g = gemm_g(nv, no, no, Ud0, nv, false, Ld, ldl, false, Ud, nv);
    g.batch = nt;
    g.sA = ldu0;
    g.sB = 0;
    g.sC = nov;
    RPA_CUDA(h, rpa::launch_gemm_f64(g, h->stream));
  } else {
    RPA_CUDA(h, cudaMemcpy2DAsync(Xd, (size_t)ng * 8, Xd0, (size_t)ldx0 * 8, (size_t)ng * 8, (size_t)no,
                                  cudaMemcpyDeviceToDevice, h->stream));
    RPA_CUDA(h, cudaMemcpy2DAsync(Ud, (size_t)nov * 8, Ud0, (size_t)ldu0 * 8, (size_t)nov * 8, (size_t)nt,
                                  cudaMemcpyDeviceToDevice, h->stream));
  }
  // max_a (aa|aa) for the Schwarz screening of the (ab|ij) blocks (Boys orbitals)
  double maxvabab = 0.0;
  if (BoysScreening) {
    RPA_CUDA(h, rpa::launch_hadamard(Yd, ldy, Yd, ldy, ng, nv, Wg, ng, h->stream));
    RPA_CUDA(h, rpa::launch_gemm_f64(gemm_g(nq, nv, ng, Zd, ldz, true, Wg, ng, false, ZYXk, nq), h->stream));
    std::vector<double> zz((size_t)nq * nv);
    RPA_CUDA(h, cudaMemcpyAsync(zz.data(), ZYXk, zz.size() * 8, cudaMemcpyDeviceToHost, h->stream));
    RPA_CUDA(h, cudaStreamSynchronize(h->stream));
    for (int a = 0; a < nv; ++a) {
      dd acc{0.0, 0.0};
      for (int k = 0; k < nq; ++k) {
        const double v = zz[(size_t)k + (size_t)nq * a];
        acc = rpa::dd_add(acc, v * v);
      }
      maxvabab = std::max(maxvabab, acc.hi + acc.lo);
    }
  }

  // ---- pair-natural orbitals of every pair i >= j: packed [U | s V] (nv x 2n) per pair.  Pairs
  // run in batches: one grouped GEMM forms every T_ij, one batched GEMM every T T^T, one batched
  // eigensolver call diagonalises them, one column map gathers the kept singular vectors and one
  // grouped GEMM forms every s V = T^T U.
  std::vector<int64_t> poff((size_t)no * no, -1);
  std::vector<int> pn((size_t)no * no, 0);
  size_t pno_used = 0;
  const double thr2 = CutoffThreshPNO * CutoffThreshPNO;
  int64_t max_n = 0, sum_n = 0, zero_pairs = 0;
  std::vector<std::pair<int, int>> plist;
  for (int j = 0; j < no; ++j)
    for (int i = j; i < no; ++i) plist.push_back({i, j});
  const size_t per_pair = 3 * nvv * 8 + (rpa::syevd_workspace_bytes(nv, 2) - rpa::syevd_workspace_bytes(nv, 1));
  const int bmax = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)plist.size(),
                                                               (int64_t)((size_t)4 << 30) / (int64_t)per_pair));
  RPA_CUDA(h, ensure(h->jD, (size_t)(std::max(8 * no, bmax) + 8) * sizeof(rpa::GemmF64Args) +
                                (size_t)(std::max(8 * no, bmax) + 16) * sizeof(int)));
  for (size_t b0 = 0; b0 < plist.size(); b0 += bmax) {
    const int nbat = (int)std::min<size_t>(bmax, plist.size() - b0);
    RPA_CUDA(h, ensure(h->jT, (size_t)nbat * nvv * 8));
    RPA_CUDA(h, ensure(h->jM, (size_t)nbat * nvv * 8));
    RPA_CUDA(h, ensure(h->jV, (size_t)nbat * nvv * 8));
    RPA_CUDA(h, ensure(h->eW, rpa::syevd_workspace_bytes(nv, nbat)));
    double* Tb = static_cast<double*>(h->jT.p);
    double* Mb = static_cast<double*>(h->jM.p);
    double* Vb = static_cast<double*>(h->jV.p);
    std::vector<rpa::GemmF64Args> tp;
    for (int q = 0; q < nbat; ++q) {  // T(a, b) = sum_mu U(a, i, mu) A_mu U(b, j, mu)
      const int i = plist[b0 + q].first, j = plist[b0 + q].second;
      rpa::GemmF64Args gt =
          gemm_g(nv, nv, nt, Ud + (int64_t)nv * i, ldu, false, Ud + (int64_t)nv * j, ldu, true, Tb + nvv * q, nv);
      gt.kscale = Ad;
      tp.push_back(gt);
    }
    RPA_CUDA(h, rpa::launch_gemm_f64_grouped(tp, h->jD.p, h->jD.bytes, h->stream));
    rpa::GemmF64Args gm = gemm_g(nv, nv, nv, Tb, nv, false, Tb, nv, true, Mb, nv);
    gm.batch = nbat;
    gm.sA = gm.sB = gm.sC = (int64_t)nvv;
    RPA_CUDA(h, rpa::launch_gemm_f64(gm, h->stream));
    std::vector<double> ev;
    bool conv = false;
    RPA_CUDA(h, rpa::syevd_batched(Mb, nv, nbat, Vb, h->eW.p, h->eW.bytes, ev, conv, h->stream));
    if (!conv) return fail(h, RPA_ERR_NOT_CONVERGED, "PNO eigensolver: a leaf did not converge");
    // keep singular values above the cutoff (eigenvalues of T T^T above its square), descending
    std::vector<int64_t> map;
    std::vector<rpa::GemmF64Args> sv;
    size_t need = pno_used;
    std::vector<std::pair<int, size_t>> placed(nbat, {0, 0});
    for (int q = 0; q < nbat; ++q) {
      std::vector<int> order(nv);
      for (int c = 0; c < nv; ++c) order[c] = c;
      const double* evq = ev.data() + (size_t)nv * q;
      std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return evq[a] > evq[b]; });
      int n = 0;
      while (n < nv && evq[order[n]] > thr2) ++n;
      max_n = std::max<int64_t>(max_n, n);
      sum_n += n;
      if (n == 0) {
        ++zero_pairs;
        continue;
      }
      placed[q] = {n, need};
      for (int c = 0; c < n; ++c) {
        map.push_back((int64_t)q * nv + order[c]);
        map.push_back((int64_t)(need / 8 / nv) + c);
      }
      need += (size_t)nv * 2 * n * 8;
    }
    if ((s = grow_keep(h, h->jPno, std::max<size_t>(need, 8), pno_used))) return s;
    double* pnob = static_cast<double*>(h->jPno.p);
    RPA_CUDA(h, ensure(h->jMap, std::max<size_t>(map.size(), 2) * sizeof(int64_t)));
    if (!map.empty()) {
      RPA_CUDA(h, cudaMemcpyAsync(h->jMap.p, map.data(), map.size() * sizeof(int64_t), cudaMemcpyHostToDevice,
                                  h->stream));
      RPA_CUDA(h, rpa::launch_copy_columns(Vb, pnob, static_cast<const int64_t*>(h->jMap.p),
                                           (int64_t)(map.size() / 2), nv, h->stream));  // U
    }
    for (int q = 0; q < nbat; ++q) {
      const int n = placed[q].first;
      if (n == 0) continue;
      const int i = plist[b0 + q].first, j = plist[b0 + q].second;
      double* dst = pnob + placed[q].second / 8;
      sv.push_back(gemm_g(nv, n, nv, Tb + nvv * q, nv, true, dst, nv, false, dst + (size_t)nv * n, nv));  // s V
      poff[(size_t)i + (size_t)no * j] = poff[(size_t)j + (size_t)no * i] = (int64_t)(placed[q].second / 8);
      pn[(size_t)i + (size_t)no * j] = pn[(size_t)j + (size_t)no * i] = n;
    }
    RPA_CUDA(h, rpa::launch_gemm_f64_grouped(sv, h->jD.p, h->jD.bytes, h->stream));
    pno_used = need;
    RPA_CUDA(h, cudaStreamSynchronize(h->stream));  // map and the descriptors must outlive their uploads
  }
  if (PNOStats) {
    PNOStats[0] = max_n;
    PNOStats[1] = sum_n;
    PNOStats[2] = zero_pairs;
  }
  RPA_CUDA(h, cudaEventRecord(h->ev[2], h->stream));
  const double* pno = static_cast<const double*>(h->jPno.p);
  // per-orbital packs (rpa_JCTC2024_PackTransfMatrices): pack[o] = the [U | s V] blocks of the
  // pairs {k, o}, k = 0 .. NOcc-1, side by side; kcol[o * no + k] = first column of pair {k, o}
  std::vector<int64_t> pack_off(no + 1, 0);
  std::vector<int> ncol(no, 0), kcol((size_t)no * no, 0);
  for (int o = 0; o < no; ++o) {
    for (int k = 0; k < no; ++k) {
      kcol[(size_t)o * no + k] = ncol[o];
      ncol[o] += 2 * pn[(size_t)k + (size_t)no * o];
    }
    pack_off[o + 1] = pack_off[o] + ncol[o];
  }
  int maxcol = 1;
  for (int o = 0; o < no; ++o) maxcol = std::max(maxcol, ncol[o]);
  RPA_CUDA(h, ensure(h->jPack, (size_t)std::max<int64_t>(pack_off[no], 1) * nv * 8));
  double* pack = static_cast<double*>(h->jPack.p);
  for (int o = 0; o < no; ++o)
    for (int k = 0; k < no; ++k) {
      const int n = pn[(size_t)k + (size_t)no * o];
      if (n > 0)
        RPA_CUDA(h, cudaMemcpyAsync(pack + (size_t)nv * (pack_off[o] + kcol[(size_t)o * no + k]),
                                    pno + poff[(size_t)k + (size_t)no * o], (size_t)nv * 2 * n * 8,
                                    cudaMemcpyDeviceToDevice, h->stream));
    }
  RPA_CUDA(h, ensure(h->jQS, (size_t)nv * maxcol * 2 * 8));
  RPA_CUDA(h, ensure(h->jSK, (size_t)64 * nvv * 8));
  RPA_CUDA(h, ensure(h->jS, (size_t)4 * no * std::max<int64_t>(max_n * max_n, 1) * 8));
  RPA_CUDA(h, ensure(h->jD, (size_t)(8 * no + 8) * sizeof(rpa::GemmF64Args) + (size_t)(8 * no + 16) * sizeof(int)));

  // ---- energy terms (rpa_JCTC2024_Gaibj_Gabij_v2)
  const double c2b = -2.0, c2c = -2.0, c2d = 2.0, c2g = -4.0, c2h = -4.0, c2i = 2.0, c2j = 2.0;
  auto slot = [&](int64_t pair, int term) { return part + (size_t)(5 * pair + term) * rpa::kDotPartials; };
  auto G = [&](const rpa::GemmF64Args& g) { return rpa::launch_gemm_f64(g, h->stream); };
  // grouped-GEMM descriptors of every pair, built once and uploaded in one copy: the k sum of a
  // pair is one grouped launch for its S blocks and two for its QS slots
  struct GroupRef {
    int64_t desc, start;
    int nprob, ntiles;
    bool am, bn;
  };
  std::vector<rpa::GemmF64Args> all_desc;
  std::vector<int> all_start;
  std::vector<GroupRef> groups;
  {
    double* QSg = static_cast<double*>(h->jQS.p);
    double* QSb = QSg + (size_t)nv * maxcol;
    double* Sbase = static_cast<double*>(h->jS.p);
    auto add_group = [&](const std::vector<rpa::GemmF64Args>& v) {
      GroupRef gr{(int64_t)all_desc.size(), (int64_t)all_start.size(), (int)v.size(), 0, true, true};
      if (!v.empty()) {
        gr.am = (v[0].a_m == 1);
        gr.bn = (v[0].b_n == 1);
      }
      all_start.push_back(0);
      for (const auto& g : v) {
        all_desc.push_back(g);
        gr.ntiles += rpa::gemm_f64_tiles(g);
        all_start.push_back(gr.ntiles);
      }
      groups.push_back(gr);
    };
    for (int j = 0; j < no; ++j)
      for (int i = j; i < no; ++i) {
        std::vector<rpa::GemmF64Args> sp, q1, q2;
        size_t soff = 0;
        const double* pj = pack + (size_t)nv * pack_off[j];
        const double* pi_ = pack + (size_t)nv * pack_off[i];
        for (int k = 0; k < no; ++k) {
          const int nkj = pn[(size_t)k + (size_t)no * j], nki = pn[(size_t)k + (size_t)no * i];
          if (nkj == 0 || nki == 0) continue;
          const double* kj[2] = {pj + (size_t)nv * kcol[(size_t)j * no + k], nullptr};
          kj[1] = kj[0] + (size_t)nv * nkj;
          const double* ki[2] = {pi_ + (size_t)nv * kcol[(size_t)i * no + k], nullptr};
          ki[1] = ki[0] + (size_t)nv * nki;
          int Pki, Qki, Pik, Qik, Pkj, Qkj, Pjk, Qjk;
          if (k >= i) { Pki = 0; Qki = 1; Pik = 1; Qik = 0; } else { Pki = 1; Qki = 0; Pik = 0; Qik = 1; }
          if (k >= j) { Pkj = 0; Qkj = 1; Pjk = 1; Qjk = 0; } else { Pkj = 1; Qkj = 0; Pjk = 0; Qjk = 1; }
          double* S_jk_ki = Sbase + soff;
          double* S_jk_ik = S_jk_ki + (size_t)nkj * nki;
          double* S_kj_ki = S_jk_ik + (size_t)nkj * nki;
          double* S_kj_ik = S_kj_ki + (size_t)nkj * nki;
          soff += 4 * (size_t)nkj * nki;
          sp.push_back(gemm_g(nkj, nki, nv, kj[Qjk], nv, true, ki[Pki], nv, false, S_jk_ki, nkj));
          sp.push_back(gemm_g(nkj, nki, nv, kj[Qjk], nv, true, ki[Pik], nv, false, S_jk_ik, nkj));
          sp.push_back(gemm_g(nkj, nki, nv, kj[Qkj], nv, true, ki[Pki], nv, false, S_kj_ki, nkj));
          sp.push_back(gemm_g(nkj, nki, nv, kj[Qkj], nv, true, ki[Pik], nv, false, S_kj_ik, nkj));
          const size_t c0 = (size_t)kcol[(size_t)j * no + k];
          double* qg[2] = {QSg + (size_t)nv * c0, QSg + (size_t)nv * (c0 + nkj)};
          double* qb[2] = {QSb + (size_t)nv * c0, QSb + (size_t)nv * (c0 + nkj)};
          // alpha ki[q] S^T (+ beta slot)
          auto qs = [&](double* dst, int q, const double* S, double alpha, double beta) {
            return gemm_g(nv, nkj, nki, ki[q], nv, false, S, nkj, true, dst, nv, alpha, beta);
          };
          if (i != j) {
            q1.push_back(qs(qg[Pjk], Qki, S_jk_ki, 2.0 * c2g, 0.0));
            q2.push_back(qs(qg[Pjk], Qik, S_jk_ik, c2i + c2j, 1.0));
            q1.push_back(qs(qg[Pkj], Qik, S_kj_ik, 2.0 * c2h, 0.0));
            q2.push_back(qs(qg[Pkj], Qki, S_kj_ki, c2i + c2j, 1.0));
            q1.push_back(qs(qb[Pkj], Qik, S_kj_ik, 2.0 * c2d, 0.0));
            q2.push_back(qs(qb[Pkj], Qki, S_kj_ki, c2b + c2c, 1.0));
            q1.push_back(qs(qb[Pjk], Qik, S_jk_ik, c2b + c2c, 0.0));
          } else {
            q1.push_back(qs(qg[Pjk], Qki, S_jk_ki, c2g, 0.0));
            q2.push_back(qs(qg[Pjk], Qik, S_jk_ik, c2i + c2j, 1.0));
            q1.push_back(qs(qg[Pkj], Qik, S_kj_ik, c2h, 0.0));
            q1.push_back(qs(qb[Pkj], Qik, S_kj_ik, c2d, 0.0));  // the other slot of 2b..2d stays zero
            q2.push_back(qs(qb[Pkj], Qki, S_kj_ki, c2b + c2c, 1.0));
          }
        }

        add_group(sp);
        add_group(q1);
        add_group(q2);
      }
  }
  RPA_CUDA(h, ensure(h->jD, std::max<size_t>(all_desc.size(), 1) * sizeof(rpa::GemmF64Args) +
                                std::max<size_t>(all_start.size(), 1) * sizeof(int) + 256));
  rpa::GemmF64Args* dprob = static_cast<rpa::GemmF64Args*>(h->jD.p);
  int* dstart = reinterpret_cast<int*>(static_cast<char*>(h->jD.p) +
                                       ((std::max<size_t>(all_desc.size(), 1) * sizeof(rpa::GemmF64Args) + 255) & ~(size_t)255));
  if (!all_desc.empty())
    RPA_CUDA(h, cudaMemcpyAsync(dprob, all_desc.data(), all_desc.size() * sizeof(rpa::GemmF64Args),
                                cudaMemcpyHostToDevice, h->stream));
  RPA_CUDA(h, cudaMemcpyAsync(dstart, all_start.data(), all_start.size() * sizeof(int), cudaMemcpyHostToDevice,
                              h->stream));
  int64_t pair = 0;
  std::vector<std::pair<int, int>> pair_ij;
  for (int j = 0; j < no; ++j) {
    const double* xj = Xd + (int64_t)ldx * j;
    // ZYX(k, b) = sum_g Z(g, k) X(g, j) Y(g, b); ZYX(g, b) = Z ZYX(k, b)
    rpa::GemmF64Args g1 = gemm_g(nq, nv, ng, Zd, ldz, true, Yd, ldy, false, ZYXk, nq);
    g1.kscale = xj;
    RPA_CUDA(h, G(g1));
    RPA_CUDA(h, G(gemm_g(ng, nv, nq, Zd, ldz, false, ZYXk, nq, false, ZYXg, ng)));
    for (int i = j; i < no; ++i, ++pair) {
      pair_ij.push_back({i, j});
      const double* xi = Xd + (int64_t)ldx * i;
      // ZXX(k) = sum_g Z(g, k) X(g, i) X(g, j), its norm for the screening, ZXX(g) = Z ZXX(k)
      rpa::GemmF64Args g2 = gemm_g(nq, 1, ng, Zd, ldz, true, xj, ng, false, zk, nq);
      g2.kscale = xi;
      RPA_CUDA(h, G(g2));
      RPA_CUDA(h, rpa::launch_dot_partials(zk, nq, zk, nq, nq, 1, nullptr, slot(pair, 4), h->stream));
      RPA_CUDA(h, G(gemm_g(ng, 1, nq, Zd, ldz, false, zk, nq, false, zg, ng)));
      // S1a, S1b of the pair (i, j)
      const int nij = pn[(size_t)i + (size_t)no * j];
      if (nij > 0) {
        const double* P = pno + poff[(size_t)i + (size_t)no * j];
        const double* Q = P + (size_t)nv * nij;
        for (int t = 0; t < 2; ++t) {  // t = 0: S1b (Y Q, ZYX P); t = 1: S1a (Y P, ZYX Q)
          rpa::GemmF64Args gx = gemm_g(ng, nij, nv, Yd, ldy, false, t == 0 ? Q : P, nv, false, Wx, ng);
          gx.rowscale = xi;
          RPA_CUDA(h, G(gx));
          RPA_CUDA(h, G(gemm_g(ng, nij, nv, ZYXg, ng, false, t == 0 ? P : Q, nv, false, Wy, ng)));
          RPA_CUDA(h, rpa::launch_dot_partials(Wx, ng, Wy, ng, ng, nij, nullptr, slot(pair, t == 0 ? 1 : 0),
                                               h->stream));
        }
      }
      // G(ba; ji) for 2g..2j and G(bj; ai) for 2b..2d: the k sum becomes one GEMM over the
      // packed PNO blocks of orbital j against per-k QS slots (zero where a pair has no PNOs)
      const int ncj = ncol[j];
      const double* pj = pack + (size_t)nv * pack_off[j];
      double* QSg = static_cast<double*>(h->jQS.p);
      double* QSb = QSg + (size_t)nv * maxcol;
      RPA_CUDA(h, cudaMemsetAsync(QSg, 0, (size_t)nv * maxcol * 2 * 8, h->stream));
      for (int gi = 0; gi < 3; ++gi) {
        const GroupRef& gr = groups[(size_t)3 * pair + gi];
        RPA_CUDA(h, rpa::launch_gemm_f64_grouped_dev(dprob + gr.desc, dstart + gr.start, gr.nprob, gr.ntiles,
                                                     gr.am, gr.bn, h->stream));
      }
      // the G products have few output tiles and K = sum_k 2 Nkj: split K (about 600 CTA slots)
      for (int t = 0; t < 2; ++t) {
        rpa::GemmF64Args gk = gemm_g(nv, nv, ncj, pj, nv, false, t == 0 ? QSg : QSb, nv, true, t == 0 ? Gg : Gb, nv,
                                     1.0, 0.0);
        gk.splitk = std::max(1, std::min({64, ncj / 256, 600 / std::max(1, rpa::gemm_f64_tiles(gk))}));
        gk.work = static_cast<double*>(h->jSK.p);
        RPA_CUDA(h, G(gk));
      }
      // Tr V G: sum_ga Y(g,a) ZXX(g) (Y G)(g,a)  and  sum_ga (ZYX G)(g,a) X(g,i) Y(g,a)
      rpa::GemmF64Args gg = gemm_g(ng, nv, nv, Yd, ldy, false, Gg, nv, false, Wg, ng);
      gg.rowscale = zg;
      RPA_CUDA(h, G(gg));
      RPA_CUDA(h, rpa::launch_dot_partials(Yd, ldy, Wg, ng, ng, nv, nullptr, slot(pair, 2), h->stream));
      RPA_CUDA(h, G(gemm_g(ng, nv, nv, ZYXg, ng, false, Gb, nv, false, Wg, ng)));
      RPA_CUDA(h, rpa::launch_dot_partials(Wg, ng, Yd, ldy, ng, nv, xi, slot(pair, 3), h->stream));
    }
  }
  RPA_CUDA(h, cudaEventRecord(h->ev[3], h->stream));
  std::vector<double> ph((size_t)nslot * rpa::kDotPartials);
  RPA_CUDA(h, cudaMemcpyAsync(ph.data(), part, ph.size() * 8, cudaMemcpyDeviceToHost, h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[4], h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  auto total = [&](int64_t p, int term) {
    dd acc{0.0, 0.0};
    const double* q = ph.data() + (size_t)(5 * p + term) * rpa::kDotPartials;
    for (int b = 0; b < rpa::kDotPartials; ++b) acc = rpa::dd_add(acc, q[b]);
    return acc.hi + acc.lo;
  };
  dd erpa{0.0, 0.0}, e1b{0.0, 0.0}, e2bcd{0.0, 0.0}, e2ghij{0.0, 0.0};
  for (int64_t p = 0; p < npairs; ++p) {
    const double weight = (pair_ij[p].first != pair_ij[p].second) ? 2.0 : 1.0;
    erpa = rpa::dd_add(erpa, 2.0 * weight * total(p, 0));
    e1b = rpa::dd_add(e1b, -2.0 * weight * total(p, 1));
    bool contrib = true;
    if (BoysScreening) contrib = std::sqrt(std::fabs(maxvabab * total(p, 4))) > CutoffThreshVabij;
    if (contrib) e2ghij = rpa::dd_add(e2ghij, total(p, 2));
    e2bcd = rpa::dd_add(e2bcd, total(p, 3));
  }
  if ((s = finite_or_fail(h, {erpa.hi, e1b.hi, e2bcd.hi, e2ghij.hi}, "PNO correction energy"))) return s;
  Energies[0] = erpa.hi + erpa.lo;
  Energies[1] = e1b.hi + e1b.lo;
  Energies[2] = e2bcd.hi + e2bcd.lo;
  Energies[3] = e2ghij.hi + e2ghij.lo;
  finish_timings(h);
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}

// The batched energies of instances with at most kMaxKgLaunch frequencies each (one frequency group
// per instance).  Called by rpa_b200_ec_batched after begin_call and the argument checks.
static int ec_batched_groups(rpa_b200_handle* h, int64_t ninst, const rpa_instance* inst, int64_t prec, double* Ec,
                             double* Eu) {
  int s = RPA_OK;
  const int n = (int)ninst;
  std::vector<Validated> v(n);
  std::vector<int64_t> eu_off(n + 1, 0);
  size_t host_R = 0, total_nov = 0;
  for (int i = 0; i < n; ++i) {
    const rpa_instance& I = inst[i];
    if ((s = validate_common(h, I.NQ, I.NOcc, I.NVirt, I.R, I.ldR, I.OccEnergies, I.VirtEnergies, I.NFreqs, I.Freqs,
                             I.alpha, prec, v[i])))
      return fail(h, s, "instance %d: %s", i, h->last_error.c_str());
    if (!I.FreqWeights) return fail(h, RPA_ERR_INVALID_ARG, "instance %d: FreqWeights is NULL", i);
    if ((s = fetch_small(h, I.FreqWeights, I.NFreqs, v[i].weights))) return s;
    eu_off[i + 1] = eu_off[i] + I.NFreqs;
    if (!is_device_ptr(I.R)) host_R += (size_t)I.NQ * v[i].nov;
    total_nov += (size_t)v[i].nov;
  }
  // stage host R into one packed buffer (ld = NQ); D(ai) of every instance in one buffer
  std::vector<const double*> Rd(n);
  std::vector<int64_t> ldR(n), Doff(n);
  RPA_CUDA(h, ensure(h->R, host_R * 8));
  RPA_CUDA(h, ensure(h->D, total_nov * 8));
  {
    size_t off = 0, doff = 0;
    std::vector<double> Dh(total_nov);
    for (int i = 0; i < n; ++i) {
      const rpa_instance& I = inst[i];
      if (is_device_ptr(I.R)) {
        Rd[i] = I.R;
        ldR[i] = I.ldR;
      } else {
        double* dst = static_cast<double*>(h->R.p) + off;
        RPA_CUDA(h, cudaMemcpy2DAsync(dst, (size_t)I.NQ * 8, I.R, (size_t)I.ldR * 8, (size_t)I.NQ * 8,
                                      (size_t)v[i].nov, cudaMemcpyHostToDevice, h->stream));
        Rd[i] = dst;
        ldR[i] = I.NQ;
        off += (size_t)I.NQ * v[i].nov;
      }
      Doff[i] = (int64_t)doff;
      for (int64_t ii = 0; ii < v[i].no; ++ii)
        for (int64_t a = 0; a < v[i].nv; ++a) Dh[doff + a + v[i].nv * ii] = v[i].ev[a] - v[i].eo[ii];
      doff += (size_t)v[i].nov;
    }
    RPA_CUDA(h, cudaMemcpyAsync(h->D.p, Dh.data(), total_nov * 8, cudaMemcpyHostToDevice, h->stream));
    RPA_CUDA(h, cudaMemsetAsync(h->count_dev, 0, sizeof(int), h->stream));
    {  // one screening launch for every instance: the NQ rows of each column (not an ld > NQ padding)
      std::vector<const double*> ptrs(n);
      std::vector<int64_t> dims(3 * (size_t)n);
      int64_t widest = 0;
      for (int i = 0; i < n; ++i) {
        ptrs[i] = Rd[i];
        dims[3 * i] = ldR[i];
        dims[3 * i + 1] = v[i].NQ;
        dims[3 * i + 2] = v[i].nov;
        widest = std::max(widest, v[i].nov);
      }
      RPA_CUDA(h, ensure(h->bRes, (size_t)n * 32 + 64));
      char* scr = static_cast<char*>(h->bRes.p);
      RPA_CUDA(h, cudaMemcpyAsync(scr, ptrs.data(), (size_t)n * 8, cudaMemcpyHostToDevice, h->stream));
      RPA_CUDA(h, cudaMemcpyAsync(scr + (size_t)n * 8, dims.data(), (size_t)n * 24, cudaMemcpyHostToDevice, h->stream));
      const int per = (int)std::min<int64_t>(1024, std::max<int64_t>(1, (widest + 15) / 16));
      RPA_CUDA(h, rpa::launch_count_nonfinite_multi(reinterpret_cast<const double* const*>(scr),
                                                    reinterpret_cast<const int64_t*>(scr + (size_t)n * 8), n, per,
                                                    h->count_dev, h->stream));
      RPA_CUDA(h, cudaStreamSynchronize(h->stream));  // ptrs and dims must outlive their copies
    }
    int cnt = 0;
    RPA_CUDA(h, cudaMemcpyAsync(&cnt, h->count_dev, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    RPA_CUDA(h, cudaStreamSynchronize(h->stream));  // Dh must outlive its copy
    if (cnt) return fail(h, RPA_ERR_NONFINITE, "%d non-finite entries in the Cholesky vectors", cnt);
  }
  RPA_CUDA(h, cudaEventRecord(h->ev[1], h->stream));
  const double* D = static_cast<const double*>(h->D.p);

  // ---- batch plan: greedy packing in instance order under a memory budget
  struct Per {
    int64_t pitch;
    rpa::SplitPlan plan;
    size_t xb, pib, smallb;
  };
  std::vector<Per> per(n);
  for (int i = 0; i < n; ++i) {
    const int64_t nov = v[i].nov;
    per[i].pitch = (nov + 7) / 8 * 8;
    per[i].plan = rpa::plan_scale_split(v[i].NQ, nov, h->num_sms);
    per[i].xb = prec == RPA_PREC_SPLIT_BF16 ? (size_t)v[i].K * v[i].NQ * per[i].pitch * 2 : 0;  // each of hi, lo
    per[i].pib = (size_t)v[i].K * v[i].NQ * v[i].NQ * 8;
    per[i].smallb = (size_t)v[i].K * v[i].NQ * 8 * (2 + per[i].plan.nsplit) + 64 * (size_t)v[i].K;
  }
  if (prec == RPA_PREC_FP64) {  // the bf16 operands are not used: give their memory to Pi
    RPA_CUDA(h, cudaStreamSynchronize(h->stream));
    release(h->Xhi);
    release(h->Xlo);
  }
  size_t freeB = 0, totalB = 0;
  RPA_CUDA(h, cudaMemGetInfo(&freeB, &totalB));
  // buffers that ensure() below may free and reallocate count as available
  const size_t have = h->Xhi.bytes + h->Xlo.bytes + h->Pi.bytes + h->Ldiag.bytes;
  const size_t budget = h->batch_bytes > 0 ? h->batch_bytes : (size_t)(0.6 * (double)(freeB + have));
  std::vector<std::pair<int, int>> batches;  // [b0, b1)
  {
    size_t acc = 0;
    int b0 = 0;
    for (int i = 0; i < n; ++i) {
      const size_t need = 2 * per[i].xb + per[i].pib + per[i].smallb;
      if (i > b0 && acc + need > budget) {
        batches.push_back({b0, i});
        b0 = i;
        acc = 0;
      }
      acc += need;
    }
    batches.push_back({b0, n});
  }
  size_t maxX = 0, maxPi = 0, maxSmall = 0;
  std::vector<size_t> desc_off(batches.size() + 1, 0), res_off(batches.size() + 1, 0);
  for (size_t b = 0; b < batches.size(); ++b) {
    size_t x = 0, pi = 0, sm = 0, units = 0, work = 0, mats = 0;
    for (int i = batches[b].first; i < batches[b].second; ++i) {
      x += per[i].xb;
      pi += per[i].pib;
      sm += per[i].smallb;
      units += (size_t)v[i].K * rpa::syrk_tc_blocks(v[i].NQ);
      work += (size_t)per[i].plan.qtiles * per[i].plan.nsplit;
      mats += (size_t)v[i].K;
    }
    const int ni = batches[b].second - batches[b].first;
    const size_t desc = ((sizeof(rpa::SyrkInst) * ni + 255) / 256 + (sizeof(rpa::SplitJob) * ni + 255) / 256 +
                         (sizeof(int64_t) * (ni + 1) + 255) / 256 + (sizeof(uint4) * units + 255) / 256 +
                         (sizeof(int4) * work + 255) / 256 + (sizeof(rpa::MatDesc) * mats + 255) / 256) *
                        256;
    desc_off[b + 1] = desc_off[b] + desc;
    res_off[b + 1] = res_off[b] + mats * 4;  // tr_dd, ld_dd per matrix
    maxX = std::max(maxX, x);
    maxPi = std::max(maxPi, pi);
    maxSmall = std::max(maxSmall, sm);
  }
  if (prec == RPA_PREC_SPLIT_BF16) {
    RPA_CUDA(h, ensure(h->Xhi, maxX + 256));
    RPA_CUDA(h, ensure(h->Xlo, maxX + 256));
  }
  RPA_CUDA(h, ensure(h->Pi, maxPi + 256));
  // small per-batch buffers (exact diagonals, pivots, split partials) alternate between two halves:
  // the next batch's scale/split pass runs while this batch's log-det still reads its pivots
  const size_t smallStride = (maxSmall + 255) / 256 * 256;
  RPA_CUDA(h, ensure(h->Ldiag, 2 * smallStride + 256));
  RPA_CUDA(h, ensure(h->bDesc, desc_off.back() + 256));
  RPA_CUDA(h, ensure(h->bRes, res_off.back() * 8 + 256));

  // wave-milestone counters of every batch's multi-instance SYRK, allocated once for the call
  std::vector<int64_t> sync_off(batches.size() + 1, 0);
  std::vector<int> sync_max_chunks(batches.size(), 0);
  for (size_t b = 0; b < batches.size(); ++b) {
    size_t nu = 0;
    int mc = 0;
    for (int i = batches[b].first; i < batches[b].second; ++i) {
      nu += (size_t)v[i].K * rpa::syrk_tc_blocks(v[i].NQ);
      mc = std::max(mc, (int)((v[i].nov + rpa::kSyrkTcTK - 1) / rpa::kSyrkTcTK));
    }
    sync_max_chunks[b] = mc;
    const int64_t words =
        prec == RPA_PREC_SPLIT_BF16 ? rpa::syrk_tc_multi_sync_words((int)nu, mc, h->num_sms, h->sync_every) : 0;
    sync_off[b + 1] = sync_off[b] + words;
  }
  if (sync_off.back() > 0) RPA_CUDA(h, ensure(h->syncBuf, (size_t)sync_off.back() * sizeof(int)));
  // graph cache key: shapes, pointers and workspace addresses of this call
  uint64_t key = 1469598103934665603ull;
  auto mix = [&](uint64_t x) { key = (key ^ x) * 1099511628211ull; };
  mix((uint64_t)prec);
  mix((uint64_t)h->seg_chunks);
  for (void* p : {h->Xhi.p, h->Xlo.p, h->Pi.p, h->Ldiag.p, h->bDesc.p, h->bRes.p, h->D.p, h->syncBuf.p,
                  (void*)h->stream})
    mix((uint64_t)(uintptr_t)p);
  for (int i = 0; i < n; ++i) {
    mix((uint64_t)(uintptr_t)Rd[i]);
    mix((uint64_t)ldR[i]);
    mix((uint64_t)v[i].NQ);
    mix((uint64_t)v[i].nov);
    for (int k = 0; k < v[i].K; ++k) {
      uint64_t bits;
      std::memcpy(&bits, &v[i].freqs[k], 8);
      mix(bits);
    }
    uint64_t ab;
    std::memcpy(&ab, &inst[i].alpha, 8);
    mix(ab);
  }
  // the key also covers the log-det tile plans (the tuner below may add some)
  auto keyed = [&](uint64_t version) { return (key ^ version) * 1099511628211ull; };
  const bool cached = (h->bgraph.key == keyed(h->plans_version) && h->bgraph.execs.size() == 1);
  if (!cached) {
    for (auto e : h->bgraph.execs) cudaGraphExecDestroy(e);
    h->bgraph.execs.clear();
    h->bgraph.launches.clear();
    h->bgraph.key = 0;
  }
  uint8_t* descBase = static_cast<uint8_t*>(h->bDesc.p);
  double* resBase = static_cast<double*>(h->bRes.p);
  if (cached) {
    RPA_CUDA(h, cudaGraphLaunch(h->bgraph.execs[0], h->stream));
    rpa::g_launches += h->bgraph.launches[0];
  } else {
    // ---- per batch: descriptors on the device, log-det order buckets, milestone counters
    struct Bucket {
      int first, count, nmax;  // matrices [first, first + count) of the batch's (bucket-sorted) list
      int tune_count, tune_nmax;  // the tuner's subset: the first tune_count of them
      double cost;                // sum of n^3
    };
    struct BatchDev {
      rpa::SyrkInst* sinst = nullptr;
      uint4* units = nullptr;
      int nunits = 0;
      rpa::SplitJob* jobs = nullptr;
      int4* work = nullptr;
      int nwork = 0;
      int64_t* offs = nullptr;
      int ni = 0;
      int64_t offs_total = 0;
      rpa::MatDesc* mats = nullptr;
      std::vector<Bucket> buckets;
      std::vector<rpa::DsyrkArgs> fp64;  // FP64 form: one scaled SYRK per instance
      int* msync = nullptr;
      int64_t sync_words = 0;
      int max_chunks = 0;
    };
    std::vector<BatchDev> bd(batches.size());
    for (size_t b = 0; b < batches.size(); ++b) {
      const int i0 = batches[b].first, i1 = batches[b].second, ni = i1 - i0;
      std::vector<rpa::SyrkInst> sinst(ni);
      std::vector<rpa::SplitJob> jobs(ni);
      std::vector<int64_t> offs(ni + 1, 0);
      std::vector<uint4> units;
      std::vector<int> unit_len;  // K chunks of each instance's units
      std::vector<int4> work;
      std::vector<rpa::MatDesc> mats;
      std::vector<uint2> coords;
      size_t xo = 0, po = 0, so = smallStride * (b & 1);
      double* res = resBase + res_off[b];
      BatchDev& dv = bd[b];
      for (int t = 0; t < ni; ++t) {
        const int i = i0 + t;
        const int NQ = v[i].NQ, K = v[i].K;
        const int64_t nov = v[i].nov;
        __nv_bfloat16* xh = reinterpret_cast<__nv_bfloat16*>(static_cast<uint8_t*>(h->Xhi.p) + xo);
        __nv_bfloat16* xl = reinterpret_cast<__nv_bfloat16*>(static_cast<uint8_t*>(h->Xlo.p) + xo);
        double* Pi = reinterpret_cast<double*>(static_cast<uint8_t*>(h->Pi.p) + po);
        double* smallp = reinterpret_cast<double*>(static_cast<uint8_t*>(h->Ldiag.p) + so);
        double* diag = smallp;                          // K*NQ
        double* Ldiag = diag + (size_t)K * NQ;          // K*NQ
        double* dpart = Ldiag + (size_t)K * NQ;         // nsplit*K*NQ
        xo += (per[i].xb + 255) / 256 * 256;
        po += (per[i].pib + 255) / 256 * 256;
        so += (per[i].smallb + 255) / 256 * 256;
        if (prec == RPA_PREC_SPLIT_BF16) {
          rpa::SplitJob& j = jobs[t];
          j.R = Rd[i];
          j.ldR = ldR[i];
          j.NQ = NQ;
          j.nov = nov;
          j.D = D + Doff[i];
          j.fg.n = K;
          for (int k = 0; k < K; ++k) j.fg.u2[k] = v[i].freqs[k] * v[i].freqs[k];
          j.alpha = inst[i].alpha;
          if ((s = encode_store_maps(h, &j.tm_hi, &j.tm_lo, xh, xl, nov, NQ, K, per[i].pitch))) return s;
          j.diag_part = dpart;
          j.ai_per_split = per[i].plan.ai_per_split;
          j.nsplit = per[i].plan.nsplit;
          j.diag = diag;
          offs[t + 1] = offs[t] + (int64_t)K * NQ;
          for (int q = 0; q < per[i].plan.qtiles; ++q)
            for (int sp = 0; sp < per[i].plan.nsplit; ++sp) work.push_back(make_int4(t, q, sp, 0));
          rpa::SyrkInst& si = sinst[t];
          if ((s = encode_map(h, &si.tmAh, xh, nov, NQ, K, per[i].pitch, rpa::kSyrkTcTM))) return s;
          if ((s = encode_map(h, &si.tmAl, xl, nov, NQ, K, per[i].pitch, rpa::kSyrkTcTM))) return s;
          if ((s = encode_map(h, &si.tmBh, xh, nov, NQ, K, per[i].pitch, rpa::kSyrkTcTN))) return s;
          if ((s = encode_map(h, &si.tmBl, xl, nov, NQ, K, per[i].pitch, rpa::kSyrkTcTN))) return s;
          si.Pi = Pi;
          si.ldPi = NQ;
          si.piStride = (int64_t)NQ * NQ;
          si.diag = diag;
          si.NQ = NQ;
          si.nchunks = (int)((nov + rpa::kSyrkTcTK - 1) / rpa::kSyrkTcTK);
          rpa::syrk_tc_block_coords(NQ, coords);
          for (int k = 0; k < K; ++k)
            for (const uint2& c : coords) units.push_back(make_uint4((unsigned)t, (unsigned)k, c.x, c.y));
          unit_len.push_back(si.nchunks);
        } else {
          rpa::DsyrkArgs a{};
          a.A = Rd[i];
          a.lda = ldR[i];
          a.strideA = 0;
          a.C = Pi;
          a.ldc = NQ;
          a.strideC = (int64_t)NQ * NQ;
          a.n = NQ;
          a.kdim = nov;
          a.batch = K;
          a.D = D + Doff[i];
          a.alpha = inst[i].alpha;
          for (int k = 0; k < K; ++k) a.u2[k] = v[i].freqs[k] * v[i].freqs[k];
          dv.fp64.push_back(a);
        }
        for (int k = 0; k < K; ++k) {
          rpa::MatDesc md;
          md.A = Pi + (size_t)k * NQ * NQ;
          md.ld = NQ;
          md.n = NQ;
          md.Ldiag = Ldiag + (size_t)k * NQ;
          md.tr_dd = res + 4 * mats.size();
          md.ld_dd = md.tr_dd + 2;
          mats.push_back(md);
        }
      }
      // longest units first: the persistent CTAs take units round robin, so a descending order
      // leaves the short units for the end of the launch (stable: an instance's units stay together)
      std::stable_sort(units.begin(), units.end(),
                       [&](const uint4& a, const uint4& c) { return unit_len[a.x] > unit_len[c.x]; });
      // log-det matrices grouped by order bucket (each keeps its own result slots)
      std::stable_sort(mats.begin(), mats.end(),
                       [](const rpa::MatDesc& a, const rpa::MatDesc& c) { return plan_bucket(a.n) < plan_bucket(c.n); });
      for (int m = 0; m < (int)mats.size(); ++m) {
        if (dv.buckets.empty() || plan_bucket(mats[m].n) != plan_bucket(mats[dv.buckets.back().first].n))
          dv.buckets.push_back({m, 0, 0, 0, 0, 0.0});
        Bucket& bk = dv.buckets.back();
        ++bk.count;
        bk.nmax = std::max(bk.nmax, mats[m].n);
        bk.cost += std::pow((double)mats[m].n, 3);
        if (bk.tune_count < 128) {
          ++bk.tune_count;
          bk.tune_nmax = std::max(bk.tune_nmax, mats[m].n);
        }
      }
      // descriptors -> device (laid out as in desc_off)
      uint8_t* d = descBase + desc_off[b];
      auto put = [&](const void* src, size_t bytes) {
        uint8_t* at = d;
        if (bytes) cudaMemcpyAsync(at, src, bytes, cudaMemcpyHostToDevice, h->stream);
        d += (bytes + 255) / 256 * 256;
        return at;
      };
      dv.sinst = reinterpret_cast<rpa::SyrkInst*>(put(sinst.data(), sizeof(rpa::SyrkInst) * sinst.size()));
      dv.jobs = reinterpret_cast<rpa::SplitJob*>(put(jobs.data(), sizeof(rpa::SplitJob) * jobs.size()));
      dv.offs = reinterpret_cast<int64_t*>(put(offs.data(), sizeof(int64_t) * offs.size()));
      dv.units = reinterpret_cast<uint4*>(put(units.data(), sizeof(uint4) * units.size()));
      dv.work = reinterpret_cast<int4*>(put(work.data(), sizeof(int4) * work.size()));
      dv.mats = reinterpret_cast<rpa::MatDesc*>(put(mats.data(), sizeof(rpa::MatDesc) * mats.size()));
      RPA_CUDA(h, cudaGetLastError());
      RPA_CUDA(h, cudaStreamSynchronize(h->stream));  // host vectors must outlive their copies
      dv.nunits = (int)units.size();
      dv.nwork = (int)work.size();
      dv.ni = ni;
      dv.offs_total = offs.back();
      dv.max_chunks = sync_max_chunks[b];
      dv.sync_words = sync_off[b + 1] - sync_off[b];
      dv.msync = dv.sync_words > 0 ? static_cast<int*>(h->syncBuf.p) + sync_off[b] : nullptr;
    }
    // ---- tile plans of order buckets met for the first time, tuned on this call's own buffers
    if (h->autotune) {
      for (const BatchDev& dv : bd)
        for (const Bucket& bk : dv.buckets)
          if (!h->logdet_plans.count(plan_bucket(bk.nmax)))
            if ((s = tune_logdet_on(h, dv.mats + bk.first, bk.tune_count, bk.tune_nmax, nullptr))) return s;
      RPA_CUDA(h, cudaMemsetAsync(h->err_dev, 0, sizeof(int), h->stream));
    }
    // ---- one graph for the whole call.  Split form: batch b+1's scale/split pass (branch aux[0])
    // overlaps batch b's log-det; its SYRK waits for both.  Log-det order buckets run on up to
    // three branches, longest first.
    cudaStream_t S0 = h->stream, S1 = h->aux[0];
    cudaStream_t br[3] = {h->stream, h->aux[1], h->aux[2]};
    auto split_pass = [&](const BatchDev& dv, cudaStream_t st) {
      cudaError_t r = cudaSuccess;
      if (dv.sync_words > 0) r = cudaMemsetAsync(dv.msync, 0, (size_t)dv.sync_words * sizeof(int), st);
      if (r == cudaSuccess) r = rpa::launch_scale_split_multi(dv.jobs, dv.work, dv.nwork, dv.offs, dv.ni, dv.offs_total,
                                                           h->err_dev, st);
      return r;
    };
    auto logdet = [&](const BatchDev& dv) {
      const int nb = (int)dv.buckets.size();
      const int nbr = std::min(3, nb);
      std::vector<int> order(nb);
      for (int i = 0; i < nb; ++i) order[i] = i;
      std::stable_sort(order.begin(), order.end(),
                       [&](int a, int c) { return dv.buckets[a].cost > dv.buckets[c].cost; });
      double load[3] = {0.0, 0.0, 0.0};
      std::vector<int> branch(nb, 0);
      for (int i : order) {
        int j = 0;
        for (int q = 1; q < nbr; ++q)
          if (load[q] < load[j]) j = q;
        branch[i] = j;
        load[j] += dv.buckets[i].cost;
      }
      cudaError_t r = cudaSuccess;
      if (nbr > 1) {
        r = cudaEventRecord(h->fork_ev[0], S0);
        for (int j = 1; j < nbr && r == cudaSuccess; ++j) r = cudaStreamWaitEvent(br[j], h->fork_ev[0], 0);
      }
      for (int i : order) {
        if (r != cudaSuccess) break;
        const Bucket& bk = dv.buckets[i];
        r = rpa::launch_logdet_varlen(dv.mats + bk.first, bk.count, bk.nmax, h->err_dev, br[branch[i]],
                                      plan_for(h, bk.nmax), h->lookahead ? &h->la[branch[i]] : nullptr);
      }
      for (int j = 1; j < nbr && r == cudaSuccess; ++j) {
        r = cudaEventRecord(h->fork_ev[j], br[j]);
        if (r == cudaSuccess) r = cudaStreamWaitEvent(S0, h->fork_ev[j], 0);
      }
      return r;
    };
    const int64_t before = rpa::g_launches;
    cudaGraph_t graph = nullptr;
    RPA_CUDA(h, cudaStreamBeginCapture(S0, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    const int nbatch = (int)bd.size();
    if (prec == RPA_PREC_SPLIT_BF16) {
      e = split_pass(bd[0], S0);
      for (int b = 0; b < nbatch && e == cudaSuccess; ++b) {
        const BatchDev& dv = bd[b];
        e = rpa::launch_syrk_split_bf16_multi(dv.sinst, dv.units, dv.nunits,
                                              h->seg_chunks > 0 ? h->seg_chunks : 1 << 30, h->err_dev, h->num_sms,
                                              S0, dv.msync, h->sync_every, 2, dv.max_chunks);
        const bool next = b + 1 < nbatch;
        if (next && e == cudaSuccess) e = cudaEventRecord(h->fork_ev[3], S0);
        if (next && e == cudaSuccess) e = cudaStreamWaitEvent(S1, h->fork_ev[3], 0);
        if (next && e == cudaSuccess) e = split_pass(bd[b + 1], S1);
        if (next && e == cudaSuccess) e = cudaEventRecord(h->fork_ev[4], S1);
        if (e == cudaSuccess) e = logdet(dv);
        if (next && e == cudaSuccess) e = cudaStreamWaitEvent(S0, h->fork_ev[4], 0);
      }
    } else {
      for (int b = 0; b < nbatch && e == cudaSuccess; ++b) {
        for (const rpa::DsyrkArgs& a : bd[b].fp64) {
          e = rpa::launch_dsyrk_lower(a, S0);
          if (e != cudaSuccess) break;
        }
        if (e == cudaSuccess) e = logdet(bd[b]);
      }
    }
    cudaError_t e2 = cudaStreamEndCapture(S0, &graph);
    const int64_t count = rpa::g_launches - before;
    rpa::g_launches = before;
    if (e != cudaSuccess || e2 != cudaSuccess || !graph) {
      if (graph) cudaGraphDestroy(graph);
      return fail(h, RPA_ERR_CUDA, "capture of the batched launch sequence failed: %s",
                  cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    cudaGraphExec_t exec = nullptr;
    cudaError_t ei = cudaGraphInstantiate(&exec, graph, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return fail(h, RPA_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(ei));
    h->bgraph.execs.push_back(exec);
    h->bgraph.launches.push_back(count);
    RPA_CUDA(h, cudaGraphLaunch(exec, h->stream));
    rpa::g_launches += count;
    h->bgraph.key = keyed(h->plans_version);
  }
  RPA_CUDA(h, cudaEventRecord(h->ev[2], h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[3], h->stream));
  std::vector<double> res(res_off.back());
  RPA_CUDA(h, cudaMemcpyAsync(res.data(), resBase, res.size() * 8, cudaMemcpyDeviceToHost, h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[4], h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  if ((s = check_device_error(h))) return s;
  // energies: results are laid out per batch in instance order, 4 doubles per (instance, frequency)
  size_t m = 0;
  for (int i = 0; i < n; ++i) {
    dd ec{0.0, 0.0};
    for (int k = 0; k < v[i].K; ++k, ++m) {
      const dd trk{res[4 * m], res[4 * m + 1]};
      const dd ldk{res[4 * m + 2], res[4 * m + 3]};
      const dd eu = rpa::dd_add_dd(ldk, {-trk.hi, -trk.lo});
      if (!std::isfinite(eu.hi)) return fail(h, RPA_ERR_NONFINITE, "non-finite E(u) in instance %d", i);
      if (Eu) Eu[eu_off[i] + k] = eu.hi + eu.lo;
      const double f = v[i].weights[k] / (2.0 * kPi);
      const double p = eu.hi * f;
      ec = rpa::dd_add_dd(ec, {p, std::fma(eu.hi, f, -p) + eu.lo * f});
    }
    Ec[i] = ec.hi + ec.lo;
  }
  finish_timings(h);
  return RPA_OK;
}

// Instances with more than kMaxKgLaunch frequencies (the reference allows up to 64 points,
// src/rpa/rpa_definitions.f90:109-110) run as consecutive frequency groups of at most
// kMaxKgLaunch points, each group a sub-instance on the same R; E(u) of the groups are already in
// the caller's order, and an instance's E_c is the sum of its groups' (a sum over frequencies).
int rpa_b200_ec_batched(rpa_b200_handle* h, int64_t ninst, const rpa_instance* inst, int64_t prec, double* Ec,
                        double* Eu) try {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
  if (ninst < 1 || ninst > (1 << 24) || !inst || !Ec)
    return fail(h, RPA_ERR_INVALID_ARG, "invalid argument to rpa_b200_ec_batched");
  if (prec != RPA_PREC_FP64 && prec != RPA_PREC_SPLIT_BF16)
    return fail(h, RPA_ERR_INVALID_ARG, "unknown precision mode %lld", (long long)prec);
  bool wide = false;
  for (int64_t i = 0; i < ninst; ++i) {
    if (inst[i].NFreqs < 1 || inst[i].NFreqs > 64)
      return fail(h, RPA_ERR_INVALID_ARG, "instance %lld: NFreqs=%lld not in [1,64]", (long long)i,
                  (long long)inst[i].NFreqs);
    if (!inst[i].Freqs || !inst[i].FreqWeights)
      return fail(h, RPA_ERR_INVALID_ARG, "instance %lld: Freqs or FreqWeights is NULL", (long long)i);
    const rpa_instance& I = inst[i];
    if ((s = check_arrays(h, {I.R, I.OccEnergies, I.VirtEnergies, I.Freqs, I.FreqWeights})))
      return fail(h, s, "instance %lld: %s", (long long)i, h->last_error.c_str());
    wide = wide || inst[i].NFreqs > rpa::kMaxKgLaunch;
  }
  if (!wide) return ec_batched_groups(h, ninst, inst, prec, Ec, Eu);
  std::vector<rpa_instance> groups;
  std::vector<int64_t> owner;
  for (int64_t i = 0; i < ninst; ++i)
    for (int64_t k0 = 0; k0 < inst[i].NFreqs; k0 += rpa::kMaxKgLaunch) {
      rpa_instance g = inst[i];
      g.NFreqs = std::min<int64_t>(rpa::kMaxKgLaunch, inst[i].NFreqs - k0);
      g.Freqs = inst[i].Freqs + k0;
      g.FreqWeights = inst[i].FreqWeights + k0;
      groups.push_back(g);
      owner.push_back(i);
    }
  if (groups.size() > (size_t)(1 << 24)) return fail(h, RPA_ERR_INVALID_ARG, "too many frequency groups");
  std::vector<double> eg(groups.size());
  if ((s = ec_batched_groups(h, (int64_t)groups.size(), groups.data(), prec, eg.data(), Eu))) return s;
  std::vector<dd> acc((size_t)ninst, dd{0.0, 0.0});
  for (size_t j = 0; j < groups.size(); ++j) acc[owner[j]] = rpa::dd_add(acc[owner[j]], eg[j]);
  for (int64_t i = 0; i < ninst; ++i) Ec[i] = acc[i].hi + acc[i].lo;
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}

int rpa_b200_ec_grad(rpa_b200_handle* h, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* R, int64_t ldR,
                     const double* OccEnergies, const double* VirtEnergies, int64_t NFreqs, const double* Freqs,
                     const double* FreqWeights, double alpha, int64_t prec, double* Ec, double* dR, int64_t lddR,
                     double* dOcc, double* dVirt) try {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
  if ((s = check_arrays(h, {R, OccEnergies, VirtEnergies, Freqs, FreqWeights, dR, dOcc, dVirt}))) return s;
  Validated v;
  if ((s = validate_common(h, NQ, NOcc, NVirt, R, ldR, OccEnergies, VirtEnergies, NFreqs, Freqs, alpha, prec, v)))
    return s;
  if (!FreqWeights || !dR || lddR < NQ) return fail(h, RPA_ERR_INVALID_ARG, "invalid gradient arguments");
  if ((s = fetch_small(h, FreqWeights, NFreqs, v.weights))) return s;
  const double* Rd;
  int64_t ldd;
  if ((s = stage_R(h, v, R, ldR, &Rd, &ldd))) return s;
  RPA_CUDA(h, cudaEventRecord(h->ev[1], h->stream));
  // recompute Pi(u) for every frequency and factor 1 + Pi(u) (the energy comes out on the way)
  if ((s = build_pi(h, v, Rd, ldd, alpha, prec))) return s;
  double ec = 0.0;
  if ((s = energy_from_workspace(h, v.NQ, v.K, v.weights, &ec, nullptr))) return s;
  if (Ec) *Ec = ec;
  const int n = v.NQ;
  const int64_t nov = v.nov;
  // Y_k = (1 + Pi_k)^{-1} R for groups of frequencies sized to the free memory
  size_t freeB = 0, totalB = 0;
  RPA_CUDA(h, cudaMemGetInfo(&freeB, &totalB));
  const size_t perK = (size_t)n * nov * 8;
  int grp = (int)std::max<size_t>(1, std::min<size_t>(16, (size_t)(0.5 * (double)(freeB + h->gY.bytes)) / perK));
  grp = std::min(grp, v.K);
  RPA_CUDA(h, ensure(h->gY, perK * grp));
  RPA_CUDA(h, ensure(h->gD, (size_t)nov * 8));
  const bool dev_out = is_device_ptr(dR);
  double* dRd = dR;
  int64_t lddr = lddR;
  if (!dev_out) {
    RPA_CUDA(h, ensure(h->tU, (size_t)n * nov * 8));  // device staging of dR
    dRd = static_cast<double*>(h->tU.p);
    lddr = n;
  }
  double* Y = static_cast<double*>(h->gY.p);
  double* dD = static_cast<double*>(h->gD.p);
  const double* L = static_cast<const double*>(h->Pi.p);
  for (int g0 = 0; g0 < v.K; g0 += grp) {
    const int nb = std::min(grp, v.K - g0);
    RPA_CUDA(h, rpa::launch_replicate(Rd, ldd, n, nov, Y, n, (int64_t)n * nov, nb, h->stream));
    const double* Lg = L + (int64_t)g0 * n * n;
    RPA_CUDA(h, rpa::launch_trsm_lower_left(Lg, n, (int64_t)n * n, Y, n, (int64_t)n * nov, n, (int)nov, nb,
                                            h->stream));
    RPA_CUDA(h, rpa::launch_trsm_lower_trans_left(Lg, n, (int64_t)n * n, Y, n, (int64_t)n * nov, n, (int)nov, nb,
                                                  h->stream));
    rpa::GradGroup gg{};
    gg.n = nb;
    gg.alpha = alpha;
    for (int k = 0; k < nb; ++k) {
      gg.u2[k] = v.freqs[g0 + k] * v.freqs[g0 + k];
      gg.f[k] = v.weights[g0 + k] / (2.0 * kPi);
    }
    RPA_CUDA(h, rpa::launch_grad_accum(Rd, ldd, Y, n, (int64_t)n * nov, n, nov, static_cast<const double*>(h->D.p),
                                       gg, dRd, lddr, dD, g0 == 0, h->stream));
  }
  if (!dev_out)
    RPA_CUDA(h, cudaMemcpy2DAsync(dR, (size_t)lddR * 8, dRd, (size_t)n * 8, (size_t)n * 8, (size_t)nov,
                                  cudaMemcpyDeviceToHost, h->stream));
  std::vector<double> dDh((size_t)nov);
  RPA_CUDA(h, cudaMemcpyAsync(dDh.data(), dD, (size_t)nov * 8, cudaMemcpyDeviceToHost, h->stream));
  RPA_CUDA(h, cudaEventRecord(h->ev[4], h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  if ((s = check_device_error(h))) return s;
  // dE/de_a = sum_i dE/dD(ai), dE/de_i = -sum_a dE/dD(ai)
  if (dOcc || dVirt) {
    std::vector<double> go((size_t)v.no, 0.0), gv((size_t)v.nv, 0.0);
    for (int64_t i = 0; i < v.no; ++i)
      for (int64_t a = 0; a < v.nv; ++a) {
        const double x = dDh[(size_t)(a + v.nv * i)];
        go[i] -= x;
        gv[a] += x;
      }
    std::vector<double>* outs[2] = {&go, &gv};
    double* dst[2] = {dOcc, dVirt};
    for (int t = 0; t < 2; ++t) {
      if (!dst[t]) continue;
      if (is_device_ptr(dst[t]))
        RPA_CUDA(h, cudaMemcpy(dst[t], outs[t]->data(), outs[t]->size() * 8, cudaMemcpyHostToDevice));
      else
        std::memcpy(dst[t], outs[t]->data(), outs[t]->size() * 8);
    }
  }
  finish_timings(h);
  return RPA_OK;
} catch (...) {
  return exception_status(h);
}

}  // extern "C"
