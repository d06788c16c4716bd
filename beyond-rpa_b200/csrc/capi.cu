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
#include <string>
#include <vector>

#include "kernels.h"

using rpa::dd;

namespace rpa {
thread_local int64_t g_launches = 0;
}

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

struct rpa_b200_handle {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;      // stream the calls run on
  cudaStream_t own_stream = nullptr;  // the handle's own stream
  std::string last_error;
  DevBuf R, D, eps, Xhi, Xlo, diag_part, diag, Pi, Ldiag, ddbuf;
  int* err_dev = nullptr;    // device error word
  int* count_dev = nullptr;  // non-finite counter
  PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  cudaEvent_t ev[5] = {};
  double timings[6] = {0, 0, 0, 0, 0, 0};
  int64_t launches = 0;
  int seg_chunks = 16;  // 512-column accumulation segments of the tensor-core SYRK
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
    cudaGraphExec_t exec;
    int64_t launches;
  };
  std::vector<CholGraph> chol_graphs;
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

#define RPA_CUDA(h, call)                                                                                   \
  do {                                                                                                      \
    cudaError_t e_ = (call);                                                                                \
    if (e_ != cudaSuccess) {                                                                                \
      if (e_ == cudaErrorMemoryAllocation) return fail(h, RPA_ERR_OOM, "%s: %s", #call, cudaGetErrorString(e_)); \
      return fail(h, RPA_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));                                \
    }                                                                                                       \
  } while (0)

cudaError_t ensure(DevBuf& b, size_t bytes) {
  if (b.bytes >= bytes && b.p) return cudaSuccess;
  if (b.p) {
    cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
  }
  if (bytes == 0) bytes = 256;
  cudaError_t e = cudaMalloc(&b.p, bytes);
  if (e == cudaSuccess) b.bytes = bytes;
  return e;
}

void release(DevBuf& b) {
  if (b.p) cudaFree(b.p);
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
  // NaN/Inf screen of the Cholesky vectors (ld may exceed NQ: screen the span)
  RPA_CUDA(h, cudaMemsetAsync(h->count_dev, 0, sizeof(int), h->stream));
  RPA_CUDA(h, rpa::launch_count_nonfinite(*Rd, (*ldd) * (v.nov - 1) + v.NQ, h->count_dev, h->stream));
  // orbital energies -> D(ai)
  RPA_CUDA(h, ensure(h->eps, (size_t)(v.no + v.nv) * 8));
  double* ed = static_cast<double*>(h->eps.p);
  RPA_CUDA(h, cudaMemcpyAsync(ed, v.eo.data(), (size_t)v.no * 8, cudaMemcpyHostToDevice, h->stream));
  RPA_CUDA(h, cudaMemcpyAsync(ed + v.no, v.ev.data(), (size_t)v.nv * 8, cudaMemcpyHostToDevice, h->stream));
  RPA_CUDA(h, ensure(h->D, (size_t)v.nov * 8));
  RPA_CUDA(h, rpa::launch_dai(ed, ed + v.no, v.no, v.nv, static_cast<double*>(h->D.p), h->stream));
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

// Build the lower triangles of Pi_k (k = 0..K-1) into h->Pi (ld = NQ).
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
  const size_t perFreq = (size_t)NQ * pitch * 2 * 2;  // hi + lo
  size_t freeB = 0, totalB = 0;
  RPA_CUDA(h, cudaMemGetInfo(&freeB, &totalB));
  const size_t have = h->Xhi.bytes + h->Xlo.bytes;
  size_t budget = (size_t)((double)(freeB + have) * 0.7);
  int kg = (int)std::min<size_t>((size_t)std::min(v.K, rpa::kMaxKgLaunch), std::max<size_t>(1, budget / perFreq));
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
    cudaEvent_t e0 = pool_event(h), e1 = pool_event(h), e2 = pool_event(h);
    RPA_CUDA(h, cudaEventRecord(e0, h->stream));
    RPA_CUDA(h, rpa::launch_scale_split(Rd, ldR, NQ, nov, D, fg, alpha, static_cast<__nv_bfloat16*>(h->Xhi.p),
                                        static_cast<__nv_bfloat16*>(h->Xlo.p), pitch, (int64_t)NQ * pitch,
                                        static_cast<double*>(h->diag_part.p), diag, plan, h->stream));
    RPA_CUDA(h, cudaEventRecord(e1, h->stream));
    h->split_ev.push_back({e0, e1});
    CUtensorMap mAh, mAl, mBh, mBl;
    int s;
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
    RPA_CUDA(h, rpa::launch_syrk_split_bf16(&mAh, &mAl, &mBh, &mBl, a, h->num_sms, h->stream));
    RPA_CUDA(h, cudaEventRecord(e2, h->stream));
    h->tc_ev.push_back({e1, e2});
  }
  return RPA_OK;
}

// Blocked Cholesky of nmat matrices through a cached CUDA graph (the launch
// sequence depends only on the arguments; ~6 launches per 64 columns would
// otherwise leave the GPU idle between the small late-step kernels).
int cholesky(rpa_b200_handle* h, double* A, int64_t ld, int64_t stride, int n, int nmat, double* Ldiag) {
  for (auto& g : h->chol_graphs) {
    if (g.A == A && g.ld == ld && g.stride == stride && g.n == n && g.nmat == nmat && g.Ldiag == Ldiag &&
        g.stream == h->stream) {
      RPA_CUDA(h, cudaGraphLaunch(g.exec, h->stream));
      rpa::g_launches += g.launches;
      return RPA_OK;
    }
  }
  const int64_t before = rpa::g_launches;
  cudaGraph_t graph = nullptr;
  if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
    cudaError_t e = rpa::launch_cholesky_lower(A, ld, stride, n, nmat, Ldiag, h->err_dev, h->stream);
    cudaError_t e2 = cudaStreamEndCapture(h->stream, &graph);
    const int64_t count = rpa::g_launches - before;
    rpa::g_launches = before;
    cudaGraphExec_t exec = nullptr;
    if (e == cudaSuccess && e2 == cudaSuccess && graph &&
        cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
      cudaGraphDestroy(graph);
      if (h->chol_graphs.size() >= 8) {
        cudaGraphExecDestroy(h->chol_graphs.front().exec);
        h->chol_graphs.erase(h->chol_graphs.begin());
      }
      h->chol_graphs.push_back({A, ld, stride, n, nmat, Ldiag, h->stream, exec, count});
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
  RPA_CUDA(h, rpa::launch_cholesky_lower(A, ld, stride, n, nmat, Ldiag, h->err_dev, h->stream));
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

}  // namespace

extern "C" {

int rpa_b200_create(rpa_b200_handle** handle, int64_t device, int64_t flags) {
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
      cudaMalloc(&h->err_dev, sizeof(int)) != cudaSuccess || cudaMalloc(&h->count_dev, sizeof(int)) != cudaSuccess) {
    delete h;
    return RPA_ERR_CUDA;
  }
  h->stream = h->own_stream;
  if (const char* sc = std::getenv("RPA_B200_SEG_CHUNKS")) h->seg_chunks = std::atoi(sc);
  for (auto& e : h->ev) cudaEventCreate(&e);
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
}

int rpa_b200_destroy(rpa_b200_handle* h) {
  if (!h) return RPA_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->own_stream) cudaStreamSynchronize(h->own_stream);
  for (DevBuf* b : {&h->R, &h->D, &h->eps, &h->Xhi, &h->Xlo, &h->diag_part, &h->diag, &h->Pi, &h->Ldiag, &h->ddbuf})
    release(*b);
  if (h->err_dev) cudaFree(h->err_dev);
  if (h->count_dev) cudaFree(h->count_dev);
  for (auto& e : h->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : h->pool) cudaEventDestroy(e);
  for (auto& g : h->chol_graphs) cudaGraphExecDestroy(g.exec);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
  return RPA_OK;
}

const char* rpa_b200_status_string(int status) {
  switch (status) {
    case RPA_OK: return "success";
    case RPA_ERR_INVALID_ARG: return "invalid argument";
    case RPA_ERR_NOT_SPD: return "1+Pi(u) is not positive definite";
    case RPA_ERR_NONFINITE: return "non-finite input or result";
    case RPA_ERR_OOM: return "device out of memory";
    case RPA_ERR_CUDA: return "CUDA error";
    case RPA_ERR_TIMEOUT: return "device-side wait timed out";
    case RPA_ERR_NO_DEVICE: return "no sm_100 device";
    case RPA_ERR_NOT_CONVERGED: return "not converged";
    case RPA_ERR_TOO_LARGE: return "problem exceeds the fixed scratch of the allocation-free entry point";
    default: return "unknown status";
  }
}

const char* rpa_b200_last_error(const rpa_b200_handle* h) { return h ? h->last_error.c_str() : "null handle"; }

int rpa_b200_last_timings(const rpa_b200_handle* h, double* out, int64_t n) {
  if (!h || !out) return RPA_ERR_INVALID_ARG;
  for (int64_t i = 0; i < n && i < 6; ++i) out[i] = h->timings[i];
  return RPA_OK;
}

int64_t rpa_b200_last_launches(const rpa_b200_handle* h) { return h ? h->launches : -1; }

int rpa_b200_set_stream(rpa_b200_handle* h, void* stream) {
  if (!h) return RPA_ERR_INVALID_ARG;
  h->stream = stream ? static_cast<cudaStream_t>(stream) : h->own_stream;
  return RPA_OK;
}

int rpa_b200_pi(rpa_b200_handle* h, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* R, int64_t ldR,
                const double* OccEnergies, const double* VirtEnergies, int64_t NFreqs, const double* Freqs,
                double alpha, int64_t prec, double* PiU, int64_t ldPi) {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
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
}

int rpa_b200_ec_from_pi(rpa_b200_handle* h, int64_t NQ, int64_t NFreqs, const double* PiU, int64_t ldPi,
                        const double* FreqWeights, double* Ec, double* Eu) {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
  if (NQ < 1 || NFreqs < 1 || NFreqs > 64 || ldPi < NQ || !PiU || !FreqWeights || !Ec)
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
  RPA_CUDA(h, rpa::launch_count_nonfinite(Pi, (int64_t)K * n * n, h->count_dev, h->stream));
  int cnt = 0;
  RPA_CUDA(h, cudaMemcpyAsync(&cnt, h->count_dev, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  RPA_CUDA(h, cudaStreamSynchronize(h->stream));
  if (cnt) return fail(h, RPA_ERR_NONFINITE, "%d non-finite entries in Pi(u)", cnt);
  RPA_CUDA(h, cudaEventRecord(h->ev[1], h->stream));
  if ((s = energy_from_workspace(h, n, K, w, Ec, Eu))) return s;
  RPA_CUDA(h, cudaEventRecord(h->ev[4], h->stream));
  finish_timings(h);
  return RPA_OK;
}

int rpa_b200_ec(rpa_b200_handle* h, int64_t NQ, int64_t NOcc, int64_t NVirt, const double* R, int64_t ldR,
                const double* OccEnergies, const double* VirtEnergies, int64_t NFreqs, const double* Freqs,
                const double* FreqWeights, double alpha, int64_t prec, double* Ec, double* Eu) {
  int s = begin_call(h);
  if (s != RPA_OK) return s;
  Validated v;
  if ((s = validate_common(h, NQ, NOcc, NVirt, R, ldR, OccEnergies, VirtEnergies, NFreqs, Freqs, alpha, prec, v)))
    return s;
  if (!FreqWeights || !Ec) return fail(h, RPA_ERR_INVALID_ARG, "FreqWeights or Ec is NULL");
  if ((s = fetch_small(h, FreqWeights, NFreqs, v.weights))) return s;
  const double* Rd;
  int64_t ldd;
  if ((s = stage_R(h, v, R, ldR, &Rd, &ldd))) return s;
  RPA_CUDA(h, cudaEventRecord(h->ev[1], h->stream));
  if ((s = build_pi(h, v, Rd, ldd, alpha, prec))) return s;
  if ((s = energy_from_workspace(h, v.NQ, v.K, v.weights, Ec, Eu))) return s;
  RPA_CUDA(h, cudaEventRecord(h->ev[4], h->stream));
  finish_timings(h);
  return RPA_OK;
}

}  // extern "C"
