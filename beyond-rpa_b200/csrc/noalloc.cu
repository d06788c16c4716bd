// Allocation-free variant of the energy-from-Pi entry point.
//
// Some callers cannot call cudaMalloc: a host program whose GPU memory is
// owned by a pool or arena it cannot extend, code that runs while a
// device-memory budget is frozen (for example inside a phase that must not
// change the memory footprint), or a caller holding the device under an
// allocation lock.  For them rpa_b200_ec_from_pi_noalloc computes the same
// energy as rpa_b200_ec_from_pi with no device allocation at all: its
// working storage is the file-scope array below, a fixed 32 MiB that every
// GPU which loads this library holds until the process exits.
//
// Limits and contract:
//   * the problem must fit: NFreqs*NQ*NQ + NFreqs*NQ + 4*NFreqs + 1 doubles
//     <= kNoAllocScratchDoubles (e.g. NQ = 512 with NFreqs <= 15, NQ = 400
//     with NFreqs <= 26); larger problems return RPA_ERR_TOO_LARGE before any
//     GPU work;
//   * every call on a device shares this one array and it keeps the previous
//     call's contents; the entry point clears what must start at zero (the
//     error word and the non-finite counter) at the start of each call.
//     Calls that overlap on the GPU (concurrent streams, several host
//     threads) race on the array and must be serialised by the caller;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current); make
//     this first call before any stream capture begins.  Under CUDA's lazy
//     module loading that first call is also when the array and the kernels
//     used here are loaded onto the GPU, so a caller that freezes its device
//     footprint makes one call before freezing it.
#include <cmath>
#include <mutex>
#include <vector>

#include "abi_guard.h"
#include "kernels.h"

namespace {

constexpr size_t kNoAllocScratchBytes = RPA_B200_NOALLOC_SCRATCH_BYTES;
constexpr size_t kNoAllocScratchDoubles = kNoAllocScratchBytes / sizeof(double);

// Host code may not use this name as a device address: it is a host-side
// stand-in; the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on `device` (which must be current).
cudaError_t scratch_for_device(int device, double** out) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[device] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[device];
  return cudaSuccess;
}

bool is_device_pointer(const void* p) {
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" int rpa_b200_ec_from_pi_noalloc(int64_t device, void* stream_ptr, int64_t NQ, int64_t NFreqs,
                                           const double* PiU, int64_t ldPi, const double* FreqWeights, double* Ec,
                                           double* Eu) try {
  // the same argument limits as rpa_b200_ec_from_pi; they also keep the size arithmetic below from wrapping
  if (NQ < 1 || NQ > (1 << 20) || NFreqs < 1 || NFreqs > 64 || ldPi < NQ || !PiU || !FreqWeights || !Ec)
    return RPA_ERR_INVALID_ARG;
  if (device < 0 || device >= kMaxDevices) return RPA_ERR_INVALID_ARG;
  const size_t n = (size_t)NQ, K = (size_t)NFreqs;
  // layout of the scratch: Pi copy | L_ii | traces + log sums (double-double) | error word, counter
  const size_t need = K * n * n + K * n + 4 * K + 1;
  if (need > kNoAllocScratchDoubles) return RPA_ERR_TOO_LARGE;
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess) return RPA_ERR_NO_DEVICE;
  if (cudaSetDevice((int)device) != cudaSuccess) return RPA_ERR_NO_DEVICE;
  cudaStream_t st = static_cast<cudaStream_t>(stream_ptr);
  int status = RPA_OK;
  double* base = nullptr;
  if (scratch_for_device((int)device, &base) != cudaSuccess) {
    cudaSetDevice(prev);
    return RPA_ERR_CUDA;
  }
  double* Pi = base;
  double* Ldiag = Pi + K * n * n;
  double* tr = Ldiag + K * n;
  double* ld = tr + 2 * K;
  int* flags = reinterpret_cast<int*>(ld + 2 * K);  // flags[0] = device error word, flags[1] = non-finite count
  double w[64], host[4 * 64];  // K <= 64
  int f[2] = {0, 0};
  do {
    if (is_device_pointer(FreqWeights)) {
      if (cudaMemcpyAsync(w, FreqWeights, K * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess) {
        status = RPA_ERR_CUDA;
        break;
      }
    } else {
      for (size_t k = 0; k < K; ++k) w[k] = FreqWeights[k];
    }
    if (cudaMemsetAsync(flags, 0, 2 * sizeof(int), st) != cudaSuccess) {
      status = RPA_ERR_CUDA;
      break;
    }
    cudaError_t e;
    if (is_device_pointer(PiU)) {
      e = rpa::launch_copy_lower(PiU, ldPi, ldPi * NQ, Pi, (int64_t)n, (int64_t)(n * n), (int)n, (int)K, st);
    } else {
      // PiU(ldPi, NQ, NFreqs): K*NQ consecutive columns of length NQ, pitch ldPi
      e = cudaMemcpy2DAsync(Pi, n * 8, PiU, (size_t)ldPi * 8, n * 8, n * K, cudaMemcpyHostToDevice, st);
    }
    if (e != cudaSuccess) {
      status = RPA_ERR_CUDA;
      break;
    }
    // only the lower triangle is read: the upper half of the shared array may hold an earlier call's data
    if (rpa::launch_count_nonfinite_lower(Pi, (int64_t)n, (int64_t)(n * n), (int)n, (int)K, flags + 1, st) !=
            cudaSuccess ||
        rpa::launch_trace_shift(Pi, (int64_t)n, (int64_t)(n * n), (int)n, (int)K, nullptr, tr, st) != cudaSuccess ||
        rpa::launch_cholesky_lower(Pi, (int64_t)n, (int64_t)(n * n), (int)n, (int)K, Ldiag, flags, st,
                                   rpa::default_logdet_plan()) != cudaSuccess ||
        rpa::launch_logdet_sum(Ldiag, (int)n, (int)K, ld, st) != cudaSuccess) {
      status = RPA_ERR_CUDA;
      break;
    }
    if (cudaMemcpyAsync(host, tr, 4 * K * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(f, flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      status = RPA_ERR_CUDA;
      break;
    }
    if (f[1] != 0) {
      status = RPA_ERR_NONFINITE;
      break;
    }
    if (f[0] == rpa::kDevNotSPD) {
      status = RPA_ERR_NOT_SPD;
      break;
    }
    if (f[0] != 0) {
      status = RPA_ERR_TIMEOUT;
      break;
    }
    const double kTwoPi = 6.28318530717958647692;
    rpa::dd ec{0.0, 0.0};
    for (size_t k = 0; k < K; ++k) {
      const rpa::dd trk{host[2 * k], host[2 * k + 1]};
      const rpa::dd ldk{host[2 * K + 2 * k], host[2 * K + 2 * k + 1]};
      const rpa::dd eu = rpa::dd_add_dd(ldk, {-trk.hi, -trk.lo});
      if (!std::isfinite(eu.hi)) {
        status = RPA_ERR_NONFINITE;
        break;
      }
      if (Eu) Eu[k] = eu.hi + eu.lo;
      const double fk = w[k] / kTwoPi;
      const double p = eu.hi * fk;
      ec = rpa::dd_add_dd(ec, {p, std::fma(eu.hi, fk, -p) + eu.lo * fk});
    }
    if (status == RPA_OK) *Ec = ec.hi + ec.lo;
  } while (false);
  cudaSetDevice(prev);
  return status;
} catch (...) {
  return rpa::status_of_exception(nullptr);
}
