// Failure-detection self-test: one kernel whose wait can only end by expiring.
//
// Every spin-wait of the library's kernels is bounded (rpa_common.cuh): when its limit passes,
// the waiting thread records a code in the handle's device error word and the kernel returns,
// so that the host reports RPA_ERR_TIMEOUT and the CUDA context stays usable.  This kernel runs
// that same bounded wait on an mbarrier that no thread ever arrives on, with a caller-chosen
// limit, so a test can watch the path work end to end.  Nothing asynchronous (no TMA copy, no
// tensor-core operation) is in flight while it waits.
#include "kernels.h"
#include "rpa_common.cuh"

namespace rpa {
namespace {

__global__ void wait_timeout_selftest_kernel(int* err, unsigned long long limit_ns) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);  // expects one arrival; none comes
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_wait_slow(&bar, 0, err, kDevTimeoutSelfTest, limit_ns);
  __syncthreads();
}

}  // namespace

cudaError_t launch_wait_timeout_selftest(int* err, unsigned long long limit_ns, cudaStream_t stream) {
  wait_timeout_selftest_kernel<<<1, 32, 0, stream>>>(err, limit_ns);
  ++g_launches;
  return cudaGetLastError();
}

}  // namespace rpa
