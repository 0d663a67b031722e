// selftest.cu -- the bounded-wait path on a live GPU without a fault.
//
// Every staged copy in this library completes on an mbarrier, and every wait
// on one is bounded (mbar_wait gives up after a number of polls) and reported
// through a status word instead of hanging.  k_wait_probe exercises exactly
// that path: thread 0 arrives on a fresh barrier announcing `tx_bytes` of
// transfer; with 0 bytes the phase completes at once, with 16 bytes it never
// completes because no copy is issued (a flag that nothing sets), so the
// bounded wait runs out and the status word is set.  No memory is accessed
// out of bounds and the kernel ends in either case.
#include "fcb_common.cuh"
#include "fcb_kernels.h"

namespace fcb {

__global__ void k_wait_probe(uint32_t tx_bytes, uint32_t max_polls, int* status) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_expect_tx(&bar, tx_bytes);
  const bool ok = mbar_wait(&bar, 0u, max_polls);
  if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicExch(status, 1);
}

cudaError_t launch_wait_probe(bool arrive, uint32_t max_polls, int* status, cudaStream_t s) {
  k_wait_probe<<<1, 64, 0, s>>>(arrive ? 0u : 16u, max_polls, status);
  return cudaGetLastError();
}

}  // namespace fcb
