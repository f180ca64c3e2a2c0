// rijk_selftest.cu — self-test of the bounded device-side wait and its error path.
//
// Every mbarrier wait in the tcgen05 kernels gives up after a bounded number of SM clock cycles;
// the kernel then raises DEVERR_TIMEOUT in the context's error word, releases its TMEM and returns,
// and the next synchronising call reports RIJK_ERR_TIMEOUT.  In normal operation no wait runs out,
// so that path would go unexercised.  rijk_selftest_wait_timeout runs it on purpose, without any
// fault: one warp allocates TMEM as the exchange kernels do, waits on an mbarrier that nothing ever
// arrives on, with a short cycle limit, gives up, raises the error bit, frees the TMEM and returns.
// The context stays usable afterwards.
//
// rijk_selftest_alloc_failure makes the context's own device allocations run out on purpose, on the host:
// the chosen allocation returns RIJK_ERR_ALLOC as a cudaMalloc out of memory would, so that every
// call's allocation failure path can be exercised without exhausting a GPU.
#include <cuda_runtime.h>

#include "rijk_internal.h"
#include "tc_util.cuh"

#define RIJK_API extern "C" __attribute__((visibility("default")))

namespace rijk {
namespace {

__global__ void __launch_bounds__(32) k_wait_probe(int* err, long long limit) {
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  const int lane = threadIdx.x;
  if (lane == 0) {
    mbar_init(&bar, 1);
    abort_flag = 0;
    fence_barrier_init();
  }
  tmem_alloc(&tmem_slot, 32);  // warp-wide, as the exchange kernels' TMEM owner warp does
  tmem_relinquish();
  tc_fence_before();
  __syncwarp();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  if (lane == 0) {
    // phase 0 of `bar` never completes: its one expected arrival never comes
    if (!mbar_wait_for(&bar, 0, &abort_flag, limit)) {
      abort_flag = 1;
      atomicOr(err, DEVERR_TIMEOUT);
    }
  }
  tc_fence_before();
  __syncwarp();
  tc_fence_after();
  tmem_dealloc(tmem, 32);
}

}  // namespace
}  // namespace rijk

RIJK_API int rijk_selftest_wait_timeout(rijk_ctx* ctx, long long cycles) {
  using namespace rijk;
  if (!ctx) return RIJK_ERR_ARG;
  if (cycles < 1000 || cycles > kWaitCycles)
    return set_err(ctx, RIJK_ERR_ARG, "rijk_selftest_wait_timeout: cycles = %lld outside [1000, %lld]", cycles,
                   kWaitCycles);
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_check(ctx, e, "rijk_selftest_wait_timeout: cudaSetDevice");
  k_wait_probe<<<1, 32, 0, ctx->stream>>>(static_cast<int*>(ctx->err.p), cycles);
  return cuda_check(ctx, cudaGetLastError(), "rijk_selftest_wait_timeout launch");
}

RIJK_API int rijk_selftest_alloc_failure(rijk_ctx* ctx, long after) {
  if (!ctx) return RIJK_ERR_ARG;
  ctx->fail_alloc_after = after < 0 ? -1 : after;
  return RIJK_OK;
}
