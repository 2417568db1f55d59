// fsl_bulk.cuh -- bulk asynchronous copies from global to shared memory
// (cp.async.bulk, the TMA engine's untiled form) completed on a shared
// mbarrier, with waits that give up after a bounded number of polls.
// Included by fsl_fft.cu.
//
// Rules the callers keep: source, destination and size are multiples of
// 16 bytes; one thread registers the expected bytes (mbar_arrive_tx) before
// any copy of the phase is issued; the destination is not touched by
// ordinary stores until the phase has completed.
#pragma once

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// makes an initialised barrier visible to the copy engine
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// one arrival that also expects `bytes` more bytes in the current phase
__device__ __forceinline__ void mbar_arrive_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_test(unsigned long long* bar, unsigned phase) {
  unsigned ok;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

// Polls for the completion of phase `phase` at most `limit` times; false
// when it gave up.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned phase, long limit) {
  for (long i = 0; i < limit; ++i)
    if (mbar_test(bar, phase)) return true;
  return false;
}

// polls before a bulk load counts as lost (a copy of a few tens of KB lands
// within microseconds)
constexpr long kBulkPolls = 1L << 22;

// Waits for the block's bulk load on bar (phase 0).  If the wait gives up,
// the internal-check bit is set and the block waits once more, again
// bounded, for the copy still in flight, so that it does not leave with its
// shared memory being written; what it computes then is flagged.
__device__ __forceinline__ void bulk_wait(unsigned long long* bar, int* err) {
  if (mbar_wait(bar, 0, kBulkPolls)) return;
  if (threadIdx.x == 0) set_err(err, 4);  // FSL_ERRBIT_GRID
  mbar_wait(bar, 0, kBulkPolls);
}
