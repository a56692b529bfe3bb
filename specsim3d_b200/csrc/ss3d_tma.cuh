// ss3d_tma.cuh -- bulk tensor copies (TMA) into shared memory and the
// mbarriers that signal their completion, for the column pass that stages
// its tiles with them (k_col_tma in ss3d_fft.cu).
//
// Only plain tile loads of this GPU's own memory are issued: no multicast
// qualifier in any form.  Every wait on an mbarrier is bounded: after
// PIPE_WAIT_LIMIT polls the waiting thread reports failure, and the kernel
// sets an error flag that the host reads after the call instead of hanging.
#pragma once
#include <cuda.h>
#include <cstdint>

namespace ss3d {

constexpr long long PIPE_WAIT_LIMIT = 1LL << 22;   // polls of try_wait (each may suspend briefly)

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// makes the initialised barriers visible to the bulk-copy unit
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// arrival of the issuing thread that also announces the bytes the copies of
// this phase will deliver
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// wait for phase `parity` of bar to complete; false after PIPE_WAIT_LIMIT polls
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (long long i = 0; i < PIPE_WAIT_LIMIT; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// 3D tile load of the box at (c0, c1, c2) of `map` into dst, completing
// its bytes on bar
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
      "[%2];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

// orders this thread's earlier shared-memory accesses before later bulk
// copies that write the same shared memory
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

}  // namespace ss3d
