// 1-D bulk copies (cp.async.bulk, the tensor memory accelerator's untiled
// form) from global into shared memory, completing on mbarriers, and the
// bounded waits on them.  Used by the cell kernels to stage particle chunks.
#pragma once

#include <cstdint>

namespace dsmcb {
namespace dev {

__device__ __forceinline__ uint32_t smem_u32(const void* ptr) {
  return (uint32_t)__cvta_generic_to_shared(ptr);
}
__device__ __forceinline__ void mbar_init(unsigned long long* m, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
// Arrives on the barrier and adds `bytes` to the transaction count its phase
// waits for.
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* m, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes)
               : "memory");
}
// Copies `bytes` (a multiple of 16; both addresses 16-byte aligned) and
// reports them on the barrier's transaction count.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         unsigned long long* m) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(m))
      : "memory");
}
// Orders this thread's earlier generic-proxy accesses of shared memory before
// later bulk copies into it.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* m, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(m)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// 4-byte asynchronous copy global -> shared (a gather element); completes at
// cp_async_wait_all().
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(smem_dst)), "l"(gsrc)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}
// Closes this thread's group of asynchronous copies issued since the last
// commit; cp_async_wait_prior() waits for every group but the newest.
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_prior() {
  asm volatile("cp.async.wait_group 1;" ::: "memory");
}

// Waits for an mbarrier phase for at most about a second.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* m, uint32_t parity) {
  if (mbar_try_wait(m, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(m, parity)) {
    if (global_ns() - t0 > 1000000000ull) return false;
  }
  return true;
}

}  // namespace dev
}  // namespace dsmcb
