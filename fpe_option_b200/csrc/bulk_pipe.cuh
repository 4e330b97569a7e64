// Bulk global->shared copies completed on an mbarrier (sm_100a PTX), with
// bounded waits.  Only local (this CTA's) shared memory is ever a
// destination and there is no cluster multicast.
#pragma once

#include <stdint.h>

namespace fpe {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes barrier initialisation visible to the asynchronous proxy.
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders the generic-proxy accesses visible to this thread (its own and, after
// a CTA barrier, those of the other threads) before its later asynchronous
// copies: shared-memory destinations that were read or written normally, and
// global sources (factor blocks) written with ordinary stores.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// dst (shared, 16-byte aligned) <- src (global, 16-byte aligned), bytes a
// multiple of 16; completion is counted on bar.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// The same three operations on shared-window addresses held as 32-bit values.
__device__ __forceinline__ void mbar_arrive_expect_tx_u32(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive_u32(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void bulk_g2s_u32(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      "  .reg .pred p;\n"
      "  mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "  selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Non-blocking test of the phase (never suspends the thread).
__device__ __forceinline__ bool mbar_test_wait(unsigned long long* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      "  .reg .pred p;\n"
      "  mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "  selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Limits below this many cycles poll with test_wait: try_wait may suspend the
// thread for a system-dependent time, longer than such a limit.
constexpr long long kShortWaitCycles = 1LL << 20;

// Wait for the phase of `bar` with the given parity to complete; gives up
// after `limit` SM clock cycles and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, uint32_t parity, long long limit) {
  const long long t0 = clock64();
  if (limit < kShortWaitCycles) {
    while (!mbar_test_wait(bar, parity)) {
      if (clock64() - t0 > limit) return false;
    }
    return true;
  }
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit) return false;
  }
  return true;
}

// Asynchronous copy of one 4-, 8- or 16-byte element (global -> this CTA's
// shared memory, both naturally aligned); completes at cp_async_wait_all.
template <int B>
__device__ __forceinline__ void cp_async_elem(void* dst, const void* src) {
  static_assert(B == 4 || B == 8 || B == 16, "cp.async element size");
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(B) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// About one second at the B200's 1.965 GHz SM clock.
constexpr long long kBulkWaitLimit = 2000000000LL;

}  // namespace fpe
