// Shared helpers of liblmb200: error reporting, exact FP64 arithmetic,
// bounded waits, TMA bulk-copy and mbarrier wrappers (sm_100a inline PTX).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/lmb200.h"

namespace lmb {

// ---- error reporting (per host thread) -----------------------------------
void set_error(const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what, const char *file, int line);

#define LMB_CUDA(call)                                                   \
  do {                                                                   \
    cudaError_t _e = (call);                                             \
    if (_e != cudaSuccess) return ::lmb::cuda_fail(_e, #call, __FILE__, __LINE__); \
  } while (0)

#define LMB_REQUIRE(cond, ...)            \
  do {                                    \
    if (!(cond)) {                        \
      ::lmb::set_error(__VA_ARGS__);      \
      return LMB_ERR_INVALID;             \
    }                                     \
  } while (0)

// ---- device error flag codes ---------------------------------------------
enum DevErr : int { DEV_OK = 0, DEV_TIMEOUT_TMA = 1, DEV_BAD_ALIGN = 2, DEV_BAD_QUEUE = 3 };

// ---- exact FP64 (round to nearest, never contracted into FMA) -------------
// The reference CPU build has no fused multiply-add (x86-64 SSE2, -O3 without
// -march), so every product and sum is rounded separately.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double dsqrt(double a) { return __dsqrt_rn(a); }

// C's (int) cast of a double as x86-64 executes it (cvttsd2si): truncation
// toward zero, and INT_MIN for NaN or a result outside the int range.
__device__ __forceinline__ int x86_trunc_i32(double v) {
  return (v > -2147483649.0 && v < 2147483648.0) ? __double2int_rz(v)
                                                  : (int)0x80000000;
}

// ---- timers -----------------------------------------------------------------
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ---- mbarrier + bulk copy (TMA, non-tensor, no multicast) -------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for phase `parity` of `bar`, giving up after `limit_ns` of global time.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t i = 0;; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255u) == 255u && global_ns() - t0 > limit_ns) return false;
  }
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// L2 cache policies: the DB is streamed once (evict first); the occupancy
// words are gathered on every pass and should stay resident (evict last).
__device__ __forceinline__ uint64_t l2_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ unsigned long long ld_nc_hint(const unsigned long long *p,
                                                         uint64_t pol) {
  unsigned long long v;
  asm volatile("ld.global.nc.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(v) : "l"(p), "l"(pol));
  return v;
}

// 1-D bulk copy global -> shared with an L2 cache policy.
__device__ __forceinline__ void bulk_g2s_hint(void *dst_smem, const void *src_gmem,
                                              uint32_t bytes, uint64_t *bar, uint64_t pol) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1], %2, [%3], %4;" ::"r"(smem_u32(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
      : "memory");
}

// Prefetch `bytes` (multiple of 16, 16-byte aligned) of global memory into L2.
__device__ __forceinline__ void bulk_prefetch_l2(const void *src_gmem, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src_gmem), "r"(bytes)
               : "memory");
}

// 1-D bulk copy global -> shared of `bytes` (multiple of 16, both addresses
// 16-byte aligned), completing on `bar` via complete_tx.
__device__ __forceinline__ void bulk_g2s(void *dst_smem, const void *src_gmem, uint32_t bytes,
                                         uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace lmb
