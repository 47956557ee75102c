// Shared device and host helpers of libp6cuda: status handling, the Philox
// counter-based generator, fixed-point conversions, and the bulk-copy /
// mbarrier primitives used to stage static tables into shared memory.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "p6cuda.h"

namespace p6 {

// ---------------------------------------------------------------------------
// Host-side error reporting.  Every C-ABI entry point returns a p6_status and
// leaves a message retrievable with p6_last_error() on the calling thread.
// ---------------------------------------------------------------------------
p6_status set_error(p6_status code, const std::string &msg);
p6_status cuda_error(cudaError_t e, const char *what);
void clear_error();

#define P6_CUDA(call)                                                          \
  do {                                                                         \
    cudaError_t _e = (call);                                                   \
    if (_e != cudaSuccess) return ::p6::cuda_error(_e, #call);                 \
  } while (0)

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC 2011): a counter-based generator, so every (key, counter)
// pair is an independent draw and no state is carried between kernels.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint32_t mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
#endif
}

__host__ __device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const uint32_t m0 = 0xD2511F53u, m1 = 0xCD9E8D57u;
    uint32_t hi0 = mulhi32(m0, c.x), lo0 = m0 * c.x;
    uint32_t hi1 = mulhi32(m1, c.z), lo1 = m1 * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

// [0, 1) with 24 random bits, exactly representable.
__device__ __forceinline__ float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }
// (0, 1], for logarithms.
__device__ __forceinline__ float u01_open(uint32_t x) { return (float)((x >> 8) + 1u) * (1.0f / 16777216.0f); }

// Two standard normal deviates from two uniform words (Box-Muller).
__device__ __forceinline__ float2 gauss2(uint32_t a, uint32_t b) {
  float r = sqrtf(-2.0f * __logf(u01_open(a)));
  float s, c;
  __sincosf(6.28318530717958647f * u01(b), &s, &c);
  return make_float2(r * c, r * s);
}

// ---------------------------------------------------------------------------
// Shared-memory staging with the bulk-copy engine (cp.async.bulk), completion
// tracked on an mbarrier.  Every wait is bounded: a wait that runs out records
// an error code and returns false instead of spinning forever.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// 1-D bulk copy global -> shared; dst, src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
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

// Bounded wait on phase `parity`.  Returns false when the limit runs out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Device error word: the first failing site writes its code; the host reads it.
__device__ __forceinline__ void raise_flag(int *flag, int code) {
  if (flag) atomicCAS(flag, 0, code);
}

enum DeviceError : int {
  DEV_OK = 0,
  DEV_STAGE_TIMEOUT = 1,   // a bulk copy into shared memory did not complete within the limit
  DEV_CAPACITY = 2,        // a table exceeded what the kernel was launched for
};

}  // namespace p6
