// bulk.cuh — 1-D bulk asynchronous copies (the TMA engine's cp.async.bulk,
// no tensor map, no multicast) from global into shared memory, completed on
// a CTA-local mbarrier.
//
// A slab of consecutive floats is staged so that its 16-byte-aligned interior
// goes by one bulk copy and the ragged head and tail (fewer than 4 floats
// each) by plain loads: the shared-memory copy of element 0 sits at
// `phase(src)` in its buffer, which gives the interior the same 16-byte
// alignment on both sides.  Waits are bounded: a copy that has not completed
// after kBulkSpinLimit polls raises the caller's timeout flag and the waiting
// CTA gives up its tile (after a second bounded wait for the copies in flight).
#pragma once

#include <cstdint>

namespace snapb {

constexpr long kBulkSpinLimit = 1L << 26;

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// order this thread's (and, after a CTA barrier, the CTA's) earlier
// shared-memory accesses before later async-proxy writes to the same memory
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// bytes (a multiple of 16) from src (16-byte aligned) to dst (16-byte aligned)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// wait for the phase of the given parity; false (and *flag = 1) if it has not
// completed after kBulkSpinLimit polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int* flag) {
  const unsigned a = smem_addr(bar);
  for (long k = 0; k < kBulkSpinLimit; ++k) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  atomicExch(flag, 1);
  return false;
}

// float index of element 0 of a slab starting at src inside its shared buffer
__device__ __forceinline__ int bulk_phase(const float* src) {
  return (int)((reinterpret_cast<uintptr_t>(src) >> 2) & 3);
}

// the aligned interior of a slab of n floats at src: elements [head, head + body)
struct BulkSplit {
  int ph, head;
  int64_t body;
};
__device__ __forceinline__ BulkSplit bulk_split(const float* src, int64_t n) {
  BulkSplit s;
  s.ph = bulk_phase(src);
  s.head = (4 - s.ph) & 3;  // elements before the first 16-byte boundary
  s.body = n > s.head ? ((n - s.head) & ~(int64_t)3) : 0;
  return s;
}

// Stage n floats from src into dst[bulk_phase(src) ...] (dst 16-byte aligned,
// room for n + 3 floats): the aligned interior by one bulk copy issued by the
// issuing thread (after its mbar_arrive_expect_tx of the interiors' bytes), the
// head and tail by the plain loads of threads 0 .. 7 (threads 0 .. 7 and the
// issuer call this; the plain stores are visible after the next CTA barrier).
__device__ __forceinline__ void bulk_stage_slab(float* dst, const float* src, int64_t n,
                                                uint64_t* bar, bool issuer) {
  const BulkSplit s = bulk_split(src, n);
  const int64_t tail0 = s.head + s.body;  // first element after the interior
  const int t = threadIdx.x;
  if (t < 4) {
    if (t < s.head && t < n) dst[s.ph + t] = src[t];
  } else if (t < 8) {
    const int64_t e = tail0 + (t - 4);
    if (e < n) dst[s.ph + e] = src[e];
  }
  if (s.body > 0 && issuer)
    bulk_g2s(dst + s.ph + s.head, src + s.head, (unsigned)(s.body * 4), bar);
}

}  // namespace snapb
