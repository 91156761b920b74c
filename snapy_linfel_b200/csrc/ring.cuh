// ring.cuh — per-thread asynchronous prefetch rings in shared memory.
//
// A sequential sweep along a column (one thread per column) reads a few
// values per layer and does little work with them; waiting one memory latency
// per layer dominates it.  These helpers fetch the values of layers ahead with
// cp.async (4- and 8-byte copies, one commit group per layer) into a ring of
// slots in dynamic shared memory laid out [slot][element][thread], so the
// threads of a warp touch consecutive words.  A slot is refilled only after
// the values read from it have been consumed by dependent arithmetic.
#pragma once

namespace snapb {

__device__ __forceinline__ void cp_async_bytes8(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_bytes4(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
// wait until at most n of this thread's most recent groups are in flight
template <int n>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(n) : "memory");
}
__device__ __forceinline__ void cp_async_elem(void* smem, const double* g) { cp_async_bytes8(smem, g); }
__device__ __forceinline__ void cp_async_elem(void* smem, const float* g) { cp_async_bytes4(smem, g); }
__device__ __forceinline__ double ring_elem(const double* slot, const double*) { return *slot; }
__device__ __forceinline__ double ring_elem(const double* slot, const float*) {
  return (double)*reinterpret_cast<const float*>(slot);
}
// the element in the stored precision
__device__ __forceinline__ double ring_stored(const double* slot, const double*) { return *slot; }
__device__ __forceinline__ float ring_stored(const double* slot, const float*) {
  return *reinterpret_cast<const float*>(slot);
}

// Slot-element address of this thread in a ring of E elements per slot.
struct Ring {
  double* base;
  int E, nt, lane;
  __device__ __forceinline__ double* at(int slot, int e) const {
    return base + ((size_t)(slot * E + e) * nt + lane);
  }
};

}  // namespace snapb
