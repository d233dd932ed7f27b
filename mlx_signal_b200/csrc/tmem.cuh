// Tensor Memory (TMEM) helpers for sm_100a kernels: allocation, ordering fences and the 32x32b
// loads of a warp's lane quadrant.
//
// Each SM has 256 KB of TMEM: 128 lanes x 512 columns of 32-bit cells. A CTA allocates a power
// of two of columns (>= 32) spanning all 128 lanes; warp w of the CTA reads the 32 lanes
// 32 (w mod 4) .. 32 (w mod 4) + 31. One warp allocates and the same warp frees, before the CTA
// exits.
#pragma once

#include <stdint.h>

namespace b2s {
namespace tm {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Warp-collective: allocate `ncols` columns (power of two >= 32); the base address lands in
// *slot (shared memory).
__device__ __forceinline__ void alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_addr(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

// Warp-collective: free the columns allocated by alloc().
__device__ __forceinline__ void dealloc(uint32_t base, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols)
               : "memory");
}

// Ordering of tcgen05 operations around a thread barrier.
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Address of column `col` in the lane quadrant of warp `warp`.
__device__ __forceinline__ uint32_t lane_addr(uint32_t base, int warp, int col) {
  return base + (uint32_t(32 * (warp & 3)) << 16) + uint32_t(col);
}

// Warp-collective load of 32 consecutive columns of the thread's lane.
__device__ __forceinline__ void ld32(uint32_t a, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, "
      "%29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(a));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tm
}  // namespace b2s
