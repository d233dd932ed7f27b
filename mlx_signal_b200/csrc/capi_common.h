// Internal helpers of the C-ABI layer: status codes, thread-local error text, launch-geometry
// caching (occupancy per kernel and device).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <string>
#include <unordered_map>

#include "b200signal.h"

namespace b2s {

void set_error(const char* fmt, ...);

// Status for a CUDA error (records the text).
int cuda_status(cudaError_t e, const char* where);

// Resident CTAs per SM for (kernel, threads, dynamic smem) on the current device; also raises
// the dynamic shared-memory limit of the kernel when needed. Cached per device.
int resident_ctas(const void* kernel, int threads, size_t smem, int* num_sms);

inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

inline int ilog2_exact(int64_t v) {
  if (v <= 0 || (v & (v - 1))) return -1;
  int l = 0;
  while ((int64_t(1) << l) < v) ++l;
  return l;
}

}  // namespace b2s

#define B2S_CHECK_CUDA(expr, where)                          \
  do {                                                       \
    cudaError_t _e = (expr);                                 \
    if (_e != cudaSuccess) return ::b2s::cuda_status(_e, where); \
  } while (0)
