// Column medians over segments: the `average='median'` reduction of welch / csd.
//
// Reference behaviour replaced: spectral.csd's median branch (src/mlx_signal_processing/
// spectral.py:469-477: np.median-style median of the per-segment spectra along the segment axis,
// real and imaginary parts separately, divided by the median bias). Input is the per-frame output
// of the frame kernels, (rows, nseg, ncols) with frame stride ld_frame floats (a complex spectrum
// is passed as its float view: real and imaginary parts are separate columns).
// Design: a CTA stages C columns of one row for all segments into shared memory (coalesced
// C-float runs per segment, stored transposed with an odd column stride), then one warp per
// column finds the exact order statistic(s) by an MSB-first radix select over order-preserving
// 32-bit keys: four 8-bit passes with a shared-memory histogram, each narrowing the key prefix.
// For an even count the upper middle value is the smallest key above the lower one unless the
// lower one repeats (one more counting pass). No sort, no global scratch.
#include "capi_common.h"

namespace b2s {
namespace {

constexpr int kMedWarps = 8;                    // columns per CTA at most
constexpr int kMedSmemFloats = 48 * 1024;       // 192 KB of staged values per CTA

__device__ __forceinline__ unsigned med_key(float f) {
  const unsigned b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float med_val(unsigned k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Key of rank `rank` (0-based) among col[0..n) (one warp).
__device__ unsigned radix_select(const float* col, int n, int rank, unsigned* hist, int lane) {
  unsigned prefix = 0, pmask = 0;
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int i = lane; i < 256; i += 32) hist[i] = 0;
    __syncwarp();
    for (int s = lane; s < n; s += 32) {
      const unsigned k = med_key(col[s]);
      if ((k & pmask) == prefix) atomicAdd(&hist[(k >> shift) & 255u], 1u);
    }
    __syncwarp();
    // lane owns buckets 8*lane .. 8*lane+7: find the bucket holding `rank`
    unsigned loc[8];
    unsigned tot = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      loc[j] = hist[8 * lane + j];
      tot += loc[j];
    }
    unsigned incl = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const unsigned excl = incl - tot;
    const bool mine = unsigned(rank) >= excl && unsigned(rank) < incl;
    const unsigned owner = __ballot_sync(0xffffffffu, mine);
    const int src = __ffs(owner) - 1;
    int bucket = 0;
    unsigned below = 0;
    if (mine) {
      unsigned acc = excl;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (unsigned(rank) >= acc && unsigned(rank) < acc + loc[j]) {
          bucket = 8 * lane + j;
          below = acc;
        }
        acc += loc[j];
      }
    }
    bucket = __shfl_sync(0xffffffffu, bucket, src);
    below = __shfl_sync(0xffffffffu, below, src);
    rank -= int(below);
    prefix |= unsigned(bucket) << shift;
    pmask |= 255u << shift;
    __syncwarp();
  }
  return prefix;
}

__global__ void __launch_bounds__(32 * kMedWarps)
    k_median_cols(const float* __restrict__ in, int64_t rows, int nseg, int ncols,
                  int64_t ld_frame, int cols_per_cta, float scale, float* __restrict__ out) {
  extern __shared__ float med_smem[];
  __shared__ unsigned hist_all[kMedWarps][256];
  const int chunks = (ncols + cols_per_cta - 1) / cols_per_cta;
  const int64_t r = blockIdx.x / chunks;
  const int c0 = int(blockIdx.x - r * chunks) * cols_per_cta;
  const int cw = min(cols_per_cta, ncols - c0);
  const int stride = nseg | 1;  // odd column stride in shared memory
  const float* base = in + r * int64_t(nseg) * ld_frame + c0;
  // stage: element (s, c) -> med_smem[c * stride + s]
  const int tot = nseg * cw;
  for (int e = threadIdx.x; e < tot; e += blockDim.x) {
    const int s = e / cw, c = e - s * cw;
    med_smem[c * stride + s] = __ldg(base + int64_t(s) * ld_frame + c);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp >= cw) return;
  const float* col = med_smem + warp * stride;
  unsigned* hist = hist_all[warp];
  const int lo = (nseg - 1) / 2;
  const unsigned k1 = radix_select(col, nseg, lo, hist, lane);
  float med = med_val(k1);
  if ((nseg & 1) == 0) {
    // upper middle value: k1 again if it repeats past rank lo, else the smallest key above k1
    unsigned cnt = 0, mn = 0xffffffffu;
    for (int s = lane; s < nseg; s += 32) {
      const unsigned k = med_key(col[s]);
      cnt += k <= k1 ? 1u : 0u;
      if (k > k1) mn = min(mn, k);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
      mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    }
    const float hi = cnt >= unsigned(lo + 2) ? med : med_val(mn);
    med = 0.5f * (med + hi);
  }
  if (lane == 0) out[r * ncols + c0 + warp] = med * scale;
}

}  // namespace
}  // namespace b2s

extern "C" {

int sp_median_frames_f32(const float* in, int64_t rows, int nseg, int ncols, int64_t ld_frame,
                         float scale, float* out, void* stream) {
  using namespace b2s;
  if (rows < 0 || nseg < 1 || ncols < 1 || ld_frame < ncols) {
    set_error("invalid median arguments (rows=%lld nseg=%d ncols=%d ld_frame=%lld)",
              (long long)rows, nseg, ncols, (long long)ld_frame);
    return SP_ERR_ARG;
  }
  const int stride = nseg | 1;
  int cpc = kMedSmemFloats / stride;
  if (cpc > kMedWarps) cpc = kMedWarps;
  if (cpc < 1) {
    set_error("median over %d segments exceeds the staged maximum of %d", nseg,
              kMedSmemFloats - 1);
    return SP_ERR_UNSUPPORTED;
  }
  if (rows == 0) return SP_OK;
  if (!in || !out) {
    set_error("null pointer");
    return SP_ERR_ARG;
  }
  const size_t smem = size_t(cpc) * stride * sizeof(float);
  if (smem > 48 * 1024) {
    B2S_CHECK_CUDA(cudaFuncSetAttribute(k_median_cols, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        int(smem)),
                   "median smem attribute");
  }
  const int64_t chunks = (ncols + cpc - 1) / cpc;
  k_median_cols<<<dim3(unsigned(rows * chunks)), 32 * kMedWarps, smem,
                  static_cast<cudaStream_t>(stream)>>>(in, rows, nseg, ncols, ld_frame, cpc, scale,
                                                       out);
  B2S_CHECK_CUDA(cudaGetLastError(), "median kernel launch");
  return SP_OK;
}

}
