// Batched 32-point complex DFTs on the 5th-generation tensor cores (tcgen05.mma, kind::f16) at
// FP32-class accuracy.
//
// A DFT of length 32 is a complex 32 x 32 matrix product. With real and imaginary parts
// stacked (k = n for Re z_n, k = 32 + n for Im z_n; output column j < 32 for Re Y_j, 32 + j for
// Im Y_j) a tile of 128 vectors is one real GEMM D[128 x 64] = A[128 x 64] F[64 x 64]:
//   F[n][j] = cos t, F[32+n][j] = sin t, F[n][32+j] = -sin t, F[32+n][32+j] = cos t,
//   t = 2 pi n j / 32 (forward transform Y_j = sum_n z_n exp(-i t)).
// FP16 operands hold 11 bits, so each operand is split into an FP16 head and an FP16 tail
// (v = hi + lo, lo = fp16(v - hi): about 22 bits together) and three products are accumulated
// in FP32: A_hi F_hi + A_hi F_lo + A_lo F_hi (the dropped A_lo F_lo is ~2^-22 relative). The
// three products are one K = 192 chain of twelve K = 16 MMAs over the stacked operands
// [A_hi | A_hi | A_lo] and [F_hi ; F_lo ; F_hi]. Each vector is scaled by a power of two so its
// largest component lies in [2^13, 2^14) before the split (the FP16 range), and the output is
// scaled back.
//
// Per CTA (128 threads, persistent over tiles): F_hi / F_lo are built once in shared memory
// from FP64 sincospi of the exactly reduced phase; for each tile every thread loads its vector,
// splits it and writes its row of A_hi / A_lo (K-major, 128-byte swizzle, the canonical UMMA
// layout); one thread issues the 12 MMAs into a 128-lane x 64-column FP32 accumulator in TMEM and
// commits them to an mbarrier; every warp then reads its 32 lanes (one vector per thread) with
// tcgen05.ld. `reps` > 1 repeats the MMA chain on the same staged operands (each repetition
// overwrites the accumulator), which measures the tensor-core rate of the stage apart from the
// memory traffic; the result is the same for any reps.
//
// The wait for the MMA is bounded: on timeout the CTA records SP_ERR_TIMEOUT in the error word
// (when given), waits once more (bounded) for the chain in flight and frees its TMEM.
//
// This is the radix-32 DFT stage of the framed FFTs (in the reference: the radix-2 threadgroup
// stages of _stft_metal.py:124-144) moved onto the tensor cores; it has no counterpart in the
// reference as such.
#include <cuda_fp16.h>

#include "capi_common.h"
#include "tmem.cuh"

namespace b2s {
namespace {

constexpr int kTcRows = 128;         // vectors per tile (MMA M)
constexpr int kTcK = 64;             // stacked real inputs per vector
constexpr int kTcN = 64;             // stacked real outputs per vector (MMA N)
constexpr uint32_t kTcCols = 64;     // TMEM columns of the FP32 accumulator
constexpr uint32_t kTcSpin = 1u << 24;
constexpr int kA = kTcRows * kTcK * 2;  // bytes of one A operand (16 KB)
constexpr int kB = kTcN * kTcK * 2;     // bytes of one F operand (8 KB)
constexpr size_t kTcSmem = 1024 + 2 * kA + 2 * kB + 16;

struct TcParams {
  const float* z;  // nvec x 32 complex (interleaved re, im)
  float* y;        // nvec x 32 complex
  int64_t nvec;
  int64_t ntiles;
  int reps;
  int* err;        // device error word or nullptr
};

// Byte offset of half-precision element (row, k) in a K-major tile of 128-byte rows with the
// 128-byte swizzle (16-byte chunk index XOR row mod 8; tiles are 1024-byte aligned).
__device__ __forceinline__ uint32_t swz_off(int row, int k) {
  const int chunk = k >> 3;
  return uint32_t(row * 128 + (((chunk ^ (row & 7)) << 4)) + ((k & 7) << 1));
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
  uint64_t d = uint64_t((saddr >> 4) & 0x3FFFu);  // start address (16-byte units)
  d |= uint64_t(1) << 16;                         // leading byte offset (unused when swizzled)
  d |= uint64_t(1024 >> 4) << 32;                 // stride byte offset: next 8-row group
  d |= uint64_t(1) << 46;                         // descriptor version of sm_100
  d |= uint64_t(2) << 61;                         // layout: 128-byte swizzle
  return d;
}

// Instruction descriptor, kind::f16: FP32 accumulate, FP16 A and B, both K-major, N = 64,
// M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (uint32_t(kTcN >> 3) << 17) | (uint32_t(kTcRows >> 4) << 24);

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
          tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          tm::smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity, uint32_t polls) {
  uint32_t done = 0;
  for (uint32_t it = 0; it < polls; ++it) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(tm::smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ uint32_t pack2(__half a, __half b) {
  return uint32_t(__half_as_ushort(a)) | (uint32_t(__half_as_ushort(b)) << 16);
}

__global__ void __launch_bounds__(kTcRows, 1) k_dft32_tc(TcParams p) {
  extern __shared__ __align__(16) unsigned char sraw[];
  const uint32_t pad = (1024u - (tm::smem_addr(sraw) & 1023u)) & 1023u;
  unsigned char* sm = sraw + pad;
  unsigned char* a_hi = sm;
  unsigned char* a_lo = sm + kA;
  unsigned char* f_hi = sm + 2 * kA;
  unsigned char* f_lo = sm + 2 * kA + kB;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + 2 * kA + 2 * kB);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + 2 * kA + 2 * kB + 8);
  const int tid = threadIdx.x, warp = tid >> 5;

  // F_hi / F_lo rows j (output), K-major: element (j, k)
  for (int i = tid; i < kTcN * kTcK; i += blockDim.x) {
    const int j = i / kTcK, k = i - j * kTcK;
    const int n = k & 31, jj = j & 31;
    double s, c;
    sincospi(2.0 * double((n * jj) & 31) / 32.0, &s, &c);
    const double v = (j < 32) ? (k < 32 ? c : s) : (k < 32 ? -s : c);
    const __half h = __double2half(v);
    const __half l = __double2half(v - double(__half2float(h)));
    *reinterpret_cast<__half*>(f_hi + swz_off(j, k)) = h;
    *reinterpret_cast<__half*>(f_lo + swz_off(j, k)) = l;
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tm::smem_addr(bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tm::alloc(tslot, kTcCols);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tm::fence_before_sync();
  __syncthreads();
  tm::fence_after_sync();
  const uint32_t tbase = *tslot;
  const uint32_t tlane = tm::lane_addr(tbase, warp, 0);
  const uint32_t sa_hi = tm::smem_addr(a_hi), sa_lo = tm::smem_addr(a_lo);
  const uint32_t sf_hi = tm::smem_addr(f_hi), sf_lo = tm::smem_addr(f_lo);
  uint32_t phase = 0;
  for (int64_t tile = blockIdx.x; tile < p.ntiles; tile += gridDim.x) {
    const int64_t v = tile * kTcRows + tid;
    float val[kTcK];
    if (v < p.nvec) {
      const float4* src = reinterpret_cast<const float4*>(p.z + v * kTcK);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const float4 f = __ldg(src + q);
        val[2 * q] = f.x;
        val[32 + 2 * q] = f.y;
        val[2 * q + 1] = f.z;
        val[32 + 2 * q + 1] = f.w;
      }
    } else {
#pragma unroll
      for (int k = 0; k < kTcK; ++k) val[k] = 0.f;
    }
    // power-of-two scale: largest |component| into [2^13, 2^14)
    float mx = 0.f;
#pragma unroll
    for (int k = 0; k < kTcK; ++k) mx = fmaxf(mx, fabsf(val[k]));
    int ex = 0;
    (void)frexpf(mx, &ex);
    const int sh = mx > 0.f ? 14 - ex : 0;
    const float sc = ldexpf(1.f, sh), inv = ldexpf(1.f, -sh);
#pragma unroll
    for (int c = 0; c < kTcK / 8; ++c) {
      uint32_t hw[4], lw[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float v0 = val[8 * c + 2 * e] * sc, v1 = val[8 * c + 2 * e + 1] * sc;
        const __half h0 = __float2half_rn(v0), h1 = __float2half_rn(v1);
        hw[e] = pack2(h0, h1);
        lw[e] = pack2(__float2half_rn(v0 - __half2float(h0)),
                      __float2half_rn(v1 - __half2float(h1)));
      }
      const uint32_t off = swz_off(tid, 8 * c);
      *reinterpret_cast<uint4*>(a_hi + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
      *reinterpret_cast<uint4*>(a_lo + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    }
    // the tensor cores read shared memory through the async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tm::fence_before_sync();
    __syncthreads();
    tm::fence_after_sync();
    if (tid == 0) {
      for (int rep = 0; rep < p.reps; ++rep) {
#pragma unroll
        for (int c = 0; c < 12; ++c) {
          const int part = c >> 2, kk = c & 3;  // part 0: hi.hi, 1: hi.lo, 2: lo.hi
          const uint64_t ad = sdesc((part == 2 ? sa_lo : sa_hi) + 32u * kk);
          const uint64_t bd = sdesc((part == 1 ? sf_lo : sf_hi) + 32u * kk);
          mma_f16(tbase, ad, bd, c > 0 ? 1u : 0u);
        }
      }
      mma_commit(bar);
    }
    const bool ok = __syncthreads_and(bar_wait(bar, phase, kTcSpin) ? 1 : 0) != 0;
    if (!ok) {
      if (tid == 0) {
        if (p.err) atomicExch(p.err, SP_ERR_TIMEOUT);
        (void)bar_wait(bar, phase, kTcSpin);  // bounded second wait for the chain in flight
      }
      break;
    }
    phase ^= 1u;
    tm::fence_after_sync();
    float re[32], im[32];
    tm::ld32(tlane, re);
    tm::ld32(tlane + 32, im);
    if (v < p.nvec) {
      float4* dst = reinterpret_cast<float4*>(p.y + v * kTcK);
#pragma unroll
      for (int q = 0; q < 16; ++q)
        dst[q] = make_float4(re[2 * q] * inv, im[2 * q] * inv, re[2 * q + 1] * inv,
                             im[2 * q + 1] * inv);
    }
    // every warp has read the accumulator and the MMAs are done with the operands
    tm::fence_before_sync();
    __syncthreads();
    tm::fence_after_sync();
  }
  tm::fence_before_sync();
  __syncthreads();
  tm::fence_after_sync();
  if (warp == 0) tm::dealloc(tbase, kTcCols);
}

}  // namespace
}  // namespace b2s

extern "C" int sp_dft32_tc_c64(const float* z, float* y, int64_t nvec, int reps, int* err_word,
                               void* stream) {
  using namespace b2s;
  if (!z || !y || nvec < 0 || reps < 1 || reps > 4096 ||
      (reinterpret_cast<uintptr_t>(z) & 15u) || (reinterpret_cast<uintptr_t>(y) & 15u)) {
    set_error("sp_dft32_tc_c64: null or misaligned (16 B) pointer, nvec < 0 or reps outside "
              "[1, 4096]");
    return SP_ERR_ARG;
  }
  if (nvec == 0) return SP_OK;
  int sms = 0;
  const int nb = resident_ctas(reinterpret_cast<const void*>(&k_dft32_tc), kTcRows, kTcSmem, &sms);
  if (nb <= 0) {
    set_error("sp_dft32_tc_c64: no resident CTA");
    return SP_ERR_UNSUPPORTED;
  }
  TcParams p;
  p.z = z;
  p.y = y;
  p.nvec = nvec;
  p.ntiles = cdiv(nvec, kTcRows);
  p.reps = reps;
  p.err = err_word;
  // at most 4 CTAs of 64 TMEM columns share an SM (256 of its 512 columns)
  const int64_t per_sm = nb < 4 ? nb : 4;
  const int64_t grid = p.ntiles < per_sm * sms ? p.ntiles : per_sm * sms;
  k_dft32_tc<<<unsigned(grid), kTcRows, kTcSmem, static_cast<cudaStream_t>(stream)>>>(p);
  B2S_CHECK_CUDA(cudaGetLastError(), "sp_dft32_tc_c64 launch");
  return SP_OK;
}
