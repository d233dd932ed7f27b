// Overlap-save FFT convolution of real rows with one shared real filter, fully fused.
//
// Reference behaviour replaced: the fused block convolution of oaconvolve
// (src/mlx_signal_processing/_stft_metal.py:900-1058: forward block FFT + spectrum multiply into a
// device scratch, then an inverse-FFT kernel) followed by the gather overlap-add
// (src/mlx_signal_processing/_ola_metal.py:20-78), routed from convolution.py:288-306 for real
// float32 input and a filter of at most 1025 taps.
// Design here:
//  * overlap-save instead of overlap-add: block b of a row produces the STEP = L - (taps-1)
//    full-convolution outputs j in [jb, jb + STEP) from the L input samples starting at
//    jb - (taps-1); the circular convolution's first taps-1 outputs are the wrapped ones and are
//    dropped. Blocks never share an output, so there is no scratch and no overlap-add pass;
//  * two blocks share one complex FFT, z = a + i b: since h is real, ifft(FFT(z) H) carries a*h in
//    its real part and b*h in its imaginary part, so no untangle step is needed;
//  * the inverse is the forward engine applied to conj(Z H / L): after the forward passes thread t
//    holds bins t + e P, which is exactly the element set pass 0 of the next transform wants from
//    it, so the spectrum multiply and the switch to the inverse happen in registers (a
//    compile-time register permutation), with no exchange in between;
//  * every team computes the filter spectrum H once (same engine) and keeps its own bins
//    H[t + e P] / L in registers for all of its blocks;
//  * the output window [j0, j0 + nout) of the full convolution ('full', 'same' or 'valid') is
//    written directly.
#pragma once

#include "fft_core.cuh"
#include "spectral_params.h"
#include "team_util.cuh"

namespace b2s {

struct ConvParams {
  const float* x;   // rows x n1, row stride ld_x
  const float* h;   // n2 taps
  float* out;       // rows x nout, row stride ld_out
  int64_t ld_x, ld_out, rows, n1, j0, nout, nblk, total;
  int n2, step;
};

template <int LOG_L>
struct ConvCfg {
  using PL = Plan<LOG_L, 4>;  // 16 points per thread
  static constexpr int TEAMS = PL::P >= 64 ? 1 : 128 / PL::P;
  static constexpr int THREADS = TEAMS * PL::P;
  // <= 128 registers per thread: v (32), the filter bins (32) and addressing
  static constexpr int MIN_CTAS = 65536 / (THREADS * 128);
  static constexpr size_t SMEM = size_t(PL::TW) * 8 + size_t(TEAMS) * PL::BUF * 8;
};

// Input element of register slot `s` in the pass-0 layout, as a multiple of P beyond t:
// slot s = b R0 + bitrev(q) holds element t + P (b + B0 q).
template <class PL, int S>
constexpr int slot_index() {
  constexpr int R0 = PL::radix(0), B0 = PL::E / R0;
  return S / R0 + B0 * bitrev(S % R0, ilog2(R0));
}

// Load block g (row r, block b) of the convolution into one component of v: samples
// x[r, s0 + i], i in [0, L), zero outside [0, n1).
template <class PL, bool IM>
__device__ __forceinline__ void conv_load(float2 (&v)[PL::E], const ConvParams& p, int64_t g,
                                          int t) {
  constexpr int L = PL::L, P = PL::P, E = PL::E;
  if (g >= p.total) {
#pragma unroll
    for (int e = 0; e < E; ++e) (IM ? v[e].y : v[e].x) = 0.f;
    return;
  }
  const int64_t r = g / p.nblk, b = g - r * p.nblk;
  const int64_t s0 = p.j0 + b * p.step - (p.n2 - 1);
  const float* row = p.x + r * p.ld_x;
  if (s0 >= 0 && s0 + L <= p.n1) {
    static_for<0, E>([&](auto sc) {
      constexpr int s = decltype(sc)::value;
      const float val = __ldg(row + s0 + t + P * slot_index<PL, s>());
      if constexpr (IM) v[s].y = val; else v[s].x = val;
    });
  } else {
    static_for<0, E>([&](auto sc) {
      constexpr int s = decltype(sc)::value;
      const int64_t i = s0 + t + P * slot_index<PL, s>();
      const float val = (i >= 0 && i < p.n1) ? __ldg(row + i) : 0.f;
      if constexpr (IM) v[s].y = val; else v[s].x = val;
    });
  }
}

// Store block g's outputs from one component of v (bin/sample m = t + e P after the inverse).
template <class PL, bool IM>
__device__ __forceinline__ void conv_store(const float2 (&v)[PL::E], const ConvParams& p,
                                           int64_t g, int t) {
  constexpr int P = PL::P, E = PL::E;
  if (g >= p.total) return;
  const int64_t r = g / p.nblk, b = g - r * p.nblk;
  float* orow = p.out + r * p.ld_out;
  const int64_t base = b * p.step - (p.n2 - 1);  // output offset of sample m is base + m
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int m = t + e * P;
    const int64_t o = base + m;
    if (m >= p.n2 - 1 && o < p.nout) orow[o] = IM ? -v[e].y : v[e].x;
  }
}

template <int LOG_L>
__global__ void __launch_bounds__(ConvCfg<LOG_L>::THREADS, ConvCfg<LOG_L>::MIN_CTAS)
    k_conv_ols(ConvParams p) {
  using CFG = ConvCfg<LOG_L>;
  using PL = typename CFG::PL;
  constexpr int L = PL::L, E = PL::E, P = PL::P;
  extern __shared__ float4 smem_conv[];
  float2* tw = reinterpret_cast<float2*>(smem_conv);
  build_twiddles<PL>(tw, threadIdx.x, blockDim.x);
  __syncthreads();
  const int team = threadIdx.x / P, t = threadIdx.x - team * P;
  const unsigned mask = team_mask<P>();
  float2* buf = tw + PL::TW + team * PL::BUF;

  // filter spectrum: this thread's bins H[t + e P] / L
  float2 hb[E];
  {
    static_for<0, E>([&](auto sc) {
      constexpr int s = decltype(sc)::value;
      const int i = t + P * slot_index<PL, s>();
      hb[s] = make_float2(i < p.n2 ? __ldg(p.h + i) : 0.f, 0.f);
    });
    team_pass0<PL>(hb);
    team_passes<PL>(hb, buf, tw, t, mask);
    constexpr float inv = 1.0f / float(L);
#pragma unroll
    for (int e = 0; e < E; ++e) hb[e] = make_float2(hb[e].x * inv, hb[e].y * inv);
  }

  const int64_t nteams = int64_t(gridDim.x) * CFG::TEAMS;
  const int64_t tau = int64_t(blockIdx.x) * CFG::TEAMS + team;
  const int64_t npairs = (p.total + 1) / 2;
  const int64_t G = (npairs + nteams - 1) / nteams;
  const int64_t pend = min((tau + 1) * G, npairs);
  for (int64_t pr = tau * G; pr < pend; ++pr) {
    const int64_t ga = 2 * pr, gb = ga + 1;
    float2 v[E];
    conv_load<PL, false>(v, p, ga, t);
    conv_load<PL, true>(v, p, gb, t);
    team_pass0<PL>(v);
    team_passes<PL>(v, buf, tw, t, mask);
    // conj(Z H / L), moved into the pass-0 layout of the inverse transform
    float2 u[E];
    static_for<0, E>([&](auto sc) {
      constexpr int s = decltype(sc)::value;
      constexpr int m = slot_index<PL, s>();
      const float2 y = cmul(v[m], hb[m]);
      u[s] = make_float2(y.x, -y.y);
    });
    team_pass0<PL>(u);
    team_passes<PL>(u, buf, tw, t, mask);
    conv_store<PL, false>(u, p, ga, t);
    conv_store<PL, true>(u, p, gb, t);
  }
}

}  // namespace b2s
