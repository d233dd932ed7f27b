// Fused spectral kernels for complex input (complex64 rows), power-of-two nfft <= 4096: welch
// (two-sided mean |X|^2) and per-frame spectra (stft complex / spectrogram power).
//
// Reference behaviour replaced: the composed path the reference takes for complex input
// (src/mlx_signal_processing/spectral.py:290-298 switch to a two-sided spectrum; :127-147 frame
// gather, detrend, window and mx.fft.fft of each complex segment; `_stft_metal.eligible` admits
// real input only). Here each complex segment is one team FFT: the engine's (re, im) lanes carry
// the segment's real and imaginary parts, detrend_window removes the mean (and line) of each part
// separately — scipy's detrend of complex data — and multiplies both by the window. No pair
// packing, so no mirror untangle: bin k of the transform is bin k of the segment.
#pragma once

#include "fft_core.cuh"
#include "frame_kernels.cuh"
#include "mean_kernels.cuh"
#include "spectral_params.h"
#include "team_util.cuh"

namespace b2s {

// Sample i of a complex row under the virtual boundary extension / zero padding (the complex
// counterpart of ext_sample: even / odd / constant act on both parts).
__device__ __forceinline__ float2 ext_sample_c(const float2* __restrict__ row, int64_t n, int ext,
                                               int mode, int64_t i) {
  const int64_t j = i - ext;
  if (j >= 0 && j < n) return __ldg(row + j);
  if (mode == kExtNone || mode == kExtZeros) return make_float2(0.f, 0.f);
  if (j < 0) {
    if (j < -int64_t(ext)) return make_float2(0.f, 0.f);
    if (mode == kExtConst) return __ldg(row);
    const float2 m = __ldg(row - j);
    if (mode == kExtEven) return m;
    const float2 a = __ldg(row);
    return make_float2(2.f * a.x - m.x, 2.f * a.y - m.y);
  }
  if (j >= n + ext) return make_float2(0.f, 0.f);
  if (mode == kExtConst) return __ldg(row + n - 1);
  const float2 m = __ldg(row + 2 * (n - 1) - j);
  if (mode == kExtEven) return m;
  const float2 a = __ldg(row + n - 1);
  return make_float2(2.f * a.x - m.x, 2.f * a.y - m.y);
}

// Welch of complex rows: partial[r][slot][k] = sum over the team's segments of |X_k|^2,
// k in [0, L) (slot stride cross_q_floats(L)); pr.x is interleaved complex64, pr.ld_x in complex
// elements.
template <int LOG_L, int LOG_E, int DET>
__global__ void __launch_bounds__(MeanCfg<LOG_L, LOG_E>::THREADS, MeanCfg<LOG_L, LOG_E>::MIN_CTAS)
    k_welch_cplx(MeanParams pr) {
  using CFG = MeanCfg<LOG_L, LOG_E>;
  using PL = typename CFG::PL;
  constexpr int L = PL::L, E = PL::E, P = PL::P;
  const MeanSmem sm = mean_smem_setup<CFG>(pr.win, pr.nperseg);
  const int team = threadIdx.x / P, t = threadIdx.x - team * P;
  const unsigned mask = team_mask<P>();
  float4* scratch = sm.scratch + team * CFG::SCRATCH;
  float2* buf = sm.buf + team * PL::BUF;
  const int64_t tau = int64_t(blockIdx.x) * CFG::TEAMS + team;
  int64_t g = tau * pr.G;
  const int64_t gend = min(g + pr.G, pr.total);
  const float2* x = reinterpret_cast<const float2*>(pr.x);
  float acc[E];
#pragma unroll
  for (int e = 0; e < E; ++e) acc[e] = 0.f;
  while (g < gend) {
    const int64_t r = g / pr.nseg;
    const int s0 = int(g - r * pr.nseg);
    const int64_t lim = int64_t(s0) + (gend - g);
    const int s1 = int(lim < pr.nseg ? lim : int64_t(pr.nseg));
    const float2* xr = x + r * pr.ld_x;
    for (int s = s0; s < s1; ++s) {
      const float2* xs = xr + int64_t(s) * pr.hop;
      float2 v[E];
      static_for<0, E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        const int n = slot_elem<PL, e>(t);
        v[e] = n < pr.nperseg ? __ldg(xs + n) : make_float2(0.f, 0.f);
      });
      detrend_window<PL, DET>(v, sm.win, t, pr.nperseg, scratch, mask);
      team_pass0<PL>(v);
      team_passes<PL>(v, buf, sm.tw, t, mask);
#pragma unroll
      for (int e = 0; e < E; ++e) {
        acc[e] = fmaf(v[e].x, v[e].x, acc[e]);
        acc[e] = fmaf(v[e].y, v[e].y, acc[e]);
      }
    }
    const int64_t slot = tau - first_team(r, pr.nseg, pr.G);
    float* dst = pr.partial + (r * pr.cmax + slot) * int64_t(cross_q_floats(L));
#pragma unroll
    for (int e = 0; e < E; ++e) {
      dst[t + e * P] = acc[e];
      acc[e] = 0.f;
    }
    g += s1 - s0;
  }
}

// Per-frame spectra of complex rows: out (rows, nseg, L) complex64 (POWER = 0) or |X|^2 float32
// (POWER = 1), two-sided; frames read through the virtual boundary extension / padding.
template <int LOG_L, int LOG_E, int DET, int POWER>
__global__ void __launch_bounds__(MeanCfg<LOG_L, LOG_E>::THREADS, MeanCfg<LOG_L, LOG_E>::MIN_CTAS)
    k_frames_cplx(FrameParams pr) {
  using CFG = MeanCfg<LOG_L, LOG_E>;
  using PL = typename CFG::PL;
  constexpr int E = PL::E, P = PL::P;
  const MeanSmem sm = mean_smem_setup<CFG>(pr.win, pr.nperseg);
  const int team = threadIdx.x / P, t = threadIdx.x - team * P;
  const unsigned mask = team_mask<P>();
  float4* scratch = sm.scratch + team * CFG::SCRATCH;
  float2* buf = sm.buf + team * PL::BUF;
  const int64_t nt = int64_t(gridDim.x) * CFG::TEAMS;
  const int64_t tau = int64_t(blockIdx.x) * CFG::TEAMS + team;
  const int64_t G = (pr.total + nt - 1) / nt;
  const int64_t gend = min((tau + 1) * G, pr.total);
  const float2* x = reinterpret_cast<const float2*>(pr.x);
  for (int64_t f = tau * G; f < gend; ++f) {
    const int64_t r = f / pr.nseg;
    const int s = int(f - r * pr.nseg);
    const float2* xr = x + r * pr.ld_x;
    const int64_t sa = int64_t(s) * pr.hop;
    float2 v[E];
    if (sa >= pr.ext && sa + pr.nperseg <= pr.ext + pr.n) {
      static_for<0, E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        const int n = slot_elem<PL, e>(t);
        v[e] = n < pr.nperseg ? __ldg(xr + (sa - pr.ext) + n) : make_float2(0.f, 0.f);
      });
    } else {
      static_for<0, E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        const int n = slot_elem<PL, e>(t);
        v[e] = n < pr.nperseg ? ext_sample_c(xr, pr.n, pr.ext, pr.ext_mode, sa + n)
                              : make_float2(0.f, 0.f);
      });
    }
    detrend_window<PL, DET>(v, sm.win, t, pr.nperseg, scratch, mask);
    team_pass0<PL>(v);
    team_passes<PL>(v, buf, sm.tw, t, mask);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int k = t + e * P;
      if constexpr (POWER) {
        pr.out[f * pr.nbins + k] = fmaf(v[e].x, v[e].x, v[e].y * v[e].y);
      } else {
        reinterpret_cast<float2*>(pr.out)[f * pr.nbins + k] = v[e];
      }
    }
  }
}

// csd of complex rows x, y (interleaved complex64, ld in complex elements): partial[r][slot][k] =
// sum over the team's segments of conj(X_k) Y_k, k in [0, L) (slot stride 2L floats). Each
// segment is two team transforms; X is parked in shared memory in the thread's own bins.
template <int LOG_L, int LOG_E, int DET>
__global__ void __launch_bounds__(MeanCfg<LOG_L, LOG_E>::THREADS)
    k_csd_cplx(MeanParams pr) {
  using CFG = MeanCfg<LOG_L, LOG_E>;
  using PL = typename CFG::PL;
  constexpr int L = PL::L, E = PL::E, P = PL::P;
  const MeanSmem sm = mean_smem_setup<CFG>(pr.win, pr.nperseg);
  const int team = threadIdx.x / P, t = threadIdx.x - team * P;
  const unsigned mask = team_mask<P>();
  float4* scratch = sm.scratch + team * CFG::SCRATCH;
  float2* buf = sm.buf + team * PL::BUF;
  // per-team parking area for X after the exchange buffers
  float2* xs_park = sm.buf + CFG::TEAMS * PL::BUF + team * L;
  const int64_t tau = int64_t(blockIdx.x) * CFG::TEAMS + team;
  int64_t g = tau * pr.G;
  const int64_t gend = min(g + pr.G, pr.total);
  const float2* x = reinterpret_cast<const float2*>(pr.x);
  const float2* y = reinterpret_cast<const float2*>(pr.y);
  float2 acc[E];
#pragma unroll
  for (int e = 0; e < E; ++e) acc[e] = make_float2(0.f, 0.f);
  auto transform = [&](const float2* seg, float2 (&v)[E]) {
    static_for<0, E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const int n = slot_elem<PL, e>(t);
      v[e] = n < pr.nperseg ? __ldg(seg + n) : make_float2(0.f, 0.f);
    });
    detrend_window<PL, DET>(v, sm.win, t, pr.nperseg, scratch, mask);
    team_pass0<PL>(v);
    team_passes<PL>(v, buf, sm.tw, t, mask);
  };
  while (g < gend) {
    const int64_t r = g / pr.nseg;
    const int s0 = int(g - r * pr.nseg);
    const int64_t lim = int64_t(s0) + (gend - g);
    const int s1 = int(lim < pr.nseg ? lim : int64_t(pr.nseg));
    for (int s = s0; s < s1; ++s) {
      float2 v[E];
      transform(x + r * pr.ld_x + int64_t(s) * pr.hop, v);
#pragma unroll
      for (int e = 0; e < E; ++e) xs_park[t + e * P] = v[e];
      transform(y + r * pr.ld_y + int64_t(s) * pr.hop, v);
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const float2 a = xs_park[t + e * P];  // X_k; accumulate conj(X_k) Y_k
        acc[e].x = fmaf(a.x, v[e].x, fmaf(a.y, v[e].y, acc[e].x));
        acc[e].y = fmaf(a.x, v[e].y, fmaf(-a.y, v[e].x, acc[e].y));
      }
    }
    const int64_t slot = tau - first_team(r, pr.nseg, pr.G);
    float2* dst = reinterpret_cast<float2*>(pr.partial + (r * pr.cmax + slot) * int64_t(2 * L));
#pragma unroll
    for (int e = 0; e < E; ++e) {
      dst[t + e * P] = acc[e];
      acc[e] = make_float2(0.f, 0.f);
    }
    g += s1 - s0;
  }
}

}  // namespace b2s
