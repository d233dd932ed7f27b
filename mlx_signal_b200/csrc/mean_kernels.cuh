// Fused segment-mean spectral kernels: welch (|X|^2), csd (conj(X) Y) and coherence
// (Pxx, Pyy, Pxy) for power-of-two nfft, real float32 input.
//
// Reference behaviour replaced: _stft_metal.rfft_power_mean (src/mlx_signal_processing/
// _stft_metal.py:530-557, kernel source _SUM_SRC :458-505), csd_mean / coherence_mean
// (:739-746, _PAIR_SUM_SRC :620-667) and their host-side group reduction (_reduce_groups
// :443-455). Differences by design:
//  * welch packs TWO real segments of a row into one complex FFT (z = x_s + i x_{s+1}); the sum
//    of both power spectra is (|Z_k|^2 + |Z_{L-k}|^2)/2, so no per-segment untangle is needed and
//    the mirror combination happens once, in the final reduction;
//  * csd/coherence pack x and y of the same segment (z = x_s + i y_s); the per-bin products
//    Z_k Z_{L-k} and |Z_k|^2 carry all three cross/auto spectra;
//  * the flattened (row, segment) space is split evenly over all resident teams, each team
//    accumulating in registers and writing one partial row per row it touches; the final
//    reduction sums partials in a fixed order in FP64 (deterministic, blocked summation).
#pragma once

#include "fft_core.cuh"
#include "spectral_params.h"
#include "team_util.cuh"

namespace b2s {

template <int LOG_L, int LOG_E>
struct MeanCfg {
  using PL = Plan<LOG_L, LOG_E>;
  static constexpr int TEAMS = PL::P >= 64 ? 1 : 128 / PL::P;
  static constexpr int THREADS = TEAMS * PL::P;
  static constexpr int SCRATCH = PL::P >= 64 ? PL::P / 32 : 1;   // float4 per team
  static constexpr int WIN = (PL::L + 3) & ~3;                     // window floats (16 B multiple)
  static constexpr size_t SMEM = size_t(TEAMS) * SCRATCH * 16      // team scratch
                                 + size_t(WIN) * 4                 // window
                                 + size_t(PL::TW) * 8              // twiddle tables
                                 + size_t(TEAMS) * PL::BUF * 8;    // exchange buffers
};

struct MeanSmem {
  float4* scratch;
  float* win;
  float2* tw;
  float2* buf;
};

template <class CFG>
__device__ __forceinline__ MeanSmem mean_smem_setup(const float* win, int nperseg) {
  using PL = typename CFG::PL;
  extern __shared__ float4 smem[];
  MeanSmem s;
  s.scratch = smem;
  s.win = reinterpret_cast<float*>(smem + CFG::TEAMS * CFG::SCRATCH);
  s.tw = reinterpret_cast<float2*>(s.win + CFG::WIN);
  s.buf = s.tw + PL::TW;
  for (int i = threadIdx.x; i < PL::L; i += blockDim.x) s.win[i] = i < nperseg ? win[i] : 0.f;
  build_twiddles<PL>(s.tw, threadIdx.x, blockDim.x);
  __syncthreads();
  return s;
}

// Load two real segments into (re, im) in the pass-0 element pattern (zero beyond nperseg or
// when the second segment is absent).
template <class PL>
__device__ __forceinline__ void load_pair(float2 (&v)[PL::E], const float* __restrict__ a,
                                          const float* __restrict__ b, bool has_b, int t,
                                          int nperseg) {
  if (nperseg == PL::L) {
    static_for<0, PL::E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const int n = slot_elem<PL, e>(t);
      v[e].x = __ldg(a + n);
      v[e].y = has_b ? __ldg(b + n) : 0.f;
    });
  } else {
    static_for<0, PL::E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const int n = slot_elem<PL, e>(t);
      const bool ok = n < nperseg;
      v[e].x = ok ? __ldg(a + n) : 0.f;
      v[e].y = (ok && has_b) ? __ldg(b + n) : 0.f;
    });
  }
}

// Welch: partial[r][slot][k] = sum over the team's segments of |Z_k|^2, z = x_s + i x_{s+1}.
template <int LOG_L, int LOG_E, int DET>
__global__ void __launch_bounds__(MeanCfg<LOG_L, LOG_E>::THREADS)
    k_welch_mean(MeanParams pr) {
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
  float acc[E];
#pragma unroll
  for (int e = 0; e < E; ++e) acc[e] = 0.f;
  while (g < gend) {
    const int64_t r = g / pr.nseg;
    const int s0 = int(g - r * pr.nseg);
    const int64_t lim = int64_t(s0) + (gend - g);
    const int s1 = int(lim < pr.nseg ? lim : int64_t(pr.nseg));
    const float* xr = pr.x + r * pr.ld_x;
    for (int s = s0; s < s1; s += 2) {
      const bool two = s + 1 < s1;
      const float* xa = xr + int64_t(s) * pr.hop;
      float2 v[E];
      load_pair<PL>(v, xa, xa + pr.hop, two, t, pr.nperseg);
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
    float* dst = pr.partial + (r * pr.cmax + slot) * int64_t(L);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      dst[t + e * P] = acc[e];
      acc[e] = 0.f;
    }
    g += s1 - s0;
  }
}

// Partial-slot layout of the cross kernel: Q[cross_q_floats(L)] (|Z_k|^2, padded to an even
// count so the complex section stays 8-byte aligned) then C[L/2+1] complex.
__host__ __device__ constexpr int cross_q_floats(int L) { return L + (L & 1); }
__host__ __device__ constexpr int cross_slot_floats(int L) {
  return cross_q_floats(L) + 2 * (L / 2 + 1);
}

// csd / coherence: z = x_s + i y_s. Accumulates Q_k = sum |Z_k|^2 (all k) and
// C_k = sum Z_k Z_{L-k} for k in [0, L/2] (C is symmetric in k <-> L-k).
template <int LOG_L, int LOG_E, int DET>
__global__ void __launch_bounds__(MeanCfg<LOG_L, LOG_E>::THREADS)
    k_cross_mean(MeanParams pr) {
  using CFG = MeanCfg<LOG_L, LOG_E>;
  using PL = typename CFG::PL;
  constexpr int L = PL::L, E = PL::E, P = PL::P, EH = E / 2 + 1;
  const MeanSmem sm = mean_smem_setup<CFG>(pr.win, pr.nperseg);
  const int team = threadIdx.x / P, t = threadIdx.x - team * P;
  const unsigned mask = team_mask<P>();
  float4* scratch = sm.scratch + team * CFG::SCRATCH;
  float2* buf = sm.buf + team * PL::BUF;
  const int64_t tau = int64_t(blockIdx.x) * CFG::TEAMS + team;
  int64_t g = tau * pr.G;
  const int64_t gend = min(g + pr.G, pr.total);
  float q[E];
  float2 c[EH];
#pragma unroll
  for (int e = 0; e < E; ++e) q[e] = 0.f;
#pragma unroll
  for (int e = 0; e < EH; ++e) c[e] = make_float2(0.f, 0.f);
  while (g < gend) {
    const int64_t r = g / pr.nseg;
    const int s0 = int(g - r * pr.nseg);
    const int64_t lim = int64_t(s0) + (gend - g);
    const int s1 = int(lim < pr.nseg ? lim : int64_t(pr.nseg));
    const float* xr = pr.x + r * pr.ld_x;
    const float* yr = pr.y + r * pr.ld_y;
    for (int s = s0; s < s1; ++s) {
      float2 v[E];
      load_pair<PL>(v, xr + int64_t(s) * pr.hop, yr + int64_t(s) * pr.hop, true, t, pr.nperseg);
      detrend_window<PL, DET>(v, sm.win, t, pr.nperseg, scratch, mask);
      team_pass0<PL>(v);
      team_passes<PL>(v, buf, sm.tw, t, mask);
      // mirror exchange through the (now free) buffer
#pragma unroll
      for (int e = 0; e < E; ++e) {
        q[e] = fmaf(v[e].x, v[e].x, q[e]);
        q[e] = fmaf(v[e].y, v[e].y, q[e]);
        buf[PL::pad(t + e * P)] = v[e];
      }
      team_sync<P>(mask);
#pragma unroll
      for (int e = 0; e < EH; ++e) {
        if (e < E / 2 || t == 0) {
          const int k = t + e * P;
          const float2 m = buf[PL::pad((L - k) & (L - 1))];
          c[e].x = fmaf(v[e].x, m.x, fmaf(-v[e].y, m.y, c[e].x));
          c[e].y = fmaf(v[e].x, m.y, fmaf(v[e].y, m.x, c[e].y));
        }
      }
      team_sync<P>(mask);
    }
    const int64_t slot = tau - first_team(r, pr.nseg, pr.G);
    float* dst = pr.partial + (r * pr.cmax + slot) * int64_t(cross_slot_floats(L));
    float2* dstc = reinterpret_cast<float2*>(dst + cross_q_floats(L));
#pragma unroll
    for (int e = 0; e < E; ++e) {
      dst[t + e * P] = q[e];
      q[e] = 0.f;
    }
#pragma unroll
    for (int e = 0; e < EH; ++e) {
      if (e < E / 2 || t == 0) dstc[t + e * P] = c[e];
      c[e] = make_float2(0.f, 0.f);
    }
    g += s1 - s0;
  }
}

// Final reduction over partial slots (fixed order, FP64), mirror combination, one-sided
// doubling and 1/nseg. mode: 0 welch (float out), 1 csd (complex out), 2 coherence (float out).
struct ReduceParams {
  const float* partial;
  int64_t rows;
  int L;
  int nout;          // output bins per row
  int onesided;      // apply one-sided doubling (welch/csd)
  int nseg;
  int64_t G;
  int cmax;
  int64_t nteams;
  int mode;
  float* out;
};

}  // namespace b2s
