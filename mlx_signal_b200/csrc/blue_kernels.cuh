// Fused spectral kernels for a DFT length N that is not a power of two (2 < N <= 2048), by
// Bluestein's chirp-z identity on the power-of-two team engine.
//
// Reference behaviour replaced: the composed path of spectral._fft_frames for shapes outside the
// Metal kernels (src/mlx_signal_processing/spectral.py:127-147: frame gather, detrend, window,
// mx.fft.rfft of length nfft), used for every non-power-of-two nfft.
// Algorithm (Bluestein 1970; nk = (n^2 + k^2 - (k - n)^2) / 2):
//   X_k = d_k (a (*) b)_k,  a_n = x_n w_n e^{-i pi n^2/N} (n < N),  b_m = e^{+i pi m^2/N}
//   (m in (-N, N), wrapped mod M),  d_k = e^{-i pi k^2/N},
// with (*) the circular convolution of length M = 2^LOG_M >= 2N - 1. The convolution runs as in
// the overlap-save convolution kernel: forward FFT_M, multiply by B = FFT_M(b)/M held in
// registers (bins t + e P), conjugate, forward FFT_M again; V = conj(a (*) b), so
// X_k = d_k conj(V_k) and |X_k| = |V_k| (the power kinds skip the output chirp).
// Two real segments share one transform (z = x_s + i x_{s+1}), as in the power-of-two kernels.
// Chirp phases are exact: n^2 is reduced mod 2N in integers and sincospi runs in FP64; the chirp
// tables are built per CTA, B per team with the same engine.
#pragma once

#include "fft_core.cuh"
#include "frame_kernels.cuh"
#include "mean_kernels.cuh"
#include "spectral_params.h"
#include "team_util.cuh"

namespace b2s {

template <int LOG_M>
struct BlueCfg {
  using PL = Plan<LOG_M, 4>;  // 16 points per thread
  static constexpr int M = PL::L;
  static constexpr int NMAX = M / 2;  // N <= (M + 1) / 2
  static constexpr int TEAMS = PL::P >= 64 ? 1 : 128 / PL::P;
  static constexpr int THREADS = TEAMS * PL::P;
  static constexpr int SCRATCH = PL::P >= 64 ? PL::P / 32 : 1;  // float4 per team
  static constexpr size_t SMEM = size_t(TEAMS) * SCRATCH * 16 + size_t(PL::TW) * 8 +
                                 size_t(TEAMS) * PL::BUF * 8 + size_t(2 * NMAX) * 8;
};

struct BlueSmem {
  float4* scratch;
  float2* tw;
  float2* buf;
  float2* cin;   // win[n] e^{-i pi n^2/N}, n < N (zero beyond nperseg)
  float2* cout;  // e^{-i pi k^2/N}, k < N (frame kernels)
};

// e^{s i pi m^2 / N}, exact reduction of m^2 mod 2N
__device__ __forceinline__ float2 chirp(int64_t m, int N, double sgn) {
  const int64_t r = (m * m) % (2 * int64_t(N));
  double s, c;
  sincospi(sgn * double(r) / double(N), &s, &c);
  return make_float2(float(c), float(s));
}

template <class CFG>
__device__ __forceinline__ BlueSmem blue_smem_setup(const float* win, int nperseg, int N,
                                                    bool want_out) {
  using PL = typename CFG::PL;
  extern __shared__ float4 smem_blue[];
  BlueSmem s;
  s.scratch = smem_blue;
  s.tw = reinterpret_cast<float2*>(smem_blue + CFG::TEAMS * CFG::SCRATCH);
  s.buf = s.tw + PL::TW;
  s.cin = s.buf + CFG::TEAMS * PL::BUF;
  s.cout = s.cin + CFG::NMAX;
  build_twiddles<PL>(s.tw, threadIdx.x, blockDim.x);
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    const float w = n < nperseg ? win[n] : 0.f;
    const float2 ch = chirp(n, N, -1.0);
    s.cin[n] = make_float2(w * ch.x, w * ch.y);
    if (want_out) s.cout[n] = ch;
  }
  __syncthreads();
  return s;
}

// This thread's bins of B = FFT_M(b) / M (bin t + e P in bh[e]).
template <class PL>
__device__ __forceinline__ void blue_filter(float2 (&bh)[PL::E], int N, float2* buf,
                                            const float2* tw, int t, unsigned mask) {
  constexpr int M = PL::L;
  static_for<0, PL::E>([&](auto sc) {
    constexpr int s = decltype(sc)::value;
    const int i = slot_elem<PL, s>(t);
    bh[s] = i < N ? chirp(i, N, 1.0)
                  : (i > M - N ? chirp(M - i, N, 1.0) : make_float2(0.f, 0.f));
  });
  team_pass0<PL>(bh);
  team_passes<PL>(bh, buf, tw, t, mask);
  constexpr float inv = 1.0f / float(M);
#pragma unroll
  for (int e = 0; e < PL::E; ++e) bh[e] = make_float2(bh[e].x * inv, bh[e].y * inv);
}

// Detrend (scipy semantics over the nperseg samples of each packed segment) and multiply by the
// chirped window; v holds (x_s, x_{s+1}) in the pass-0 element pattern, zero beyond nperseg.
template <class PL, int DET>
__device__ __forceinline__ void blue_premultiply(float2 (&v)[PL::E], const float2* cin,
                                                 int nperseg, int t, float4* scratch,
                                                 unsigned mask) {
  constexpr int E = PL::E;
  float ma = 0.f, mb = 0.f, ka = 0.f, kb = 0.f;
  const float c = 0.5f * float(nperseg - 1);
  if constexpr (DET != kDetrendNone) {
    const float sa = tree_sum<E>([&](auto ec) { return v[decltype(ec)::value].x; });
    const float sb = tree_sum<E>([&](auto ec) { return v[decltype(ec)::value].y; });
    float ta = 0.f, tb = 0.f;
    if constexpr (DET == kDetrendLinear) {
      ta = tree_sum<E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        const int n = slot_elem<PL, e>(t);
        return n < nperseg ? (float(n) - c) * v[e].x : 0.f;
      });
      tb = tree_sum<E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        const int n = slot_elem<PL, e>(t);
        return n < nperseg ? (float(n) - c) * v[e].y : 0.f;
      });
    }
    const float4 s = team_sum4<PL::P>(make_float4(sa, sb, ta, tb), scratch, mask);
    const float inv = 1.0f / float(nperseg);
    ma = s.x * inv;
    mb = s.y * inv;
    if constexpr (DET == kDetrendLinear) {
      const double Nd = double(nperseg);
      const double denom = Nd * (Nd * Nd - 1.0) / 12.0;
      ka = denom > 0.0 ? float(double(s.z) / denom) : 0.f;
      kb = denom > 0.0 ? float(double(s.w) / denom) : 0.f;
    }
  }
  static_for<0, E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    const int n = slot_elem<PL, e>(t);
    if (n < nperseg) {
      const float d = float(n) - c;
      const float2 z = make_float2(v[e].x - ma - ka * d, v[e].y - mb - kb * d);
      v[e] = cmul(z, cin[n]);
    } else {
      v[e] = make_float2(0.f, 0.f);
    }
  });
}

// The chirp-z core: on entry v holds a (pass-0 pattern), on exit v[e] = V at index t + e P,
// V = conj(a (*) b).
template <class PL>
__device__ __forceinline__ void blue_core(float2 (&v)[PL::E], const float2 (&bh)[PL::E],
                                          float2* buf, const float2* tw, int t, unsigned mask) {
  team_pass0<PL>(v);
  team_passes<PL>(v, buf, tw, t, mask);
  float2 u[PL::E];
  static_for<0, PL::E>([&](auto sc) {
    constexpr int s = decltype(sc)::value;
    constexpr int R0 = PL::radix(0), B0 = PL::E / R0;
    constexpr int m = s / R0 + B0 * bitrev(s % R0, ilog2(R0));
    const float2 y = cmul(v[m], bh[m]);
    u[s] = make_float2(y.x, -y.y);
  });
  team_pass0<PL>(u);
  team_passes<PL>(u, buf, tw, t, mask);
#pragma unroll
  for (int e = 0; e < PL::E; ++e) v[e] = u[e];
}

// Welch partials for non-power-of-two nfft = pr.nfft: partial[r][slot][k] = sum |Z_k|^2 +
// |Z_{N-k}|^2 over the team's segment pairs, k in [0, N/2] (the slot layout of k_welch_mean).
template <int LOG_M, int DET>
__global__ void __launch_bounds__(BlueCfg<LOG_M>::THREADS) k_blue_welch(MeanParams pr) {
  using CFG = BlueCfg<LOG_M>;
  using PL = typename CFG::PL;
  constexpr int E = PL::E, P = PL::P;
  const int N = pr.nfft;
  const BlueSmem sm = blue_smem_setup<CFG>(pr.win, pr.nperseg, N, false);
  const int team = threadIdx.x / P, t = threadIdx.x - team * P;
  const unsigned mask = team_mask<P>();
  float4* scratch = sm.scratch + team * CFG::SCRATCH;
  float2* buf = sm.buf + team * PL::BUF;
  float2 bh[E];
  blue_filter<PL>(bh, N, buf, sm.tw, t, mask);
  const int64_t tau = int64_t(blockIdx.x) * CFG::TEAMS + team;
  int64_t g = tau * pr.G;
  const int64_t gend = min(g + pr.G, pr.total);
  float acc[E / 2];  // bins k = t + e P < N <= M/2
#pragma unroll
  for (int e = 0; e < E / 2; ++e) acc[e] = 0.f;
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
      static_for<0, E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        const int n = slot_elem<PL, e>(t);
        const bool ok = n < pr.nperseg;
        v[e].x = ok ? __ldg(xa + n) : 0.f;
        v[e].y = (ok && two) ? __ldg(xa + pr.hop + n) : 0.f;
      });
      blue_premultiply<PL, DET>(v, sm.cin, pr.nperseg, t, scratch, mask);
      blue_core<PL>(v, bh, buf, sm.tw, t, mask);
      // bins k < N <= M/2 live in registers e < E/2 (k = t + e P)
#pragma unroll
      for (int e = 0; e < E / 2; ++e) {
        acc[e] = fmaf(v[e].x, v[e].x, acc[e]);
        acc[e] = fmaf(v[e].y, v[e].y, acc[e]);
      }
    }
    // mirror-combined partials over the N-periodic spectrum
    const int64_t slot = tau - first_team(r, pr.nseg, pr.G);
    float* dst = pr.partial + (r * pr.cmax + slot) * int64_t(welch_slot_floats(N));
    float* sq = reinterpret_cast<float*>(buf);
    team_sync<P>(mask);
#pragma unroll
    for (int e = 0; e < E / 2; ++e) {
      sq[t + e * P] = acc[e];
      acc[e] = 0.f;
    }
    team_sync<P>(mask);
    for (int k = t; k <= N / 2; k += P) dst[k] = sq[k] + sq[k == 0 ? 0 : N - k];
    team_sync<P>(mask);
    g += s1 - s0;
  }
}

// Per-frame spectra (stft complex / spectrogram power) for non-power-of-two nfft = pr.nfft;
// frames read through the virtual boundary extension / padding.
template <int LOG_M, int DET, int KIND>
__global__ void __launch_bounds__(BlueCfg<LOG_M>::THREADS) k_blue_frames(FrameParams pr) {
  using CFG = BlueCfg<LOG_M>;
  using PL = typename CFG::PL;
  constexpr int E = PL::E, P = PL::P;
  const int N = pr.nfft;
  const BlueSmem sm = blue_smem_setup<CFG>(pr.win, pr.nperseg, N, true);
  const int team = threadIdx.x / P, t = threadIdx.x - team * P;
  const unsigned mask = team_mask<P>();
  float4* scratch = sm.scratch + team * CFG::SCRATCH;
  float2* buf = sm.buf + team * PL::BUF;
  float2 bh[E];
  blue_filter<PL>(bh, N, buf, sm.tw, t, mask);
  const int64_t nt = int64_t(gridDim.x) * CFG::TEAMS;
  const int64_t tau = int64_t(blockIdx.x) * CFG::TEAMS + team;
  const int64_t G = (pr.total + nt - 1) / nt;
  const int64_t Ge = G + (G & 1);
  int64_t g = tau * Ge;
  const int64_t gend = min(g + Ge, pr.total);
  const bool onesided = pr.nbins != N;
  while (g < gend) {
    const int64_t r = g / pr.nseg;
    const int s0 = int(g - r * pr.nseg);
    const int64_t lim = int64_t(s0) + (gend - g);
    const int s1 = int(lim < pr.nseg ? lim : int64_t(pr.nseg));
    const float* xr = pr.x + r * pr.ld_x;
    for (int s = s0; s < s1; s += 2) {
      const bool two = s + 1 < s1;
      const int64_t sa = int64_t(s) * pr.hop, sb = sa + pr.hop;
      float2 v[E];
      const int64_t hi = two ? sb : sa;
      if (sa >= pr.ext && hi + pr.nperseg <= pr.ext + pr.n) {
        static_for<0, E>([&](auto ec) {
          constexpr int e = decltype(ec)::value;
          const int n = slot_elem<PL, e>(t);
          const bool ok = n < pr.nperseg;
          v[e].x = ok ? __ldg(xr + (sa - pr.ext) + n) : 0.f;
          v[e].y = (ok && two) ? __ldg(xr + (sb - pr.ext) + n) : 0.f;
        });
      } else {
        static_for<0, E>([&](auto ec) {
          constexpr int e = decltype(ec)::value;
          const int n = slot_elem<PL, e>(t);
          const bool ok = n < pr.nperseg;
          v[e].x = ok ? ext_sample(xr, pr.n, pr.ext, pr.ext_mode, sa + n) : 0.f;
          v[e].y = (ok && two) ? ext_sample(xr, pr.n, pr.ext, pr.ext_mode, sb + n) : 0.f;
        });
      }
      blue_premultiply<PL, DET>(v, sm.cin, pr.nperseg, t, scratch, mask);
      blue_core<PL>(v, bh, buf, sm.tw, t, mask);
      // Z_k = d_k conj(V_k), k < N (registers e < E/2), staged for the mirror read Z_{N-k}
#pragma unroll
      for (int e = 0; e < E / 2; ++e) {
        const int k = t + e * P;
        if (k < N) {
          const float2 d = sm.cout[k];
          v[e] = cmul(d, make_float2(v[e].x, -v[e].y));
          buf[PL::pad(k)] = v[e];
        }
      }
      team_sync<P>(mask);
      const int64_t fa = r * pr.nseg + s;
#pragma unroll
      for (int e = 0; e < E / 2; ++e) {
        const int k = t + e * P;
        if (k < pr.nbins) {
          const float2 z = v[e];
          const float2 m = buf[PL::pad(k == 0 ? 0 : N - k)];
          const float2 xa = make_float2(0.5f * (z.x + m.x), 0.5f * (z.y - m.y));
          const float2 xb = make_float2(0.5f * (z.y + m.y), 0.5f * (m.x - z.x));
          if constexpr (KIND == kFrameStft) {
            float2* oa = reinterpret_cast<float2*>(pr.out) + fa * pr.nbins;
            oa[k] = xa;
            if (two) oa[pr.nbins + k] = xb;
          } else {
            const float f = (onesided && k != 0 && 2 * k != N) ? 2.f : 1.f;
            float* oa = pr.out + fa * pr.nbins;
            oa[k] = f * fmaf(xa.x, xa.x, xa.y * xa.y);
            if (two) oa[pr.nbins + k] = f * fmaf(xb.x, xb.x, xb.y * xb.y);
          }
        }
      }
      team_sync<P>(mask);
    }
    g += s1 - s0;
  }
}

// csd / coherence partials for non-power-of-two nfft = pr.nfft, z = x_s + i y_s per segment: the
// slot layout of k_cross_mean with the N-periodic mirror, Q_k = sum |Z_k|^2 (k < N) and
// C_k = sum Z_k Z_{N-k} (k <= N/2), Z_k = d_k conj(V_k).
template <int LOG_M, int DET>
__global__ void __launch_bounds__(BlueCfg<LOG_M>::THREADS) k_blue_cross(MeanParams pr) {
  using CFG = BlueCfg<LOG_M>;
  using PL = typename CFG::PL;
  constexpr int E = PL::E, P = PL::P;
  const int N = pr.nfft;
  const BlueSmem sm = blue_smem_setup<CFG>(pr.win, pr.nperseg, N, true);
  const int team = threadIdx.x / P, t = threadIdx.x - team * P;
  const unsigned mask = team_mask<P>();
  float4* scratch = sm.scratch + team * CFG::SCRATCH;
  float2* buf = sm.buf + team * PL::BUF;
  float2 bh[E];
  blue_filter<PL>(bh, N, buf, sm.tw, t, mask);
  const int64_t tau = int64_t(blockIdx.x) * CFG::TEAMS + team;
  int64_t g = tau * pr.G;
  const int64_t gend = min(g + pr.G, pr.total);
  float q[E / 2];  // bins k = t + e P < N <= M/2
  float2 c[E / 2];
#pragma unroll
  for (int e = 0; e < E / 2; ++e) {
    q[e] = 0.f;
    c[e] = make_float2(0.f, 0.f);
  }
  while (g < gend) {
    const int64_t r = g / pr.nseg;
    const int s0 = int(g - r * pr.nseg);
    const int64_t lim = int64_t(s0) + (gend - g);
    const int s1 = int(lim < pr.nseg ? lim : int64_t(pr.nseg));
    const float* xr = pr.x + r * pr.ld_x;
    const float* yr = pr.y + r * pr.ld_y;
    for (int s = s0; s < s1; ++s) {
      const float* xs = xr + int64_t(s) * pr.hop;
      const float* ys = yr + int64_t(s) * pr.hop;
      float2 v[E];
      static_for<0, E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        const int n = slot_elem<PL, e>(t);
        const bool ok = n < pr.nperseg;
        v[e].x = ok ? __ldg(xs + n) : 0.f;
        v[e].y = ok ? __ldg(ys + n) : 0.f;
      });
      blue_premultiply<PL, DET>(v, sm.cin, pr.nperseg, t, scratch, mask);
      blue_core<PL>(v, bh, buf, sm.tw, t, mask);
#pragma unroll
      for (int e = 0; e < E / 2; ++e) {
        const int k = t + e * P;
        if (k < N) {
          q[e] = fmaf(v[e].x, v[e].x, fmaf(v[e].y, v[e].y, q[e]));
          v[e] = cmul(sm.cout[k], make_float2(v[e].x, -v[e].y));
          buf[PL::pad(k)] = v[e];
        }
      }
      team_sync<P>(mask);
#pragma unroll
      for (int e = 0; e < E / 2; ++e) {
        const int k = t + e * P;
        if (2 * k <= N) {
          const float2 m = buf[PL::pad(k == 0 ? 0 : N - k)];
          c[e].x = fmaf(v[e].x, m.x, fmaf(-v[e].y, m.y, c[e].x));
          c[e].y = fmaf(v[e].x, m.y, fmaf(v[e].y, m.x, c[e].y));
        }
      }
      team_sync<P>(mask);
    }
    const int64_t slot = tau - first_team(r, pr.nseg, pr.G);
    float* dst = pr.partial + (r * pr.cmax + slot) * int64_t(cross_slot_floats(N));
    float2* dstc = reinterpret_cast<float2*>(dst + cross_q_floats(N));
#pragma unroll
    for (int e = 0; e < E / 2; ++e) {
      const int k = t + e * P;
      if (k < N) dst[k] = q[e];
      if (2 * k <= N) dstc[k] = c[e];
      q[e] = 0.f;
      c[e] = make_float2(0.f, 0.f);
    }
    g += s1 - s0;
  }
}

}  // namespace b2s
