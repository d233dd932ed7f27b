// Per-frame spectral kernels: stft (complex frames), spectrogram psd (power frames) and
// per-frame cross spectra conj(X) Y (used for median averaging), power-of-two nfft.
//
// Reference behaviour replaced: _stft_metal.rfft_frames (src/mlx_signal_processing/
// _stft_metal.py:192-220, kernel _SRC :104-147 with _LOAD_* :33-61, _OUT_* :63-78) and
// csd_frames / coherence_frames (:412-419, _PAIR_SRC :318-351), plus the materialised boundary
// extension and end padding of spectral._spectral_helper (spectral.py:275-288).
// Differences by design:
//  * two consecutive frames of a row share one complex FFT (z = x_s + i x_{s+1}); the frames are
//    separated after the transform: X_s = (Z_k + conj Z_{L-k})/2, X_{s+1} = (Z_k - conj Z_{L-k})/2i;
//  * boundary extension (zeros/even/odd/constant) and the zero tail of `padded` are virtual:
//    frames touching them map indices on the fly, interior frames load directly;
//  * output rows are frame-major (rows, nseg, nbins) so every warp store is contiguous; the host
//    returns the (freq, time) view scipy returns.
#pragma once

#include "fft_core.cuh"
#include "mean_kernels.cuh"
#include "spectral_params.h"
#include "team_util.cuh"

namespace b2s {

enum : int { kFrameStft = 0, kFramePower = 1, kFrameCross = 2 };
enum : int { kExtNone = 0, kExtZeros = 1, kExtEven = 2, kExtOdd = 3, kExtConst = 4 };

// Sample i of the extended/padded signal (extension `ext` per side, original length n).
__device__ __forceinline__ float ext_sample(const float* __restrict__ row, int64_t n, int ext,
                                            int mode, int64_t i) {
  const int64_t j = i - ext;
  if (j >= 0 && j < n) return __ldg(row + j);
  if (mode == kExtNone || mode == kExtZeros) return 0.f;
  if (j < 0) {
    if (j < -int64_t(ext)) return 0.f;
    if (mode == kExtConst) return __ldg(row);
    const float m = __ldg(row - j);
    return mode == kExtEven ? m : 2.f * __ldg(row) - m;
  }
  if (j >= n + ext) return 0.f;  // zero padding tail
  if (mode == kExtConst) return __ldg(row + n - 1);
  const float m = __ldg(row + 2 * (n - 1) - j);
  return mode == kExtEven ? m : 2.f * __ldg(row + n - 1) - m;
}

// Load frame(s) starting at extended positions sa (and sb = sa + hop when has_b) into (re, im).
template <class PL>
__device__ __forceinline__ void load_frames(float2 (&v)[PL::E], const float* __restrict__ row,
                                            int64_t n, int ext, int mode, int64_t sa, int64_t sb,
                                            bool has_b, int t, int nperseg) {
  const int64_t hi = sa > sb ? sa : sb;
  const bool interior = sa >= ext && hi + nperseg <= ext + n;
  if (interior) {
    load_pair<PL>(v, row + (sa - ext), row + (sb - ext), has_b, t, nperseg);
  } else {
    static_for<0, PL::E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const int ne = slot_elem<PL, e>(t);
      const bool ok = ne < nperseg;
      v[e].x = ok ? ext_sample(row, n, ext, mode, sa + ne) : 0.f;
      v[e].y = (ok && has_b) ? ext_sample(row, n, ext, mode, sb + ne) : 0.f;
    });
  }
}

// Extra shared memory of the spectral-detrend frame kernels: the low-bin window spectrum
// (2P complex) after the exchange buffers.
template <class CFG>
constexpr size_t frame_spectral_extra() {
  return size_t(2 * CFG::PL::P) * 8;
}

// DET == kDetrendConstantSpectral: the constant detrend as a spectral correction. The two frames
// of a pair share one FFT of z = x_s + i x_{s+1} (or x + i y for the cross kind), so
// FFT(w (z - m)) = FFT(w z) - (m_s + i m_{s+1}) DFT(w): only the low bins where the window's
// spectrum is non-zero (k < n_low, k > L - n_low) are corrected, after the transform.
template <int LOG_L, int LOG_E, int DET, int KIND>
__global__ void __launch_bounds__(MeanCfg<LOG_L, LOG_E>::THREADS, MeanCfg<LOG_L, LOG_E>::MIN_CTAS)
    k_frames(FrameParams pr) {
  using CFG = MeanCfg<LOG_L, LOG_E>;
  using PL = typename CFG::PL;
  constexpr int L = PL::L, E = PL::E, P = PL::P;
  constexpr bool SPEC = DET == kDetrendConstantSpectral;
  const MeanSmem sm = mean_smem_setup<CFG>(pr.win, pr.nperseg);
  float2* wlo = sm.buf + CFG::TEAMS * PL::BUF;
  float2* whi = wlo + P;
  if constexpr (SPEC) {
    load_window_lowbins<P>(wlo, whi, pr.wdft, pr.n_low, threadIdx.x, blockDim.x);
    __syncthreads();
  }
  const int team = threadIdx.x / P, t = threadIdx.x - team * P;
  const unsigned mask = team_mask<P>();
  float4* scratch = sm.scratch + team * CFG::SCRATCH;
  float2* buf = sm.buf + team * PL::BUF;
  const int64_t tau = int64_t(blockIdx.x) * CFG::TEAMS + team;
  // frames per team (G) travels in ext_mode's high bits? no: reuse `total` / grid split below
  const int64_t G = (pr.total + int64_t(gridDim.x) * CFG::TEAMS - 1) / (int64_t(gridDim.x) * CFG::TEAMS);
  const int64_t Ge = KIND == kFrameCross ? G : G + (G & 1);
  int64_t g = tau * Ge;
  const int64_t gend = min(g + Ge, pr.total);
  const bool onesided = pr.nbins != L || L == 1;
  while (g < gend) {
    const int64_t r = g / pr.nseg;
    const int s0 = int(g - r * pr.nseg);
    const int64_t lim = int64_t(s0) + (gend - g);
    const int s1 = int(lim < pr.nseg ? lim : int64_t(pr.nseg));
    const float* xr = pr.x + r * pr.ld_x;
    for (int s = s0; s < s1; s += (KIND == kFrameCross ? 1 : 2)) {
      const bool two = KIND != kFrameCross && s + 1 < s1;
      float2 v[E];
      const int64_t sa = int64_t(s) * pr.hop;
      {  // warm L2 with the samples the next step adds (frames s+2, s+3 / s+1), inside the row
        constexpr int STEP = KIND == kFrameCross ? 1 : 2;
        // this step covers [sa, sa + (STEP-1) hop + nperseg); the next adds STEP hops beyond it
        const int64_t lo = int64_t(sa) - pr.ext + int64_t(STEP - 1) * pr.hop + pr.nperseg;
        const int64_t hi = lo + int64_t(STEP) * pr.hop;
        if (s + 2 * STEP <= s1 && lo >= 0 && hi <= pr.n) {
          for (int64_t o = lo + t * 32; o < hi; o += P * 32) {
            asm volatile("prefetch.global.L2 [%0];" ::"l"(xr + o));
            if constexpr (KIND == kFrameCross)
              asm volatile("prefetch.global.L2 [%0];" ::"l"(pr.y + r * pr.ld_y + o));
          }
        }
      }
      if constexpr (KIND == kFrameCross) {
        const float* yr = pr.y + r * pr.ld_y;
        float2 vy[E];
        load_frames<PL>(v, xr, pr.n, pr.ext, pr.ext_mode, sa, sa, false, t, pr.nperseg);
        load_frames<PL>(vy, yr, pr.n, pr.ext, pr.ext_mode, sa, sa, false, t, pr.nperseg);
#pragma unroll
        for (int e = 0; e < E; ++e) v[e].y = vy[e].x;
      } else {
        load_frames<PL>(v, xr, pr.n, pr.ext, pr.ext_mode, sa, sa + pr.hop, two, t, pr.nperseg);
      }
      float2 m = make_float2(0.f, 0.f);
      if constexpr (SPEC) {
        const float sa = tree_sum<E>([&](auto ec) { return v[decltype(ec)::value].x; });
        const float sb = tree_sum<E>([&](auto ec) { return v[decltype(ec)::value].y; });
        const float4 s4 = team_sum4<P>(make_float4(sa, sb, 0.f, 0.f), scratch, mask);
        const float inv = 1.0f / float(pr.nperseg);
        m = make_float2(s4.x * inv, s4.y * inv);
        detrend_window<PL, kDetrendNone>(v, sm.win, t, pr.nperseg, scratch, mask);
      } else {
        detrend_window<PL, DET>(v, sm.win, t, pr.nperseg, scratch, mask);
      }
      team_pass0<PL>(v);
      team_passes<PL>(v, buf, sm.tw, t, mask);
      if constexpr (SPEC) {
        v[0] = csub(v[0], cmul(m, wlo[t]));
        v[E - 1] = csub(v[E - 1], cmul(m, whi[t]));
      }
#pragma unroll
      for (int e = 0; e < E; ++e) buf[PL::pad(t + e * P)] = v[e];
      team_sync<P>(mask);
      const int64_t fa = r * pr.nseg + s;  // output frame index of segment a
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int k = t + e * P;
        if (k < pr.nbins) {
          const float2 z = v[e];
          const float2 m = buf[PL::pad((L - k) & (L - 1))];
          // a = (z + conj m)/2 ; b = (z - conj m)/(2i) = ((z.y + m.y), -(z.x - m.x)) / 2
          const float2 xa = make_float2(0.5f * (z.x + m.x), 0.5f * (z.y - m.y));
          const float2 xb = make_float2(0.5f * (z.y + m.y), 0.5f * (m.x - z.x));
          if constexpr (KIND == kFrameStft) {
            float2* oa = reinterpret_cast<float2*>(pr.out) + fa * pr.nbins;
            oa[k] = xa;
            if (two) oa[pr.nbins + k] = xb;
          } else if constexpr (KIND == kFramePower) {
            const float f = (onesided && k != 0 && 2 * k != L) ? 2.f : 1.f;
            float* oa = pr.out + fa * pr.nbins;
            oa[k] = f * fmaf(xa.x, xa.x, xa.y * xa.y);
            if (two) oa[pr.nbins + k] = f * fmaf(xb.x, xb.x, xb.y * xb.y);
          } else {
            // conj(X) Y per frame (no one-sided factor: applied after averaging)
            float2* oa = reinterpret_cast<float2*>(pr.out) + fa * pr.nbins;
            oa[k] = make_float2(fmaf(xa.x, xb.x, xa.y * xb.y), fmaf(xa.x, xb.y, -xa.y * xb.x));
          }
        }
      }
      team_sync<P>(mask);
    }
    g += s1 - s0;
  }
}

}  // namespace b2s
