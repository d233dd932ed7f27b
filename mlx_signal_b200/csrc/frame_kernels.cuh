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
      const int64_t fa = r * pr.nseg + s;  // output frame index of segment a
      // f: the one-sided factor of bin k (power kind only)
      auto emit = [&](int e, float f) {
        const int k = t + e * P;
        const float2 z = v[e];
        const float2 m = buf[PL::pad((L - k) & (L - 1))];
        if constexpr (KIND == kFramePower) {
          // |X_a|^2 = |z + conj m|^2 / 4, |X_b|^2 = |z - conj m|^2 / 4
          const float sc = 0.25f * f;
          const float a1 = z.x + m.x, a2 = z.y - m.y, b1 = z.y + m.y, b2 = m.x - z.x;
          float* oa = pr.out + fa * pr.nbins;
          oa[k] = sc * fmaf(a1, a1, a2 * a2);
          if (two) oa[pr.nbins + k] = sc * fmaf(b1, b1, b2 * b2);
          return;
        }
        // a = (z + conj m)/2 ; b = (z - conj m)/(2i) = ((z.y + m.y), -(z.x - m.x)) / 2
        const float2 xa = make_float2(0.5f * (z.x + m.x), 0.5f * (z.y - m.y));
        const float2 xb = make_float2(0.5f * (z.y + m.y), 0.5f * (m.x - z.x));
        if constexpr (KIND == kFrameStft) {
          float2* oa = reinterpret_cast<float2*>(pr.out) + fa * pr.nbins;
          oa[k] = xa;
          if (two) oa[pr.nbins + k] = xb;
        } else if constexpr (KIND == kFrameCross) {
          // conj(X) Y per frame (no one-sided factor: applied after averaging)
          float2* oa = reinterpret_cast<float2*>(pr.out) + fa * pr.nbins;
          oa[k] = make_float2(fmaf(xa.x, xb.x, xa.y * xb.y), fmaf(xa.x, xb.y, -xa.y * xb.x));
        }
      };
      bool done = false;
      if constexpr (E >= 2) {
        if (pr.nbins == L / 2 + 1) {
          // one-sided: bins k <= L/2 sit in registers e <= E/2 (k = L/2 only at t = 0), their
          // mirrors in registers e >= E/2; bin 0 is its own mirror
#pragma unroll
          for (int e = E / 2; e < E; ++e) buf[PL::pad(t + e * P)] = v[e];
          if (t == 0) buf[0] = v[0];
          team_sync<P>(mask);
          // bins 0 < k < L/2 take the factor 2, DC (t = 0, e = 0) and Nyquist (e = E/2) 1
          emit(0, t == 0 ? 1.f : 2.f);
#pragma unroll
          for (int e = 1; e < E / 2; ++e) emit(e, 2.f);
          if (t == 0) emit(E / 2, 1.f);
          done = true;
        }
      }
      if (!done) {
#pragma unroll
        for (int e = 0; e < E; ++e) buf[PL::pad(t + e * P)] = v[e];
        team_sync<P>(mask);
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int k = t + e * P;
          if (k < pr.nbins) emit(e, (onesided && k != 0 && 2 * k != L) ? 2.f : 1.f);
        }
      }
      team_sync<P>(mask);
    }
    g += s1 - s0;
  }
}

// ------------------------------------------------------------------------------------------
// Per-frame spectra for hop == nperseg/2 == nfft/2 (stft's and the bench spectrogram's case).
// The structure of welch_half_range (mean_kernels.cuh): a frame pair (s, s+1) spans half-blocks
// A | B | C of the extended signal, each half-block is loaded once (C is carried into the next
// pair as its A) and the window multiply is fused into the first radix-2 stage. Differences:
// half-blocks that touch the boundary extension or the zero padding are read through
// ext_sample (virtual extension), and every pair ends in the per-frame untangle and store of
// k_frames instead of a power accumulation. DET: kDetrendNone, kDetrendConstant (time domain,
// from the half-block sums) or kDetrendConstantSpectral (low-bin correction after the FFT).
// ------------------------------------------------------------------------------------------
template <class PL, int KIND, int DET, bool WT>
__device__ __forceinline__ void frames_half_range(const HalfCtx<PL>& c, const FrameParams& pr,
                                                  int64_t r, int s0, int s1) {
  constexpr int L = PL::L, E = PL::E, P = PL::P, H = L / 2, EH = E / 2;
  constexpr int R0 = PL::radix(0), B0 = E / R0;
  const int t = c.t;
  const float* __restrict__ xr = pr.x + r * pr.ld_x;
  const float inv_n = 1.0f / float(L);
  const bool onesided = pr.nbins != L || L == 1;
  float A[EH], B[EH], C[EH];
  bool carry = false;
  float sum_c = 0.f;
  // half-block j of the extended signal: samples j*H + n, n in [0, H)
  auto load_block = [&](float (&dst)[EH], int64_t j) {
    const int64_t p0 = j * H - pr.ext;  // index of the block start in the original row
    if (p0 >= 0 && p0 + H <= pr.n) {
      static_for<0, EH>([&](auto gc) {
        constexpr int gi = decltype(gc)::value;
        dst[gi] = __ldg(xr + p0 + slot_elem<PL, 2 * gi>(t));
      });
    } else {
      static_for<0, EH>([&](auto gc) {
        constexpr int gi = decltype(gc)::value;
        dst[gi] = ext_sample(xr, pr.n, pr.ext, pr.ext_mode, j * H + slot_elem<PL, 2 * gi>(t));
      });
    }
  };
  auto step = [&](int s, auto two_c) {
    const bool TWO = bool(two_c);
    {  // warm L2 with the next pair's two new half-blocks when they lie inside the row
      const int64_t lo = int64_t(s + 3) * H - pr.ext, hi = lo + 2 * H;
      if (s + 3 < s1 && lo >= 0 && hi <= pr.n) {
        for (int o = t * 32; o < 2 * H; o += P * 32)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(xr + lo + o));
      }
    }
    if (!carry) load_block(A, s);
    load_block(B, s + 1);
    if (TWO) {
      load_block(C, s + 2);
    } else {
#pragma unroll
      for (int i = 0; i < EH; ++i) C[i] = 0.f;
    }
    float ma = 0.f, mb = 0.f;
    if constexpr (DET == kDetrendConstant || DET == kDetrendConstantSpectral) {
      float sa = sum_c;
      if (!carry) {
        float sums[1] = {tree_sum<EH>([&](auto gc) { return A[decltype(gc)::value]; })};
        team_sum<P, 1>(sums, c.scratch, c.mask);
        sa = sums[0];
      }
      float sums[2] = {tree_sum<EH>([&](auto gc) { return B[decltype(gc)::value]; }),
                       TWO ? tree_sum<EH>([&](auto gc) { return C[decltype(gc)::value]; })
                           : 0.f};
      team_sum<P, 2>(sums, c.scratch, c.mask);
      ma = (sa + sums[0]) * inv_n;
      mb = TWO ? (sums[0] + sums[1]) * inv_n : 0.f;
      sum_c = sums[1];
    }
    float2 v[E];
    auto fuse = [&](auto gc, float wl, float wh) {
      constexpr int gi = decltype(gc)::value;
      float2 zl = make_float2(A[gi], TWO ? B[gi] : 0.f);
      float2 zh = make_float2(B[gi], C[gi]);
      if constexpr (DET == kDetrendConstant) {
        zl = make_float2(zl.x - ma, TWO ? zl.y - mb : 0.f);
        zh = make_float2(zh.x - ma, TWO ? zh.y - mb : 0.f);
      }
      const float2 a = make_float2(zl.x * wl, zl.y * wl);
      v[2 * gi] = make_float2(fmaf(zh.x, wh, a.x), fmaf(zh.y, wh, a.y));
      v[2 * gi + 1] = make_float2(fmaf(-zh.x, wh, a.x), fmaf(-zh.y, wh, a.y));
    };
    if constexpr (WT) {
      static_for<0, EH / 2>([&](auto pc) {
        constexpr int gp = decltype(pc)::value;
        const float4 w4 = c.wt[gp];
        fuse(std::integral_constant<int, 2 * gp>{}, w4.x, w4.y);
        fuse(std::integral_constant<int, 2 * gp + 1>{}, w4.z, w4.w);
      });
    } else {
      static_for<0, EH>([&](auto gc) {
        constexpr int gi = decltype(gc)::value;
        const int n = slot_elem<PL, 2 * gi>(t);
        fuse(gc, c.win[n], c.win[n + H]);
      });
    }
    static_for<0, B0>([&](auto bc) {
      constexpr int b = decltype(bc)::value;
      dft_dit<R0, b * R0, 2>(v);
    });
    team_passes<PL>(v, c.buf, c.tw, t, c.mask);
    if constexpr (DET == kDetrendConstantSpectral) {
      const float2 m = make_float2(ma, mb);
      v[0] = csub(v[0], cmul(m, c.wlo[t]));
      v[E - 1] = csub(v[E - 1], cmul(m, c.whi[t]));
    }
    const int64_t fa = r * pr.nseg + s;
    // bin k of frames s (a) and s+1 (b) from the packed Z_k and its mirror Z_{L-k}
    // f: the one-sided factor of bin k (power kind only)
    auto emit = [&](int e, float f) {
      const int k = t + e * P;
      const float2 z = v[e];
      const float2 m = c.buf[PL::pad((L - k) & (L - 1))];
      if constexpr (KIND == kFrameStft) {
        const float2 xa = make_float2(0.5f * (z.x + m.x), 0.5f * (z.y - m.y));
        const float2 xb = make_float2(0.5f * (z.y + m.y), 0.5f * (m.x - z.x));
        float2* oa = reinterpret_cast<float2*>(pr.out) + fa * pr.nbins;
        oa[k] = xa;
        if (TWO) oa[pr.nbins + k] = xb;
      } else {
        // |X_a|^2 = |z + conj m|^2 / 4, |X_b|^2 = |z - conj m|^2 / 4
        const float sc = 0.25f * f;
        const float a1 = z.x + m.x, a2 = z.y - m.y, b1 = z.y + m.y, b2 = m.x - z.x;
        float* oa = pr.out + fa * pr.nbins;
        oa[k] = sc * fmaf(a1, a1, a2 * a2);
        if (TWO) oa[pr.nbins + k] = sc * fmaf(b1, b1, b2 * b2);
      }
    };
    if (pr.nbins == L / 2 + 1 && E >= 2) {
      // one-sided: bins k <= L/2 sit in registers e <= E/2 (k = L/2 only at t = 0); their
      // mirrors L - k in registers e >= E/2, and bin 0 is its own mirror
#pragma unroll
      for (int e = E / 2; e < E; ++e) c.buf[PL::pad(t + e * P)] = v[e];
      if (t == 0) c.buf[0] = v[0];
      team_sync<P>(c.mask);
      // bins 0 < k < L/2 take the factor 2, DC (t = 0, e = 0) and Nyquist (e = E/2) 1
      emit(0, t == 0 ? 1.f : 2.f);
#pragma unroll
      for (int e = 1; e < E / 2; ++e) emit(e, 2.f);
      if (t == 0) emit(E / 2, 1.f);
    } else {
#pragma unroll
      for (int e = 0; e < E; ++e) c.buf[PL::pad(t + e * P)] = v[e];
      team_sync<P>(c.mask);
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int k = t + e * P;
        if (k < pr.nbins) emit(e, (onesided && k != 0 && 2 * k != L) ? 2.f : 1.f);
      }
    }
    team_sync<P>(c.mask);
#pragma unroll
    for (int i = 0; i < EH; ++i) A[i] = C[i];
    carry = true;
  };
  int s = s0;
  for (; s + 1 < s1; s += 2) step(s, std::true_type{});
  if (s < s1) step(s, std::false_type{});
}

template <int LOG_L, int LOG_E, int KIND, int DET>
__global__ void __launch_bounds__(MeanCfg<LOG_L, LOG_E>::THREADS, MeanCfg<LOG_L, LOG_E>::MIN_CTAS)
    k_frames_half(FrameParams pr) {
  using CFG = MeanCfg<LOG_L, LOG_E>;
  using PL = typename CFG::PL;
  constexpr int L = PL::L, P = PL::P;
  constexpr bool WT = HalfWinT<PL>::USE;
  extern __shared__ float4 smem[];
  float* win1 = reinterpret_cast<float*>(smem + CFG::TEAMS * CFG::SCRATCH);
  float2* wlo = reinterpret_cast<float2*>(win1 + HalfSmem<CFG>::WINF);
  float2* whi = wlo + P;
  float2* tw = whi + P;
  float2* sbuf = tw + PL::TW;
  if constexpr (WT) {
    build_half_wint<PL>(win1, pr.win, threadIdx.x);
  } else {
    for (int i = threadIdx.x; i < L; i += blockDim.x) win1[i] = pr.win[i];
  }
  if constexpr (DET == kDetrendConstantSpectral)
    load_window_lowbins<P>(wlo, whi, pr.wdft, pr.n_low, threadIdx.x, blockDim.x);
  build_twiddles<PL>(tw, threadIdx.x, blockDim.x);
  __syncthreads();
  const int team = threadIdx.x / P;
  HalfCtx<PL> c;
  c.win = win1;
  c.wt = reinterpret_cast<const float4*>(win1) +
         (threadIdx.x - team * P) * (HalfWinT<PL>::WS / 4);
  c.wlo = wlo;
  c.whi = whi;
  c.tw = tw;
  c.buf = sbuf + team * PL::BUF;
  c.scratch = smem + team * CFG::SCRATCH;
  c.t = threadIdx.x - team * P;
  c.mask = team_mask<P>();
  const int64_t tau = int64_t(blockIdx.x) * CFG::TEAMS + team;
  const int64_t nt = int64_t(gridDim.x) * CFG::TEAMS;
  const int64_t G = (pr.total + nt - 1) / nt;
  const int64_t Ge = G + (G & 1);
  int64_t g = tau * Ge;
  const int64_t gend = min(g + Ge, pr.total);
  while (g < gend) {
    const int64_t r = g / pr.nseg;
    const int s0 = int(g - r * pr.nseg);
    const int64_t lim = int64_t(s0) + (gend - g);
    const int s1 = int(lim < pr.nseg ? lim : int64_t(pr.nseg));
    frames_half_range<PL, KIND, DET, WT>(c, pr, r, s0, s1);
    g += s1 - s0;
  }
}

}  // namespace b2s
