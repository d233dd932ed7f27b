// Kernel dispatch tables shared by the split translation units (one TU per kernel family so
// the template instantiations compile in parallel).
#pragma once

#include <cuda_runtime.h>

#include <utility>

#include "blue_kernels.cuh"
#include "cplx_kernels.cuh"
#include "frame_kernels.cuh"
#include "istft_kernels.cuh"
#include "mean_kernels.cuh"

namespace b2s {

// Points per thread for a team FFT of length 2^LOG_L: single-thread FFTs up to 32 points, then
// 16 points per thread (8 at L = 64), except L = 1024, whose 32 x 32 split needs one register
// exchange. Measured on 64 x 2^20: 16 points beat 32 at L = 512, 2048 and 4096 (a quarter of the
// registers, so twice the resident warps), and lose at L = 1024.
template <int LOG_L>
constexpr int team_log_e() {
  return LOG_L <= 5 ? LOG_L : (LOG_L == 6 ? 3 : (LOG_L == 10 ? 5 : 4));
}

// Points per thread of the batched kernels' classes: the single-request team shapes (the 4096
// class runs in its own 256-thread kernel, 16 points per thread).
template <int LOG_L>
constexpr int batch_log_e() {
  return team_log_e<LOG_L>();
}

constexpr int kMaxLogL = 12;
// The real-input segment-mean and per-frame families (welch, csd, coherence, stft,
// spectrogram) also take nfft = 2^13: one 512-thread team per CTA (16 points per thread).
constexpr int kMaxLogLReal = 13;

// Runtime twin of team_log_e.
inline int team_log_e_rt(int log_l) {
  return log_l <= 5 ? log_l : (log_l == 6 ? 3 : (log_l == 10 ? 5 : 4));
}
inline int batch_log_e_rt(int log_l) { return team_log_e_rt(log_l); }

template <class P>
using LaunchFnT = void (*)(dim3, int, size_t, cudaStream_t, const P&);

template <class P>
struct KernelInfo {
  const void* fn = nullptr;
  int threads = 0;
  size_t smem = 0;
  int teams = 0;
  LaunchFnT<P> launch = nullptr;
};

using MeanInfo = KernelInfo<MeanParams>;
using FrameInfo = KernelInfo<FrameParams>;
using IstftInfo = KernelInfo<IstftParams>;
IstftInfo istft_lookup(int log_l);       // log_l in [1, kMaxLogL]
IstftInfo istft_half_lookup(int log_l);  // hop == nperseg / 2
IstftInfo istft_cplx_lookup(int log_l);  // two-sided input, complex output
IstftInfo istft_blue_lookup(int log_m);  // non-power-of-two nfft <= kBlueIstftMaxN (chirp-z)
constexpr int kBlueIstftMaxN = 2048;

// family: 0 welch mean, 1 cross mean
// (log_l in [0, kMaxLogLReal] for the real-input families below)
MeanInfo mean_lookup_welch(int log_l, int det);
MeanInfo mean_lookup_cross(int log_l, int det);
// det 0/1/2(spectral), log_l >= 1; blocked: the instantiation with shared-memory block totals
MeanInfo mean_lookup_welch_half(int log_l, int det, bool blocked);
MeanInfo mean_lookup_cross_half(int log_l, int det, bool csd);  // det 0/1/2(spectral)
FrameInfo frame_lookup_stft(int log_l, int det);
FrameInfo frame_lookup_power(int log_l, int det);
FrameInfo frame_lookup_stft_spectral(int log_l);   // constant detrend, spectral correction
FrameInfo frame_lookup_power_spectral(int log_l);
FrameInfo frame_lookup_cross(int log_l, int det);
// Bluestein kernels for a non-power-of-two nfft in [3, kBlueMaxN]: transform length
// M = 2^log_m >= 2 nfft - 1 (log_m in [4, 13]); det 0 none, 1 constant, 2 linear.
constexpr int kBlueMaxN = 4096;
inline int blue_log_m(int nfft) {
  int lm = 4;
  while ((1 << lm) < 2 * nfft - 1) ++lm;
  return lm;
}
MeanInfo blue_lookup_welch(int log_m, int det);
MeanInfo blue_lookup_cross(int log_m, int det);  // csd / coherence (same slots as k_cross_mean)
// complex input, power-of-two nfft (log_l in [0, kMaxLogL]); det 0 none, 1 constant, 2 linear
MeanInfo cplx_lookup_welch(int log_l, int det);
FrameInfo cplx_lookup_frames_stft(int log_l, int det);
FrameInfo cplx_lookup_frames_power(int log_l, int det);
MeanInfo cplx_lookup_csd(int log_l, int det);  // csd of two complex signals
FrameInfo blue_lookup_frames_stft(int log_m, int det);
FrameInfo blue_lookup_frames_power(int log_m, int det);
// hop == nperseg/2 == nfft/2, nfft >= 64 (empty info below); det 0/1/2(spectral)
FrameInfo frame_half_lookup_stft(int log_l, int det);
FrameInfo frame_half_lookup_power(int log_l, int det);

// Fold-expression lookup over LOG_L = 0..kMaxLogL and detrend 0..2 of an info factory.
template <class INFO, template <int, int> class F, int... LS>
INFO lookup_seq(int log_l, int det, std::integer_sequence<int, LS...>) {
  INFO out;
  (void)((log_l == LS ? (out = det == 0 ? F<LS, 0>::get()
                                        : (det == 1 ? F<LS, 1>::get() : F<LS, 2>::get()),
                         true)
                      : false) ||
         ...);
  return out;
}

template <class INFO, template <int, int> class F, int MAXL = kMaxLogL>
INFO lookup_all(int log_l, int det) {
  return lookup_seq<INFO, F>(log_l, det, std::make_integer_sequence<int, MAXL + 1>{});
}

}  // namespace b2s
