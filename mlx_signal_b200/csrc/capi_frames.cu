// C-ABI: per-frame spectra (stft, spectrogram psd, per-frame cross spectra).
#include <utility>

#include "capi_common.h"
#include "dispatch.cuh"

namespace b2s {
namespace {

FrameInfo lookup(int kind, int log_l, int det, bool spectral) {
  if (spectral) {
    return kind == kFrameStft ? frame_lookup_stft_spectral(log_l)
                              : frame_lookup_power_spectral(log_l);
  }
  if (kind == kFrameStft) return frame_lookup_stft(log_l, det);
  if (kind == kFramePower) return frame_lookup_power(log_l, det);
  return frame_lookup_cross(log_l, det);
}

int run_frames(int kind, const float* x, const float* y, int64_t rows, int64_t n, int64_t ldx,
               int64_t ldy, int ext, int ext_mode, int64_t n_total, const float* win,
               int nperseg, int nfft, int hop, int detrend, int onesided, float* out,
               void* stream, const float* wdft = nullptr, int n_low = 0) {
  if (!x || !win || !out || (kind == kFrameCross && !y) || ldx < n ||
      (kind == kFrameCross && ldy < n)) {
    set_error("null pointer or row stride smaller than n");
    return SP_ERR_ARG;
  }
  if (rows < 0 || n < 1 || ext < 0 || ext_mode < 0 || ext_mode > 4 || n_total < n + 2 * ext ||
      nperseg < 1 || nperseg > n_total || hop < 1 || hop > nperseg || nfft < nperseg ||
      detrend < 0 || detrend > 2 || n_total >= (int64_t(1) << 31) ||
      ((ext_mode == kExtEven || ext_mode == kExtOdd) && ext > n - 1)) {
    set_error("invalid frame arguments (n=%lld ext=%d n_total=%lld nperseg=%d hop=%d)",
              (long long)n, ext, (long long)n_total, nperseg, hop);
    return SP_ERR_ARG;
  }
  const int log_l = ilog2_exact(nfft);
  // stft / spectrogram with a non-power-of-two nfft: the Bluestein frame kernels
  const bool blue = log_l < 0 && kind != kFrameCross && nfft >= 3 && nfft <= kBlueMaxN;
  if (!blue && (log_l < 0 || log_l > kMaxLogLReal)) {
    set_error("nfft=%d: fused kernels need a power of two <= %d (stft/spectrogram: or any "
              "nfft <= %d)", nfft, 1 << kMaxLogLReal, kBlueMaxN);
    return SP_ERR_UNSUPPORTED;
  }
  // the spectral correction applies to the constant detrend when the window's spectrum is
  // confined to bins a team thread holds in its first and last register
  const bool spectral = !blue && kind != kFrameCross && detrend == kDetrendConstant &&
                        wdft != nullptr && n_low >= 1 &&
                        n_low <= ((1 << log_l) >> team_log_e_rt(log_l));
  FrameInfo f;
  if (blue) {
    const int lm = blue_log_m(nfft);
    f = kind == kFrameStft ? blue_lookup_frames_stft(lm, detrend)
                           : blue_lookup_frames_power(lm, detrend);
  } else {
    f = lookup(kind, log_l, detrend, spectral);
  }
  // 50% overlap with nperseg == nfft: the half-block kernel (each half-block loaded once, window
  // fused into the first butterfly stage) for no / constant detrend
  const bool half = !blue && kind != kFrameCross && nperseg == nfft && 2 * hop == nperseg &&
                    detrend <= 1;
  if (half) {
    const int hdet = spectral ? 2 : detrend;
    const FrameInfo fh = kind == kFrameStft ? frame_half_lookup_stft(log_l, hdet)
                                            : frame_half_lookup_power(log_l, hdet);
    if (fh.fn != nullptr) f = fh;
  }
  const int nseg = int((n_total - nperseg) / hop + 1);
  const int64_t total = rows * nseg;
  if (total == 0) return SP_OK;
  int sms = 0;
  const int nb = resident_ctas(f.fn, f.threads, f.smem, &sms);
  if (nb <= 0) {
    set_error("no resident CTA for frame kernel (nfft=%d)", nfft);
    return SP_ERR_UNSUPPORTED;
  }
  const int64_t per = kind == kFrameCross ? 1 : 2;
  const int64_t want_teams = cdiv(total, per);
  int64_t blocks = cdiv(want_teams, f.teams);
  const int64_t cap = int64_t(nb) * sms;
  if (blocks > cap) blocks = cap;
  FrameParams p;
  p.x = x;
  p.y = y;
  p.ld_x = ldx;
  p.ld_y = ldy;
  p.rows = rows;
  p.n = n;
  p.ext = ext;
  p.ext_mode = ext_mode;
  p.n_ext = n_total;
  p.nperseg = nperseg;
  p.hop = hop;
  p.nseg = nseg;
  p.detrend = detrend;
  p.win = win;
  p.nbins = onesided ? nfft / 2 + 1 : nfft;
  p.total = total;
  p.out = out;
  p.out2 = nullptr;
  p.out3 = nullptr;
  p.wdft = spectral ? reinterpret_cast<const float2*>(wdft) : nullptr;
  p.n_low = spectral ? n_low : 0;
  p.nfft = nfft;
  f.launch(dim3(unsigned(blocks)), f.threads, f.smem, static_cast<cudaStream_t>(stream), p);
  B2S_CHECK_CUDA(cudaGetLastError(), "frame kernel launch");
  return SP_OK;
}

// Per-frame spectra of complex rows (x interleaved complex64, ld in complex elements):
// power-of-two nfft, two-sided, one frame per transform.
int run_frames_cplx(const float* x, int64_t rows, int64_t n, int64_t ld, int ext, int ext_mode,
                    int64_t n_total, const float* win, int nperseg, int nfft, int hop, int detrend,
                    int power, float* out, void* stream) {
  if (!x || !win || !out || ld < n) {
    set_error("null pointer or row stride smaller than n");
    return SP_ERR_ARG;
  }
  if (rows < 0 || n < 1 || ext < 0 || ext_mode < 0 || ext_mode > 4 || n_total < n + 2 * ext ||
      nperseg < 1 || nperseg > n_total || hop < 1 || hop > nperseg || nfft < nperseg ||
      detrend < 0 || detrend > 2 || n_total >= (int64_t(1) << 31) ||
      ((ext_mode == kExtEven || ext_mode == kExtOdd) && ext > n - 1)) {
    set_error("invalid frame arguments (n=%lld ext=%d n_total=%lld nperseg=%d hop=%d)",
              (long long)n, ext, (long long)n_total, nperseg, hop);
    return SP_ERR_ARG;
  }
  const int log_l = ilog2_exact(nfft);
  if (log_l < 0 || log_l > kMaxLogL) {
    set_error("nfft=%d: complex-input frame kernels need a power of two <= %d", nfft,
              1 << kMaxLogL);
    return SP_ERR_UNSUPPORTED;
  }
  const FrameInfo f = power ? cplx_lookup_frames_power(log_l, detrend)
                            : cplx_lookup_frames_stft(log_l, detrend);
  const int nseg = int((n_total - nperseg) / hop + 1);
  const int64_t total = rows * nseg;
  if (total == 0) return SP_OK;
  int sms = 0;
  const int nb = resident_ctas(f.fn, f.threads, f.smem, &sms);
  if (nb <= 0) {
    set_error("no resident CTA for complex frame kernel (nfft=%d)", nfft);
    return SP_ERR_UNSUPPORTED;
  }
  int64_t blocks = cdiv(total, f.teams);
  const int64_t cap = int64_t(nb) * sms;
  if (blocks > cap) blocks = cap;
  FrameParams p = {};
  p.x = x;
  p.ld_x = ld;
  p.rows = rows;
  p.n = n;
  p.ext = ext;
  p.ext_mode = ext_mode;
  p.n_ext = n_total;
  p.nperseg = nperseg;
  p.hop = hop;
  p.nseg = nseg;
  p.detrend = detrend;
  p.win = win;
  p.nbins = nfft;
  p.total = total;
  p.out = out;
  p.nfft = nfft;
  f.launch(dim3(unsigned(blocks)), f.threads, f.smem, static_cast<cudaStream_t>(stream), p);
  B2S_CHECK_CUDA(cudaGetLastError(), "complex frame kernel launch");
  return SP_OK;
}

}  // namespace
}  // namespace b2s

extern "C" {

int sp_frames_cplx(const float* x, int64_t rows, int64_t n, int64_t ld, int ext, int ext_mode,
                   int64_t n_total, const float* win, int nperseg, int nfft, int hop, int detrend,
                   int power, float* out, void* stream) {
  return b2s::run_frames_cplx(x, rows, n, ld, ext, ext_mode, n_total, win, nperseg, nfft, hop,
                              detrend, power, out, stream);
}

int sp_stft_c64(const float* x, int64_t rows, int64_t n, int64_t ld, int ext, int ext_mode,
                int64_t n_total, const float* win, int nperseg, int nfft, int hop, int detrend,
                int onesided, float* out, void* stream) {
  return b2s::run_frames(b2s::kFrameStft, x, nullptr, rows, n, ld, 0, ext, ext_mode, n_total,
                         win, nperseg, nfft, hop, detrend, onesided, out, stream);
}

int sp_stft_c64_ex(const float* x, int64_t rows, int64_t n, int64_t ld, int ext, int ext_mode,
                   int64_t n_total, const float* win, const float* win_dft_low, int n_low,
                   int nperseg, int nfft, int hop, int detrend, int onesided, float* out,
                   void* stream) {
  return b2s::run_frames(b2s::kFrameStft, x, nullptr, rows, n, ld, 0, ext, ext_mode, n_total,
                         win, nperseg, nfft, hop, detrend, onesided, out, stream, win_dft_low,
                         n_low);
}

int sp_spectrogram_f32_ex(const float* x, int64_t rows, int64_t n, int64_t ld, int ext,
                          int ext_mode, int64_t n_total, const float* win,
                          const float* win_dft_low, int n_low, int nperseg, int nfft, int hop,
                          int detrend, int onesided, float* out, void* stream) {
  return b2s::run_frames(b2s::kFramePower, x, nullptr, rows, n, ld, 0, ext, ext_mode, n_total,
                         win, nperseg, nfft, hop, detrend, onesided, out, stream, win_dft_low,
                         n_low);
}

int sp_spectrogram_f32(const float* x, int64_t rows, int64_t n, int64_t ld, int ext,
                       int ext_mode, int64_t n_total, const float* win, int nperseg, int nfft,
                       int hop, int detrend, int onesided, float* out, void* stream) {
  return b2s::run_frames(b2s::kFramePower, x, nullptr, rows, n, ld, 0, ext, ext_mode, n_total,
                         win, nperseg, nfft, hop, detrend, onesided, out, stream);
}

int sp_csd_frames_c64(const float* x, const float* y, int64_t rows, int64_t n, int64_t ldx,
                      int64_t ldy, const float* win, int nperseg, int nfft, int hop, int detrend,
                      int onesided, float* out, void* stream) {
  return b2s::run_frames(b2s::kFrameCross, x, y, rows, n, ldx, ldy, 0, 0, n, win, nperseg, nfft,
                         hop, detrend, onesided, out, stream);
}

}
