// Parameter blocks passed by value from the C-ABI layer to the framed-spectral kernels.
#pragma once

#include <stdint.h>

namespace b2s {

// Mean-of-segments kernels (welch / csd / coherence).
struct MeanParams {
  const float* x;      // (rows, n) with row stride ld, float32
  const float* y;      // second signal for csd/coherence (same layout), else nullptr
  int64_t ld_x, ld_y;  // row strides in elements
  int64_t rows;
  int nperseg;         // samples per segment (<= L)
  int hop;             // nperseg - noverlap
  int nseg;            // segments per row
  int detrend;         // kDetrend*
  const float* win;    // nperseg window values, sqrt(scale) folded in
  int64_t G;           // segments per team
  int cmax;            // partial-sum slots per row
  int64_t total;       // rows * nseg
  float* partial;      // workspace: [rows][cmax][slot_floats]
  const float2* wdft;  // DFT_L(win)[0..n_low) for the spectral detrend correction, else nullptr
  int n_low;           // bins of the window spectrum that are non-zero: |k| < n_low (mod L)
  int nfft;            // DFT length (the Bluestein kernels' N; equals L for the others)
};

// Per-frame kernels (stft / spectrogram / per-frame cross spectra).
struct FrameParams {
  const float* x;
  const float* y;
  int64_t ld_x, ld_y;
  int64_t rows;
  int64_t n;           // samples per row of the ORIGINAL signal
  int ext;             // boundary extension length on each side (nperseg/2 or 0)
  int ext_mode;        // 0 none, 1 zeros, 2 even, 3 odd, 4 constant
  int64_t n_ext;       // length after extension and padding (frames index into this)
  int nperseg;
  int hop;
  int nseg;
  int detrend;
  const float* win;
  int nbins;           // bins written per frame
  int64_t total;       // rows * nseg
  float* out;          // (rows, nseg, nbins) complex interleaved, or power
  float* out2;         // second output (per-frame pyy for coherence frames), else nullptr
  float* out3;         // third output (per-frame pxy), else nullptr
  const float2* wdft;  // DFT_nfft(win)[0..n_low) for the spectral constant detrend, else nullptr
  int n_low;
  int nfft;            // DFT length (the Bluestein kernels' N; equals L for the others)
};

}  // namespace b2s
