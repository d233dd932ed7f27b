/*
 * b200signal: C-ABI of the B200 (sm_100a) framed-FFT spectral kernels.
 *
 * Every entry point takes raw device pointers, plain sizes and a CUDA stream (cudaStream_t
 * passed as void*), launches asynchronously on that stream and returns an int status
 * (SP_OK = 0, negative on error; sp_last_error() gives the text of the calling thread's last
 * error). Nothing here synchronises the device, allocates device memory or falls back to a
 * CPU path: shapes the kernels do not cover return SP_ERR_UNSUPPORTED.
 *
 * The functions replace the kernel-module boundary of the reference library
 * (src/mlx_signal_processing/_stft_metal.py and _fourstep_metal.py): Python functions that
 * take MLX arrays plus integers and launch JIT-compiled Metal kernels. Citations below are to
 * those files. Windows arrive with the scipy scale factor already folded in (sqrt(scale) for
 * PSD/CSD, as at src/mlx_signal_processing/spectral.py:312-316).
 *
 * Layout conventions: a signal is `rows` rows of `n` float32 samples with row stride `ld`
 * (elements); complex outputs are interleaved (re, im) float32 pairs (complex64).
 */
#ifndef B200SIGNAL_H
#define B200SIGNAL_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SP_API __attribute__((visibility("default")))
#else
#define SP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define SP_VERSION 100

enum {
  SP_OK = 0,
  SP_ERR_ARG = -1,          /* invalid argument (null pointer, bad size) */
  SP_ERR_UNSUPPORTED = -2,  /* shape outside the fused kernels (e.g. non power-of-two nfft) */
  SP_ERR_WORKSPACE = -3,    /* workspace smaller than the size query returned */
  SP_ERR_CUDA = -4,         /* CUDA runtime error (text in sp_last_error) */
  SP_ERR_TIMEOUT = -5       /* a bounded device-side wait gave up */
};

enum { SP_DETREND_NONE = 0, SP_DETREND_CONSTANT = 1, SP_DETREND_LINEAR = 2 };

/* Library version (SP_VERSION). */
SP_API int sp_version(void);

/* Text of the calling thread's last error ("" if none). */
SP_API const char* sp_last_error(void);

/*
 * Workspace bytes for sp_welch_f32 (kind 0), sp_csd_c64 / sp_coherence_f32 (kind 1),
 * sp_welch_c64 (kind 3) or sp_csd_cplx (kind 4) on the current device. Negative return = error
 * status.
 * Replaces the implicit group-partial buffers of _stft_metal.rfft_power_mean
 * (_stft_metal.py:530-557) and _pair_sum_launch (_stft_metal.py:703-736).
 */
SP_API int64_t sp_mean_workspace_size(int kind, int64_t rows, int64_t n, int nperseg, int nfft, int hop,
                               int detrend);

/*
 * Welch PSD: out[r][k] = (onesided ? f_k : 1) / nseg * sum_s |FFT_nfft(win * detrend(x_rs))_k|^2
 * for k < (onesided ? nfft/2+1 : nfft), segments x_rs = x[r, s*hop : s*hop+nperseg].
 * nfft: a power of two in [1, 8192], or any other value in [3, 4096] (chirp-z kernels), with
 * nperseg <= nfft; win holds nperseg values.
 * Replaces _stft_metal.rfft_power_mean (_stft_metal.py:530-557) together with the deferred
 * one-sided factor of spectral.csd (spectral.py:468-488); for a non-power-of-two nfft the composed
 * frames + mx.fft.rfft path of spectral._fft_frames (spectral.py:127-147).
 */
SP_API int sp_welch_f32(const float* x, int64_t rows, int64_t n, int64_t ld, const float* win,
                 int nperseg, int nfft, int hop, int detrend, int onesided, float* out,
                 void* workspace, size_t workspace_bytes, void* stream);

/*
 * Welch PSD of complex rows (x interleaved complex64, ld in complex elements), two-sided:
 * out[r][k] = 1/nseg * sum_s |FFT_nfft(win * detrend(x_rs))_k|^2, k < nfft; the detrend acts on
 * the real and imaginary parts separately. nfft a power of two in [1, 4096]. Workspace:
 * sp_mean_workspace_size(3, ...). Replaces the composed complex path of spectral.csd
 * (spectral.py:290-298 two-sided switch, :127-147 frames + mx.fft.fft).
 */
SP_API int sp_welch_c64(const float* x, int64_t rows, int64_t n, int64_t ld, const float* win,
                        int nperseg, int nfft, int hop, int detrend, float* out, void* workspace,
                        size_t workspace_bytes, void* stream);

/*
 * Cross spectral density of complex rows x, y (interleaved complex64, ld in complex elements),
 * two-sided: out[r][k] = 1/nseg * sum_s conj(X_rs[k]) Y_rs[k] (complex64), k < nfft, nfft a power
 * of two in [1, 4096]. Workspace: sp_mean_workspace_size(4, ...). Replaces the composed complex
 * path of spectral.csd (spectral.py:290-298, :127-147: frames + mx.fft.fft of x and y).
 */
SP_API int sp_csd_cplx(const float* x, const float* y, int64_t rows, int64_t n, int64_t ldx,
                       int64_t ldy, const float* win, int nperseg, int nfft, int hop, int detrend,
                       float* out, void* workspace, size_t workspace_bytes, void* stream);

/*
 * sp_welch_f32 with the constant detrend applied in the frequency domain. `win_dft_low` is a
 * device pointer to n_low complex64 values DFT_nfft(win)[0..n_low) (win zero-padded to nfft);
 * the caller guarantees that DFT_nfft(win)[k] is zero (to float32 rounding) for
 * n_low <= k <= nfft - n_low, as for hann / hamming / blackman / boxcar. The segment means are
 * then removed as Z_k -= m * DFT(win)_k on those bins only, off the FFT's critical path. Used
 * when detrend == SP_DETREND_CONSTANT, nperseg == nfft == 2*hop and
 * 1 <= n_low <= sp_welch_spectral_bins(nfft); otherwise identical to sp_welch_f32 (pass NULL).
 * Same reference counterpart as sp_welch_f32 (_stft_metal.py:530-557; the reference subtracts
 * the mean in the time domain, _stft_metal.py:40-61).
 */
SP_API int sp_welch_f32_ex(const float* x, int64_t rows, int64_t n, int64_t ld, const float* win,
                           const float* win_dft_low, int n_low, int nperseg, int nfft, int hop,
                           int detrend, int onesided, float* out, void* workspace,
                           size_t workspace_bytes, void* stream);

/* Largest n_low sp_welch_f32_ex accepts for this nfft (0 if nfft is not a supported power of
 * two). */
SP_API int sp_welch_spectral_bins(int nfft);

/*
 * sp_welch_f32 without a workspace argument, for callers that cannot allocate device memory
 * (plugin hosts that only receive input/output pointers, latency-critical loops that must not
 * call cudaMalloc after start-up). No counterpart in the reference: it is an addition of this
 * library. The partial sums live in a fixed 16 MiB static device array, held on each device from
 * the first use of the library's spectral-mean kernels there (modules load lazily by default)
 * until the process exits; shapes needing more scratch than that return SP_ERR_WORKSPACE
 * (sp_mean_workspace_size(0, ...) gives the need). It calls no cudaMalloc/cudaFree. The first
 * call on a device resolves the array's device address (cudaGetSymbolAddress, with that device
 * current) and should come before any stream capture; the address is cached per device and
 * resolved again when the device's context changes (after a cudaDeviceReset). All calls share
 * the one array: calls that overlap on the GPU (for example on two streams at once) race and
 * must be serialised by the caller. Nothing from a previous call is read: every partial sum a
 * call reads is written by that call first.
 */
SP_API int sp_welch_f32_noalloc(const float* x, int64_t rows, int64_t n, int64_t ld,
                                const float* win, int nperseg, int nfft, int hop, int detrend,
                                int onesided, float* out, void* stream);

/*
 * Cross spectral density mean conj(X_s) Y_s over segments (complex64 out, same bin count and
 * one-sided doubling as sp_welch_f32). Replaces _stft_metal.csd_mean (_stft_metal.py:739-741).
 */
SP_API int sp_csd_c64(const float* x, const float* y, int64_t rows, int64_t n, int64_t ldx,
               int64_t ldy, const float* win, int nperseg, int nfft, int hop, int detrend,
               int onesided, float* out, void* workspace, size_t workspace_bytes, void* stream);

/*
 * Magnitude-squared coherence |Pxy|^2 / (Pxx Pyy) from one sweep (float32 out, nfft/2+1 bins),
 * guarded (0 where Pxx Pyy == 0) and clamped to [0, 1]. Replaces _stft_metal.coherence_mean
 * (_stft_metal.py:744-746) plus the unguarded ratio of spectral.coherence (spectral.py:609-613).
 */
SP_API int sp_coherence_f32(const float* x, const float* y, int64_t rows, int64_t n, int64_t ldx,
                     int64_t ldy, const float* win, int nperseg, int nfft, int hop, int detrend,
                     float* out, void* workspace, size_t workspace_bytes, void* stream);

/*
 * sp_csd_c64 / sp_coherence_f32 with the constant detrend applied in the frequency domain, as
 * sp_welch_f32_ex: win_dft_low = DFT_nfft(win)[0..n_low) (complex), used by the 50%-overlap
 * kernels (nperseg == nfft == 2*hop) when detrend == SP_DETREND_CONSTANT and
 * 1 <= n_low <= sp_welch_spectral_bins(nfft); otherwise identical to the plain entry points.
 * Same workspace size (sp_mean_workspace_size kind 1). Same reference counterparts.
 */
SP_API int sp_csd_c64_ex(const float* x, const float* y, int64_t rows, int64_t n, int64_t ldx,
                         int64_t ldy, const float* win, const float* win_dft_low, int n_low,
                         int nperseg, int nfft, int hop, int detrend, int onesided, float* out,
                         void* workspace, size_t workspace_bytes, void* stream);
SP_API int sp_coherence_f32_ex(const float* x, const float* y, int64_t rows, int64_t n,
                               int64_t ldx, int64_t ldy, const float* win,
                               const float* win_dft_low, int n_low, int nperseg, int nfft,
                               int hop, int detrend, float* out, void* workspace,
                               size_t workspace_bytes, void* stream);


/*
 * Per-frame spectra of complex rows (x interleaved complex64, ld in complex elements), two-sided:
 * out (rows, nseg, nfft) complex64 X_s (power = 0) or float32 |X_s|^2 (power = 1), with the same
 * boundary extension / padding arguments as sp_stft_c64; nfft a power of two in [1, 4096].
 * Replaces the composed complex path of spectral._fft_frames (spectral.py:127-147) used by
 * stft / spectrogram on complex input.
 */
SP_API int sp_frames_cplx(const float* x, int64_t rows, int64_t n, int64_t ld, int ext,
                          int ext_mode, int64_t n_total, const float* win, int nperseg, int nfft,
                          int hop, int detrend, int power, float* out, void* stream);

/*
 * Column medians over segments (average='median'): out[r * ncols + c] = scale * median over
 * s < nseg of in[(r * nseg + s) * ld_frame + c] (mean of the two middle values for an even nseg),
 * for per-frame spectra (rows, nseg, ncols) with frame stride ld_frame floats; a complex spectrum
 * is passed as its float view (real and imaginary parts are separate columns). nseg up to 49151
 * (staged in shared memory), else SP_ERR_UNSUPPORTED. Replaces the median branch of spectral.csd
 * (spectral.py:469-477: median of the per-segment spectra along the segment axis / median bias).
 */
SP_API int sp_median_frames_f32(const float* in, int64_t rows, int nseg, int ncols,
                                int64_t ld_frame, float scale, float* out, void* stream);

/* Boundary extension modes of the per-frame entry points (scipy stft `boundary`). */
enum { SP_EXT_NONE = 0, SP_EXT_ZEROS = 1, SP_EXT_EVEN = 2, SP_EXT_ODD = 3, SP_EXT_CONSTANT = 4 };

/*
 * Per-frame windowed FFT (stft). The signal is virtually extended by `ext` samples per side
 * with `ext_mode` and zero-padded to `n_total` (>= n + 2*ext); frame s covers extended samples
 * [s*hop, s*hop + nperseg). Output: (rows, nseg, nbins) complex64, nseg = (n_total-nperseg)/hop+1,
 * nbins = onesided ? nfft/2+1 : nfft. Replaces _stft_metal.rfft_frames(power=False)
 * (_stft_metal.py:192-220) and the materialised boundary/pad concatenates of
 * spectral._spectral_helper (spectral.py:275-288).
 */
SP_API int sp_stft_c64(const float* x, int64_t rows, int64_t n, int64_t ld, int ext, int ext_mode,
                       int64_t n_total, const float* win, int nperseg, int nfft, int hop,
                       int detrend, int onesided, float* out, void* stream);

/*
 * Per-frame power |X|^2 with the one-sided doubling applied (spectrogram mode 'psd'), same
 * framing and layout as sp_stft_c64 (float32 out). Replaces _stft_metal.rfft_frames(power=True)
 * (_stft_metal.py:192-220) plus the one-sided factor of spectral.py:348-353.
 */
SP_API int sp_spectrogram_f32(const float* x, int64_t rows, int64_t n, int64_t ld, int ext,
                              int ext_mode, int64_t n_total, const float* win, int nperseg,
                              int nfft, int hop, int detrend, int onesided, float* out,
                              void* stream);

/*
 * sp_stft_c64 / sp_spectrogram_f32 with the constant detrend (detrend == SP_DETREND_CONSTANT)
 * applied after the transform as a correction on the window's non-zero low bins: win_dft_low
 * holds DFT_nfft(win)[0..n_low) as complex (re, im); it is used when 1 <= n_low <=
 * sp_welch_spectral_bins(nfft), otherwise the time-domain detrend runs. Same outputs as the plain
 * entry points (scipy's detrend='constant': mean removed per segment before the window).
 */
SP_API int sp_stft_c64_ex(const float* x, int64_t rows, int64_t n, int64_t ld, int ext,
                          int ext_mode, int64_t n_total, const float* win,
                          const float* win_dft_low, int n_low, int nperseg, int nfft, int hop,
                          int detrend, int onesided, float* out, void* stream);
SP_API int sp_spectrogram_f32_ex(const float* x, int64_t rows, int64_t n, int64_t ld, int ext,
                                 int ext_mode, int64_t n_total, const float* win,
                                 const float* win_dft_low, int n_low, int nperseg, int nfft,
                                 int hop, int detrend, int onesided, float* out, void* stream);

/*
 * Per-frame cross spectra conj(X_s) Y_s, (rows, nseg, nbins) complex64, no one-sided factor.
 * Replaces _stft_metal.csd_frames (_stft_metal.py:412-414), used for average='median'.
 */
SP_API int sp_csd_frames_c64(const float* x, const float* y, int64_t rows, int64_t n,
                             int64_t ldx, int64_t ldy, const float* win, int nperseg, int nfft,
                             int hop, int detrend, int onesided, float* out, void* stream);

/*
 * Fused inverse STFT of one-sided spectra: z is (rows, nseg, ldf) complex64 (row stride ld_row
 * complex elements), bins k < nbins_in used, missing bins up to nperseg/2 taken as zero, the
 * DC and Nyquist bins taken as real (irfft semantics). Output: (rows, outlen) float32 with
 * outlen = nperseg + (nseg-1)*hop, x = OLA(irfft(z) * win * scale) / norm where
 * norm = OLA(win^2) and samples with norm <= 1e-10 are not divided (scipy's rule); the caller
 * trims the boundary. nperseg (== nfft) must be a power of two in [2, 4096].
 * Replaces _stft_metal.istft_frames (_stft_metal.py:851-887: _ISTFT_SRC :753-795 then the
 * gather OLA _OLA_SRC :797-820) and the norm division of spectral.istft (spectral.py:929-943).
 */
SP_API int sp_istft_f32(const float* z, int64_t rows, int nseg, int64_t ld_row, int ldf,
                        int nbins_in, const float* win, float scale, int nperseg, int hop,
                        float* out, void* stream);

/*
 * sp_istft_f32 with an FFT length nfft >= nperseg (a power of two in [2, 4096], or any other
 * value in [3, 2048]: chirp-z kernel; any nperseg >= 1): each frame is the first nperseg samples
 * of the nfft-point inverse real DFT of its one-sided spectrum (nbins_in <= nfft/2 + 1 bins),
 * windowed by the nperseg-point win; outlen = nperseg + (nseg-1)*hop. nfft == nperseg is
 * sp_istft_f32. Replaces the composed branch of spectral.istft (spectral.py:929-950:
 * irfft(n=nfft)[:nperseg], then overlap-add).
 */
SP_API int sp_istft_f32_ex(const float* z, int64_t rows, int nseg, int64_t ld_row, int ldf,
                           int nbins_in, const float* win, float scale, int nperseg, int nfft,
                           int hop, float* out, void* stream);

/*
 * Two-sided inverse STFT (input_onesided=False): z (rows, nseg, ldf) complex64 two-sided spectra
 * (bins k < nbins_in <= nfft used, the rest zero); each frame is the first nperseg samples of the
 * nfft-point inverse complex FFT, windowed, overlap-added and divided by the window energy as in
 * sp_istft_f32; out (rows, outlen) complex64. nfft a power of two in [2, 4096]. Replaces the
 * two-sided branch of spectral.istft (spectral.py:929-950: ifft, then overlap-add).
 */
SP_API int sp_istft_c64(const float* z, int64_t rows, int nseg, int64_t ld_row, int ldf,
                        int nbins_in, const float* win, float scale, int nperseg, int nfft,
                        int hop, float* out, void* stream);

/* Workspace bytes for the long transforms below (two N-point complex intermediates + the device
 * error word; N = n for sp_fft_c64, n/2 for the real transforms, where N may also be C 2^e with
 * C odd <= 15). Negative = error status. */
SP_API int64_t sp_fft_workspace_size(int64_t n, int batch);

/*
 * Complex FFT (inverse != 0: inverse FFT including 1/n) of `batch` contiguous rows of n complex64
 * values, n a power of two in [2^12, 2^26], in three TMA-staged passes; in/out/workspace 16-byte
 * aligned, out must not alias in. Replaces _fourstep_metal.fft3_last (_fourstep_metal.py:272-303)
 * and _fourstep._fft_4step_last / _ifft_4step_last (_fourstep.py:100-150).
 */
SP_API int sp_fft_c64(const float* in, float* out, int batch, int64_t n, int inverse,
                      void* workspace, size_t workspace_bytes, void* stream);

/*
 * Real-input FFT of `batch` contiguous rows of n float32: X rows of n/2+1 complex64 bins with row
 * stride ldx_out (complex elements). n = 2 C 2^e with C odd in [1, 15] and e in [12, 26]: C = 1
 * is the packed power-of-two transform (three passes + untangle); C > 1 splits the rows into C
 * decimated branches (one deinterleave kernel), runs their packed 2^e-point transforms as one
 * batch, and untangles and combines them with one radix-C kernel. Replaces _fourstep.rfft_large
 * (_fourstep.py:213-231) with its untangle (:195-210) and, for composite lengths, the divisor
 * split of _fourstep._choose_split (:55-72) over MLX's mixed-radix FFT.
 */
SP_API int sp_rfft_c64(const float* x, float* X, int batch, int64_t n, int64_t ldx_out,
                       void* workspace, size_t workspace_bytes, void* stream);

/*
 * Inverse real FFT: X rows (stride ldx complex, nbins valid bins, DC/Nyquist taken as real,
 * missing bins zero) -> batch contiguous rows of n float32, n = 2 C 2^e as for sp_rfft_c64
 * (C > 1: one radix-C fold + pretwist kernel, the C branch inverses as one batch, one interleave
 * kernel). Replaces _fourstep.irfft_large (_fourstep.py:372-408).
 */
SP_API int sp_irfft_f32(const float* X, int64_t ldx, int nbins, float* x, int batch, int64_t n,
                        void* workspace, size_t workspace_bytes, void* stream);

/*
 * Analytic signal (scipy.signal.hilbert) of `batch` contiguous rows of n real float32 samples:
 * out (batch, n) complex64 = IFFT_n(h FFT_n(x)) with h = 1 at 0 and n/2, 2 between, 0 above.
 * n even with n/2 and n powers of two in [2^12, 2^26]; workspace sp_fft_workspace_size(n, batch)
 * bytes (same error word as sp_fft_c64). Forward packed real transform (three passes), one
 * kernel that untangles it and writes the masked spectrum into `out`, and the n-point inverse
 * transform in place. Replaces the reference's hilbert (filtering.py:43-84: rfft, mask, ifft as
 * separate array operations).
 */
SP_API int sp_hilbert_c64(const float* x, float* out, int batch, int64_t n, void* workspace,
                          size_t workspace_bytes, void* stream);

/*
 * Fourier-method resampling of `batch` contiguous real rows from n to num samples
 * (scipy.signal.resample for real input, no window, time domain): the min(n, num)/2 + 1 lowest
 * bins of rfft_n(x), the unpaired bin m/2 of an even m = min(n, num) doubled when num < n or
 * halved when num > n, scaled by num/n, inverse-transformed to num samples. n and num each
 * 2 C 2^e as for sp_rfft_c64; x, y, workspace 16-byte aligned; workspace
 * sp_resample_workspace_size(n, num, batch) bytes, its error word at
 * sp_fft_error_word(workspace, max(n, num)/2, batch). One forward and one inverse transform with
 * the bin selection and scaling folded into their untangle / pretwist kernels. Replaces the
 * reference's resample (resampling.py:60-176: rfft, slice, bin fix-up, scale, irfft as separate
 * array operations).
 */
SP_API int64_t sp_resample_workspace_size(int64_t n, int64_t num, int batch);
SP_API int sp_resample_f32(const float* x, int batch, int64_t n, float* y, int64_t num,
                           void* workspace, size_t workspace_bytes, void* stream);

/*
 * Process-wide sticky error of the long transforms: SP_ERR_TIMEOUT once any of their bounded
 * waits has run out since the last clear (the kernels store it in mapped pinned host memory as
 * well as in the workspace word), else 0. clear != 0 resets it after reading. A plain host load:
 * no CUDA call, no synchronisation (a timeout becomes visible once the failing CTA has stored
 * it; synchronise the stream first to cover every transform issued). No counterpart in the
 * reference (its waits are not bounded).
 */
SP_API int sp_fft_sticky_error(int clear);

/* Byte offset of the int error word inside a long-transform workspace (0 = ok, SP_ERR_TIMEOUT if
 * a tile copy wait gave up); read it after synchronising the stream. */
SP_API int sp_fft_error_word(const void* workspace, int64_t n, int batch, int64_t* offset);

/*
 * Poll limit of the bounded wait each long-transform CTA makes for a tile's TMA copy (process
 * wide, read at every launch; 0xffffffff restores the default of 2^22 polls). A wait that runs
 * out records SP_ERR_TIMEOUT in the error word, drains its own copies (bounded by the default
 * limit) and returns; the transform's output is then undefined. A host watchdog test sets it to
 * 0 to make every wait run out. Returns the previous limit. No counterpart in the reference
 * (its Metal kernels have no device-side waits, _fourstep_metal.py:58-185).
 */
SP_API uint32_t sp_fft_set_wait_limit(uint32_t polls);

/*
 * Batched 32-point complex DFTs on the tensor cores: y[v] = DFT_32(z[v]) for v < nvec (z, y:
 * nvec x 32 interleaved complex64, 16-byte aligned device pointers). Each tile of 128 vectors is
 * one tcgen05 GEMM (M 128, N 64, K 192) over FP16 head/tail splits of the vectors and of the
 * DFT matrix (three products, FP32 accumulation in tensor memory; each vector scaled by a power
 * of two into the FP16 range first): error ~1e-7 of the vector's peak, the class of an FP32 FFT.
 * reps > 1 repeats the MMA chain on the staged operands (same result) to measure the tensor-core
 * rate alone. err_word (device int, may be NULL) receives SP_ERR_TIMEOUT if the bounded wait for
 * the MMAs runs out. The radix-32 DFT stage of the framed FFTs, which the reference computes as
 * radix-2 threadgroup butterflies (_stft_metal.py:124-144), on the tensor cores.
 */
SP_API int sp_dft32_tc_c64(const float* z, float* y, int64_t nvec, int reps, int* err_word,
                           void* stream);

/*
 * FFT convolution of each of `rows` real rows x (n1 samples, row stride ld_x) with one real filter
 * h of n2 <= 2049 taps: out[r * ld_out + i] = (x_r * h)[j0 + i] for i in [0, nout), where
 * (x_r * h)[j] = sum_k h[k] x_r[j - k] is the full linear convolution (length n1 + n2 - 1;
 * j0 = 0 gives 'full', the centred windows 'same' / 'valid'). One fused overlap-save kernel:
 * blocks of L = sp_conv_block_len(n2) samples, two blocks per complex FFT, spectrum multiply and
 * inverse in registers; no workspace. Replaces the fused block convolution and gather overlap-add
 * of oaconvolve (_stft_metal.fftconv_blocks, _stft_metal.py:1024-1058 with kernels :900-1003;
 * _ola_metal.ola_gather, _ola_metal.py:63-78; routed from convolution.py:288-306).
 */
SP_API int sp_conv_ols_f32(const float* x, int64_t rows, int64_t n1, int64_t ld_x, const float* h,
                           int n2, int64_t j0, int64_t nout, float* out, int64_t ld_out,
                           void* stream);

/* Block length the convolution uses for n2 taps, or SP_ERR_UNSUPPORTED when n2 > 2049. */
SP_API int sp_conv_block_len(int n2);

/* ------------------------------------------------------------------------------------------
 * Batched persistent launch: many welch requests and streaming-STFT chunks of uneven size and
 * nperseg in one kernel launch over a device work queue. The reference has no batched form; a
 * batch replaces one welch (spectral.py:492-526 -> _stft_metal.rfft_power_mean :530-557) or
 * stft (spectral.py:694-738 -> _stft_metal.rfft_frames :192-220) call per request.
 *
 * Usage: sp_batch_plan -> sizes; sp_batch_encode writes the descriptor table into host memory
 * (pinned, so the caller's host-to-device copy can be asynchronous or graph-captured); the
 * caller copies it to a device buffer of the same size; sp_batch_run launches. The workspace
 * must be zero-filled before its first run; every run leaves its queue and counters zero again,
 * and sp_batch_run's arguments do not depend on the batch, so one captured launch replays for
 * any batch encoded into the same descriptor buffer and workspace. Outputs must not alias
 * inputs or one another. Batched classes: nperseg == nfft in {256, 512, 1024, 2048, 4096}.
 * ------------------------------------------------------------------------------------------ */
enum { SP_BATCH_WELCH = 0, SP_BATCH_STFT_STREAM = 1 };

typedef struct sp_batch_request {
  int kind;          /* SP_BATCH_WELCH or SP_BATCH_STFT_STREAM */
  int nperseg;       /* == nfft: 256, 512, 1024 or 4096 */
  int hop;           /* welch: nperseg/2; stream: 1..nperseg */
  int detrend;       /* welch: SP_DETREND_NONE or SP_DETREND_CONSTANT (spectral form) */
  int onesided;      /* welch: 1 one-sided (interior bins doubled), 0 two-sided; stream: 1 */
  int n_low;         /* welch constant detrend: complex values in win_dft_low (1..nperseg/32) */
  int seg_per_task;  /* schedule: segments (welch) or frames (stream) per team task; 0 default */
  int tail_len;      /* stream: samples held in tail_in (0 <= tail_len < nperseg) */
  int64_t rows;      /* channels / independent rows */
  int64_t n;         /* samples per row (stream: new samples in this chunk) */
  int64_t ld;        /* row stride of x, elements */
  int64_t tail_ld;   /* stream: row stride of tail_in and tail_out (>= nperseg) */
  const float* x;
  const float* win;          /* nperseg window values (no scale folded in) */
  const float* win_dft_low;  /* welch constant detrend: DFT_nperseg(win)[0..n_low) as (re, im) */
  const float* tail_in;      /* stream: previous tail, rows x tail_ld */
  float* tail_out;           /* stream: receives the new tail (must differ from tail_in) */
  float* out;  /* welch: rows x nbins float32 (nbins = nperseg/2+1 or nperseg);
                  stream: rows x frames x (nperseg/2+1) complex64 */
  float scale; /* welch: PSD scale (1/(fs*sum w^2) density, 1/(sum w)^2 spectrum);
                  stream: frame scale (1/sum w for scipy's 'spectrum' stft) */
} sp_batch_request;

/* Frames a stream chunk of n samples yields after a tail of tail_len samples (frames start every
 * hop samples of tail || chunk), and the length of the tail it leaves. Negative = error. */
SP_API int64_t sp_batch_stream_frames(int64_t tail_len, int64_t n, int nperseg, int hop,
                                      int64_t* new_tail_len);

/* 1 if nperseg is a batched class, else 0. */
SP_API int sp_batch_supported(int nperseg);

/* Validate a batch; *desc_bytes = descriptor table size, *ws_bytes = workspace size. */
SP_API int sp_batch_plan(const sp_batch_request* reqs, int nreq, int64_t* desc_bytes,
                         int64_t* ws_bytes);

/* Write the descriptor table for a batch whose launch will use workspace ws (device). */
SP_API int sp_batch_encode(const sp_batch_request* reqs, int nreq, void* ws, size_t ws_bytes,
                           void* desc_host, size_t desc_bytes);

/* Resident CTAs of the 128-thread batch kernel (classes 256 ... 2048) on the current device (its
 * default persistent grid). */
SP_API int sp_batch_max_grid(void);

/* Launch a batch from its device descriptor table: the 4096-point class on a 256-thread
 * persistent kernel (resident maximum), then the other classes on the 128-thread kernel (grid
 * CTAs; grid <= 0: resident maximum) as its programmatic dependent. The first run on a device
 * builds a twiddle table and must not be inside a stream capture. */
SP_API int sp_batch_run(const void* desc_dev, void* ws, int grid, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* B200SIGNAL_H */
