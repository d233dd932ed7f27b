// C-ABI: fused inverse STFT (inverse rfft + window + overlap-add + normalisation).
#include "capi_common.h"
#include "dispatch.cuh"

extern "C" {

int sp_istft_f32_ex(const float* z, int64_t rows, int nseg, int64_t ld_row, int ldf,
                    int nbins_in, const float* win, float scale, int nperseg, int nfft, int hop,
                    float* out, void* stream) {
  using namespace b2s;
  if (!z || !win || !out || rows < 0 || nseg < 1 || nperseg < 1 || nfft < nperseg || nfft < 2 ||
      hop < 1 || hop > nperseg || nbins_in < 1 || ldf < nbins_in ||
      ld_row < int64_t(nseg) * ldf) {
    set_error("invalid istft arguments (nseg=%d nperseg=%d nfft=%d hop=%d nbins=%d ldf=%d)",
              nseg, nperseg, nfft, hop, nbins_in, ldf);
    return SP_ERR_ARG;
  }
  int log_l = ilog2_exact(nfft);
  // a non-power-of-two nfft: the chirp-z kernel on a power-of-two transform
  const bool blue = log_l < 0 && nfft >= 3 && nfft <= kBlueIstftMaxN;
  if (!blue && (log_l < 1 || log_l > kMaxLogL)) {
    set_error("nfft=%d: the fused istft needs a power of two in [2, %d] or any nfft in [3, %d]",
              nfft, 1 << kMaxLogL, kBlueIstftMaxN);
    return SP_ERR_UNSUPPORTED;
  }
  if (rows == 0) return SP_OK;
  // register overlap-add (no ring buffer) for whole-length frames at half overlap
  const bool half = !blue && nperseg == nfft && 2 * hop == nperseg;
  const IstftInfo k = blue ? istft_blue_lookup(blue_log_m(nfft))
                           : (half ? istft_half_lookup(log_l) : istft_lookup(log_l));
  int sms = 0;
  const int nb = resident_ctas(k.fn, k.threads, k.smem, &sms);
  if (nb <= 0) {
    set_error("no resident CTA for the istft kernel (nperseg=%d)", nperseg);
    return SP_ERR_UNSUPPORTED;
  }
  IstftParams p;
  p.z = reinterpret_cast<const float2*>(z);
  p.ld_row = ld_row;
  p.ldf = ldf;
  p.nbins_in = nbins_in;
  p.rows = rows;
  p.nseg = nseg;
  p.hop = hop;
  p.win = win;
  p.scale = scale;
  p.nper = nperseg;
  p.nfft = nfft;
  p.outlen = int64_t(nperseg) + int64_t(nseg - 1) * hop;
  p.out = out;
  p.total = rows * nseg;
  const int64_t cap = int64_t(nb) * sms * k.teams;
  // at least a few frames per team so the recomputed halo frames stay a small overhead
  const int halo = (nperseg + hop - 1) / hop - 1;
  int64_t G = cdiv(p.total, cap);
  if (half) {
    // one recomputed frame per team range: keep ranges >= 16 frames, whole pairs
    if (G < 16) G = 16;
    G += G & 1;
  } else if (G < 4 * (halo + 1)) {
    G = 4 * (halo + 1);
  }
  p.G = G;
  const int64_t nteams = cdiv(p.total, G);
  const int64_t blocks = cdiv(nteams, k.teams);
  k.launch(dim3(unsigned(blocks)), k.threads, k.smem, static_cast<cudaStream_t>(stream), p);
  B2S_CHECK_CUDA(cudaGetLastError(), "istft kernel launch");
  return SP_OK;
}

int sp_istft_c64(const float* z, int64_t rows, int nseg, int64_t ld_row, int ldf, int nbins_in,
                 const float* win, float scale, int nperseg, int nfft, int hop, float* out,
                 void* stream) {
  using namespace b2s;
  if (!z || !win || !out || rows < 0 || nseg < 1 || nperseg < 1 || nfft < nperseg || nfft < 2 ||
      hop < 1 || hop > nperseg || nbins_in < 1 || ldf < nbins_in ||
      ld_row < int64_t(nseg) * ldf) {
    set_error("invalid istft arguments (nseg=%d nperseg=%d nfft=%d hop=%d nbins=%d ldf=%d)",
              nseg, nperseg, nfft, hop, nbins_in, ldf);
    return SP_ERR_ARG;
  }
  const int log_l = ilog2_exact(nfft);
  if (log_l < 1 || log_l > kMaxLogL) {
    set_error("nfft=%d: the fused istft needs a power of two in [2, %d]", nfft, 1 << kMaxLogL);
    return SP_ERR_UNSUPPORTED;
  }
  if (rows == 0) return SP_OK;
  const IstftInfo k = istft_cplx_lookup(log_l);
  int sms = 0;
  const int nb = resident_ctas(k.fn, k.threads, k.smem, &sms);
  if (nb <= 0) {
    set_error("no resident CTA for the complex istft kernel (nfft=%d)", nfft);
    return SP_ERR_UNSUPPORTED;
  }
  IstftParams p;
  p.z = reinterpret_cast<const float2*>(z);
  p.ld_row = ld_row;
  p.ldf = ldf;
  p.nbins_in = nbins_in;
  p.rows = rows;
  p.nseg = nseg;
  p.hop = hop;
  p.win = win;
  p.scale = scale;
  p.nper = nperseg;
  p.nfft = nfft;
  p.outlen = int64_t(nperseg) + int64_t(nseg - 1) * hop;
  p.out = out;
  p.total = rows * nseg;
  const int64_t cap = int64_t(nb) * sms * k.teams;
  const int halo = (nperseg + hop - 1) / hop - 1;
  int64_t G = cdiv(p.total, cap);
  if (G < 4 * (halo + 1)) G = 4 * (halo + 1);
  p.G = G;
  const int64_t blocks = cdiv(cdiv(p.total, G), k.teams);
  k.launch(dim3(unsigned(blocks)), k.threads, k.smem, static_cast<cudaStream_t>(stream), p);
  B2S_CHECK_CUDA(cudaGetLastError(), "complex istft kernel launch");
  return SP_OK;
}

int sp_istft_f32(const float* z, int64_t rows, int nseg, int64_t ld_row, int ldf, int nbins_in,
                 const float* win, float scale, int nperseg, int hop, float* out, void* stream) {
  return sp_istft_f32_ex(z, rows, nseg, ld_row, ldf, nbins_in, win, scale, nperseg, nperseg, hop,
                         out, stream);
}

}
