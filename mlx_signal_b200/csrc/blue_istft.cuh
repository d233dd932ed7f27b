// Fused inverse STFT for a non-power-of-two nfft (one-sided input): each frame pair's inverse
// DFT of length N = nfft through the chirp-z (Bluestein) engine, then window, overlap-add and
// window-energy normalisation as in k_istft.
//
// With Z = X_s + i X_{s+1} (both spectra extended Hermitian-symmetrically to N bins, DC and, for
// even N, the Nyquist bin taken as real), IDFT_N(Z) = x_s + i x_{s+1} (both frames real), and
//   IDFT_N(Z)_n = conj(DFT_N(conj Z)_n) / N,
//   DFT_N(a)_n = d_n conj(V_n),  V = blue_core(a_k e^{-i pi k^2/N}),  d_n = e^{-i pi n^2/N},
// so x_n = conj(d_n) V_n / N (the 1/N folded into the window table). Frames are the first
// nper <= N samples; the overlap-add ring and the normalisation follow k_istft.
//
// Reference behaviour replaced: the composed branch of spectral.istft (spectral.py:929-950:
// irfft of length nfft on the MLX FFT, window, scatter overlap-add) for nfft that the fused
// power-of-two kernel of the reference does not take (_stft_metal.eligible_istft, :823-827).
#pragma once

#include "blue_kernels.cuh"
#include "istft_kernels.cuh"

namespace b2s {

template <int LOG_M>
struct BlueIstftCfg {
  using PL = Plan<LOG_M, 4>;
  static constexpr int M = PL::L;
  static constexpr int NMAX = M / 2;  // N <= (M + 1) / 2
  static constexpr int TEAMS = PL::P >= 64 ? 1 : 128 / PL::P;
  static constexpr int THREADS = TEAMS * PL::P;
  static constexpr int SCRATCH = PL::P >= 64 ? PL::P / 32 : 1;
  static constexpr int RING = M;      // >= hop + nper for hop <= nper <= N, M >= 2N
  static constexpr size_t SMEM = size_t(TEAMS) * SCRATCH * 16 + size_t(PL::TW) * 8 +
                                 size_t(TEAMS) * PL::BUF * 8 + size_t(2 * NMAX) * 8 +
                                 size_t(2 * NMAX) * 4 + size_t(TEAMS) * RING * 4;
};

template <int LOG_M>
__global__ void __launch_bounds__(BlueIstftCfg<LOG_M>::THREADS) k_blue_istft(IstftParams pr) {
  using CFG = BlueIstftCfg<LOG_M>;
  using PL = typename CFG::PL;
  constexpr int E = PL::E, P = PL::P, RING = CFG::RING;
  extern __shared__ float4 smem[];
  float2* tw = reinterpret_cast<float2*>(smem + CFG::TEAMS * CFG::SCRATCH);
  float2* sbuf = tw + PL::TW;
  float2* cin = sbuf + CFG::TEAMS * PL::BUF;  // e^{-i pi k^2/N}
  float2* cdn = cin + CFG::NMAX;               // conj(d_n) = e^{+i pi n^2/N}
  float* weff = reinterpret_cast<float*>(cdn + CFG::NMAX);  // win * scale / N, zero past nper
  float* normp = weff + CFG::NMAX;                          // periodic window energy (o mod hop)
  float* rings = normp + CFG::NMAX;
  const int N = pr.nfft, NP = pr.nper, hop = pr.hop;
  build_twiddles<PL>(tw, threadIdx.x, blockDim.x);
  const float fs = pr.scale / float(N);
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    cin[n] = chirp(n, N, -1.0);
    cdn[n] = chirp(n, N, 1.0);
    weff[n] = n < NP ? pr.win[n] * fs : 0.f;
  }
  for (int r = threadIdx.x; r < hop; r += blockDim.x) {
    float s = 0.f;
    for (int n = r; n < NP; n += hop) s = fmaf(pr.win[n], pr.win[n], s);
    normp[r] = s;
  }
  __syncthreads();
  const int team = threadIdx.x / P, t = threadIdx.x - team * P;
  const unsigned mask = team_mask<P>();
  float2* buf = sbuf + team * PL::BUF;
  float* ring = rings + team * RING;
  float2 bh[E];
  blue_filter<PL>(bh, N, buf, tw, t, mask);
  for (int i = t; i < RING; i += P) ring[i] = 0.f;
  team_sync<P>(mask);
  const int64_t tau = int64_t(blockIdx.x) * CFG::TEAMS + team;
  int64_t g = tau * pr.G;
  const int64_t gend = min(g + pr.G, pr.total);
  const int halo = (NP + hop - 1) / hop - 1;
  while (g < gend) {
    const int64_t r = g / pr.nseg;
    const int f0 = int(g - r * pr.nseg);
    const int64_t lim = int64_t(f0) + (gend - g);
    const int f1 = int(lim < pr.nseg ? lim : int64_t(pr.nseg));
    const int64_t own_lo = int64_t(f0) * hop;
    const int64_t own_hi = f1 == pr.nseg ? pr.outlen : int64_t(f1) * hop;
    const int sa = f0 - halo > 0 ? f0 - halo : 0;
    const float2* zr = pr.z + r * pr.ld_row;
    float* orow = pr.out + r * pr.outlen;
    int64_t done = int64_t(sa) * hop;
    for (int s = sa; s < f1; s += 2) {
      const bool two = s + 1 < f1;
      const float2* za = zr + int64_t(s) * pr.ldf;
      const float2* zb = za + pr.ldf;
      float2 v[E];
      // a_k = conj(Z_k) e^{-i pi k^2/N}, Z = X_s + i X_{s+1} Hermitian-extended, k < N
      static_for<0, E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        const int k = slot_elem<PL, e>(t);
        float2 val = make_float2(0.f, 0.f);
        if (k < N) {
          const bool upper = 2 * k > N;
          const int kk = upper ? N - k : k;
          float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
          if (kk < pr.nbins_in) {
            a = za[kk];
            if (two) b = zb[kk];
          }
          if (kk == 0 || 2 * kk == N) {
            a.y = 0.f;
            b.y = 0.f;
          }
          if (upper) {
            a.y = -a.y;
            b.y = -b.y;
          }
          val = cmul(make_float2(a.x - b.y, -(a.y + b.x)), cin[k]);
        }
        v[e] = val;
      });
      blue_core<PL>(v, bh, buf, tw, t, mask);
      // x_n = conj(d_n) V_n / N at n = t + e P (n < nper <= N <= M/2: registers e < E/2)
      const int64_t pa = int64_t(s) * hop;
      float2 xv[E / 2];
#pragma unroll
      for (int e = 0; e < E / 2; ++e) {
        const int n = t + e * P;
        xv[e] = n < NP ? cmul(cdn[n], v[e]) : make_float2(0.f, 0.f);
        if (n < NP) ring[(pa + n) & (RING - 1)] += xv[e].x * weff[n];
      }
      team_sync<P>(mask);
      if (two) {
#pragma unroll
        for (int e = 0; e < E / 2; ++e) {
          const int n = t + e * P;
          if (n < NP) ring[(pa + hop + n) & (RING - 1)] += xv[e].y * weff[n];
        }
      }
      team_sync<P>(mask);
      const bool last = s + 2 >= f1;
      const int64_t fin = last ? own_hi : int64_t(s + 2) * hop;
      int res = int((done + t) % hop);
      const int pstep = P % hop;
      for (int64_t o = done + t; o < fin; o += P) {
        const int slot = int(o & (RING - 1));
        if (o >= own_lo) {
          float nrm;
          if (o >= NP - hop && o < int64_t(pr.nseg) * hop) {
            nrm = normp[res];
          } else {
            nrm = 0.f;
            int64_t slo = o - NP + 1 > 0 ? (o - NP + 1 + hop - 1) / hop : 0;
            int64_t shi = o / hop;
            if (shi > pr.nseg - 1) shi = pr.nseg - 1;
            for (int64_t q = slo; q <= shi; ++q) {
              const float w = pr.win[o - q * hop];
              nrm = fmaf(w, w, nrm);
            }
          }
          orow[o] = ring[slot] / (nrm > 1e-10f ? nrm : 1.0f);
        }
        ring[slot] = 0.f;
        res += pstep;
        if (res >= hop) res -= hop;
      }
      done = fin;
      team_sync<P>(mask);
    }
    for (int i = t; i < RING; i += P) ring[i] = 0.f;
    team_sync<P>(mask);
    g += f1 - f0;
  }
}

}  // namespace b2s
