// Fused inverse STFT: per-frame inverse real FFT, synthesis window, overlap-add and the
// window-energy normalisation in one pass (power-of-two nperseg == nfft, one-sided input).
//
// Reference behaviour replaced: _stft_metal.istft_frames (src/mlx_signal_processing/
// _stft_metal.py:851-887) -- kernel _ISTFT_SRC (:753-795) writes windowed frames to device
// memory, then _OLA_SRC (:797-820) re-reads them to gather the overlap-add -- plus the norm
// division of spectral.istft (spectral.py:929-943, 982). Differences by design:
//  * two consecutive frames share one complex inverse FFT: with X_s, X_{s+1} extended
//    Hermitian-symmetrically, IFFT(X_s + i X_{s+1}) = x_s + i x_{s+1} (both real);
//  * each team owns a contiguous output range and accumulates the overlap-add in a
//    shared-memory ring buffer, recomputing the few halo frames that reach into its range from
//    the left, so every output sample is summed in a fixed order by one team (deterministic,
//    no second pass over HBM);
//  * the normalisation sum_s win^2[t - s hop] comes from a per-CTA periodic table in the
//    interior and is summed directly near the row ends; samples with norm <= 1e-10 are not
//    divided (scipy's rule).
#pragma once

#include "fft_core.cuh"
#include "mean_kernels.cuh"
#include "team_util.cuh"

namespace b2s {

struct IstftParams {
  const float2* z;   // (rows, nseg, ldf) complex64 one-sided spectra, bins k < nbins_in valid
  int64_t ld_row;    // complex elements between rows
  int ldf;           // complex elements between frames
  int nbins_in;      // valid bins per frame (missing bins up to L/2 are zero)
  int64_t rows;
  int nseg;
  int hop;
  const float* win;  // nper window values
  float scale;       // istft scale (spectrum: sum(win); psd: sqrt(fs sum(win^2)))
  int nper;          // frame length (nperseg <= L): the first nper samples of each inverse FFT
  int nfft;          // DFT length of the chirp-z (non-power-of-two) kernel; L for the others
  int64_t outlen;    // nper + (nseg - 1) * hop
  float* out;        // (rows, outlen)
  int64_t G;         // output frames owned per team
  int64_t total;     // rows * nseg
};

template <int LOG_L, int LOG_E>
struct IstftCfg {
  using PL = Plan<LOG_L, LOG_E>;
  static constexpr int TEAMS = PL::P >= 64 ? 1 : 128 / PL::P;
  static constexpr int THREADS = TEAMS * PL::P;
  static constexpr int SCRATCH = PL::P >= 64 ? PL::P / 32 : 1;
  static constexpr int WIN = (PL::L + 3) & ~3;
  // ring of >= 2L floats per team: holds [s*hop, (s+1)*hop + L) for any hop <= L
  static constexpr int RING = 2 * PL::L;
  static constexpr size_t SMEM = size_t(TEAMS) * SCRATCH * 16 + size_t(WIN) * 4 * 2 +
                                 size_t(PL::TW) * 8 + size_t(TEAMS) * PL::BUF * 8 +
                                 size_t(TEAMS) * RING * 4;
};

template <int LOG_L, int LOG_E>
__global__ void __launch_bounds__(IstftCfg<LOG_L, LOG_E>::THREADS) k_istft(IstftParams pr) {
  using CFG = IstftCfg<LOG_L, LOG_E>;
  using PL = typename CFG::PL;
  constexpr int L = PL::L, E = PL::E, P = PL::P, RING = CFG::RING;
  extern __shared__ float4 smem[];
  float* weff = reinterpret_cast<float*>(smem + CFG::TEAMS * CFG::SCRATCH);  // win*scale/L
  float* normp = weff + CFG::WIN;  // periodic window-energy table, index o mod hop
  float2* tw = reinterpret_cast<float2*>(normp + CFG::WIN);
  float2* sbuf = tw + PL::TW;
  float* rings = reinterpret_cast<float*>(sbuf + CFG::TEAMS * PL::BUF);
  const int hop = pr.hop;
  const int N = pr.nper;  // frame length; samples N .. L-1 of each inverse FFT are dropped
  const float fs = pr.scale / float(L);
  for (int i = threadIdx.x; i < L; i += blockDim.x) weff[i] = i < N ? pr.win[i] * fs : 0.f;
  for (int r = threadIdx.x; r < hop; r += blockDim.x) {
    float s = 0.f;
    for (int n = r; n < N; n += hop) s = fmaf(pr.win[n], pr.win[n], s);
    normp[r] = s;
  }
  build_twiddles<PL>(tw, threadIdx.x, blockDim.x);
  __syncthreads();
  const int team = threadIdx.x / P, t = threadIdx.x - team * P;
  const unsigned mask = team_mask<P>();
  float2* buf = sbuf + team * PL::BUF;
  float* ring = rings + team * RING;
  for (int i = t; i < RING; i += P) ring[i] = 0.f;
  team_sync<P>(mask);
  const int64_t tau = int64_t(blockIdx.x) * CFG::TEAMS + team;
  int64_t g = tau * pr.G;
  const int64_t gend = min(g + pr.G, pr.total);
  const int halo = (N + hop - 1) / hop - 1;  // frames starting left of a range that reach into it
  while (g < gend) {
    const int64_t r = g / pr.nseg;
    const int f0 = int(g - r * pr.nseg);
    const int64_t lim = int64_t(f0) + (gend - g);
    const int f1 = int(lim < pr.nseg ? lim : int64_t(pr.nseg));
    // owned output samples: [f0*hop, f1*hop), the last range of a row extends to outlen
    const int64_t own_lo = int64_t(f0) * hop;
    const int64_t own_hi = f1 == pr.nseg ? pr.outlen : int64_t(f1) * hop;
    const int sa = f0 - halo > 0 ? f0 - halo : 0;
    const float2* zr = pr.z + r * pr.ld_row;
    float* orow = pr.out + r * pr.outlen;
    int64_t done = int64_t(sa) * hop;  // samples below this are final (and already written)
    for (int s = sa; s < f1; s += 2) {
      const bool two = s + 1 < f1;
      const float2* za = zr + int64_t(s) * pr.ldf;
      const float2* zb = za + pr.ldf;
      float2 v[E];
      // conj of the Hermitian-extended pair spectrum Z = X_s + i X_{s+1}, DC/Nyquist real
      static_for<0, E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        const int k = slot_elem<PL, e>(t);
        const bool upper = k > L / 2;
        const int kk = upper ? L - k : k;
        float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
        if (kk < pr.nbins_in) {
          a = za[kk];
          if (two) b = zb[kk];
        }
        if (kk == 0 || 2 * kk == L) {
          a.y = 0.f;
          b.y = 0.f;
        }
        if (upper) {
          a.y = -a.y;
          b.y = -b.y;
        }
        // Z = a + i b ; conj(Z) = (a.x - b.y, -(a.y + b.x))
        v[e] = make_float2(a.x - b.y, -(a.y + b.x));
      });
      team_pass0<PL>(v);
      team_passes<PL>(v, buf, tw, t, mask);
      // x_s[n] = Re(v)/L, x_{s+1}[n] = -Im(v)/L (1/L folded into weff); overlap-add in two
      // phases so no ring slot is written by two lanes at once
      const int64_t pa = int64_t(s) * hop;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int n = t + e * P;
        ring[(pa + n) & (RING - 1)] += v[e].x * weff[n];
      }
      team_sync<P>(mask);
      if (two) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int n = t + e * P;
          ring[(pa + hop + n) & (RING - 1)] -= v[e].y * weff[n];
        }
      }
      team_sync<P>(mask);
      // final samples: below the start of the next unprocessed frame (or everything at the end)
      const bool last = s + 2 >= f1;
      const int64_t fin = last ? own_hi : int64_t(s + 2) * hop;
      int res = int((done + t) % hop);  // (o mod hop), advanced incrementally
      const int pstep = P % hop;
      for (int64_t o = done + t; o < fin; o += P) {
        const int slot = int(o & (RING - 1));
        if (o >= own_lo) {
          float nrm;
          if (o >= N - hop && o < int64_t(pr.nseg) * hop) {
            nrm = normp[res];
          } else {
            nrm = 0.f;
            int64_t slo = o - N + 1 > 0 ? (o - N + 1 + hop - 1) / hop : 0;
            int64_t shi = o / hop;
            if (shi > pr.nseg - 1) shi = pr.nseg - 1;
            for (int64_t q = slo; q <= shi; ++q) {
              const float w = pr.win[o - q * hop];
              nrm = fmaf(w, w, nrm);
            }
          }
          const float val = ring[slot];
          orow[o] = val / (nrm > 1e-10f ? nrm : 1.0f);
        }
        ring[slot] = 0.f;
        res += pstep;
        if (res >= hop) res -= hop;
      }
      done = fin;
      team_sync<P>(mask);
    }
    // partial sums past own_hi belong to the next team's range: clear the ring for the next range
    for (int i = t; i < RING; i += P) ring[i] = 0.f;
    team_sync<P>(mask);
    g += f1 - f0;
  }
}

// Two-sided inverse STFT (input_onesided=False): each frame is its own complex inverse FFT of
// length L, x_s = IFFT_L(Z_s)[0 : nper] (complex), windowed and overlap-added into a complex
// shared-memory ring with the window-energy normalisation of k_istft; the output is complex64
// (scipy's istft returns the complex result for two-sided input). Inverse by conjugation:
// IFFT(Z) = conj(FFT(conj Z)) / L, the 1/L folded into the window table.
template <int LOG_L, int LOG_E>
struct IstftCplxCfg {
  using PL = Plan<LOG_L, LOG_E>;
  static constexpr int TEAMS = PL::P >= 64 ? 1 : 128 / PL::P;
  static constexpr int THREADS = TEAMS * PL::P;
  static constexpr int SCRATCH = PL::P >= 64 ? PL::P / 32 : 1;
  static constexpr int WIN = (PL::L + 3) & ~3;
  static constexpr int RING = 2 * PL::L;  // complex samples: [s*hop, s*hop + nper) for hop <= L
  static constexpr size_t SMEM = size_t(TEAMS) * SCRATCH * 16 + size_t(WIN) * 4 * 2 +
                                 size_t(PL::TW) * 8 + size_t(TEAMS) * PL::BUF * 8 +
                                 size_t(TEAMS) * RING * 8;
};

template <int LOG_L, int LOG_E>
__global__ void __launch_bounds__(IstftCplxCfg<LOG_L, LOG_E>::THREADS)
    k_istft_cplx(IstftParams pr) {
  using CFG = IstftCplxCfg<LOG_L, LOG_E>;
  using PL = typename CFG::PL;
  constexpr int L = PL::L, E = PL::E, P = PL::P, RING = CFG::RING;
  extern __shared__ float4 smem[];
  float* weff = reinterpret_cast<float*>(smem + CFG::TEAMS * CFG::SCRATCH);  // win*scale/L
  float* normp = weff + CFG::WIN;  // periodic window-energy table, index o mod hop
  float2* tw = reinterpret_cast<float2*>(normp + CFG::WIN);
  float2* sbuf = tw + PL::TW;
  float2* rings = sbuf + CFG::TEAMS * PL::BUF;
  const int hop = pr.hop;
  const int N = pr.nper;
  const float fs = pr.scale / float(L);
  for (int i = threadIdx.x; i < L; i += blockDim.x) weff[i] = i < N ? pr.win[i] * fs : 0.f;
  for (int r = threadIdx.x; r < hop; r += blockDim.x) {
    float s = 0.f;
    for (int n = r; n < N; n += hop) s = fmaf(pr.win[n], pr.win[n], s);
    normp[r] = s;
  }
  build_twiddles<PL>(tw, threadIdx.x, blockDim.x);
  __syncthreads();
  const int team = threadIdx.x / P, t = threadIdx.x - team * P;
  const unsigned mask = team_mask<P>();
  float2* buf = sbuf + team * PL::BUF;
  float2* ring = rings + team * RING;
  for (int i = t; i < RING; i += P) ring[i] = make_float2(0.f, 0.f);
  team_sync<P>(mask);
  const int64_t tau = int64_t(blockIdx.x) * CFG::TEAMS + team;
  int64_t g = tau * pr.G;
  const int64_t gend = min(g + pr.G, pr.total);
  const int halo = (N + hop - 1) / hop - 1;
  float2* out = reinterpret_cast<float2*>(pr.out);
  while (g < gend) {
    const int64_t r = g / pr.nseg;
    const int f0 = int(g - r * pr.nseg);
    const int64_t lim = int64_t(f0) + (gend - g);
    const int f1 = int(lim < pr.nseg ? lim : int64_t(pr.nseg));
    const int64_t own_lo = int64_t(f0) * hop;
    const int64_t own_hi = f1 == pr.nseg ? pr.outlen : int64_t(f1) * hop;
    const int sa = f0 - halo > 0 ? f0 - halo : 0;
    const float2* zr = pr.z + r * pr.ld_row;
    float2* orow = out + r * pr.outlen;
    int64_t done = int64_t(sa) * hop;
    for (int s = sa; s < f1; ++s) {
      const float2* za = zr + int64_t(s) * pr.ldf;
      float2 v[E];
      static_for<0, E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        const int k = slot_elem<PL, e>(t);
        const float2 a = k < pr.nbins_in ? za[k] : make_float2(0.f, 0.f);
        v[e] = make_float2(a.x, -a.y);  // conj
      });
      team_pass0<PL>(v);
      team_passes<PL>(v, buf, tw, t, mask);
      // x_s[n] = conj(v[n]) / L, the 1/L in weff
      const int64_t pa = int64_t(s) * hop;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int n = t + e * P;
        float2& q = ring[(pa + n) & (RING - 1)];
        q.x = fmaf(v[e].x, weff[n], q.x);
        q.y = fmaf(-v[e].y, weff[n], q.y);
      }
      team_sync<P>(mask);
      const bool last = s + 1 >= f1;
      const int64_t fin = last ? own_hi : int64_t(s + 1) * hop;
      int res = int((done + t) % hop);
      const int pstep = P % hop;
      for (int64_t o = done + t; o < fin; o += P) {
        const int slot = int(o & (RING - 1));
        if (o >= own_lo) {
          float nrm;
          if (o >= N - hop && o < int64_t(pr.nseg) * hop) {
            nrm = normp[res];
          } else {
            nrm = 0.f;
            int64_t slo = o - N + 1 > 0 ? (o - N + 1 + hop - 1) / hop : 0;
            int64_t shi = o / hop;
            if (shi > pr.nseg - 1) shi = pr.nseg - 1;
            for (int64_t q = slo; q <= shi; ++q) {
              const float w = pr.win[o - q * hop];
              nrm = fmaf(w, w, nrm);
            }
          }
          const float2 val = ring[slot];
          const float d = nrm > 1e-10f ? nrm : 1.0f;
          orow[o] = make_float2(val.x / d, val.y / d);
        }
        ring[slot] = make_float2(0.f, 0.f);
        res += pstep;
        if (res >= hop) res -= hop;
      }
      done = fin;
      team_sync<P>(mask);
    }
    for (int i = t; i < RING; i += P) ring[i] = make_float2(0.f, 0.f);
    team_sync<P>(mask);
    g += f1 - f0;
  }
}

// Half-overlap inverse STFT (hop == L/2, scipy's default noverlap): the overlap-add needs no
// shared-memory ring. With H = L/2 and output block j = [jH, (j+1)H), block j receives the second
// half of frame j-1 and the first half of frame j. After the pair IFFT of frames (s, s+1) a
// thread holds sample n = t + e*P of both frames in v[e] (re: frame s, -im: frame s+1), and
// e < E/2 <=> n < H, so
//     block s   = carry           + x_s[n]       (n < H)
//     block s+1 = x_s[n + H]      + x_{s+1}[n]
//     carry'    = x_{s+1}[n + H]
// all in registers, stored coalesced. A team owns a contiguous frame range [f0, f1) and writes
// blocks f0 .. f1-1 (and block nseg, the lone second half of the last frame, when f1 == nseg);
// it first recomputes frame f0-1 alone for its carry. Interior blocks divide by the periodic
// window energy w^2[n] + w^2[n+H] (a reciprocal table); blocks 0 and nseg use w^2[n] and
// w^2[n+H]; samples whose energy is <= 1e-10 are not divided (scipy's rule).
template <int LOG_L, int LOG_E>
struct IstftHalfCfg {
  using PL = Plan<LOG_L, LOG_E>;
  static constexpr int TEAMS = PL::P >= 64 ? 1 : 128 / PL::P;
  static constexpr int THREADS = TEAMS * PL::P;
  static constexpr int H = PL::L / 2 > 0 ? PL::L / 2 : 1;
  // per-team staging of one frame pair's one-sided spectra (bins 0..L/2), filled by cp.async
  static constexpr int NBP = PL::L / 2 + 2;
  static constexpr int STAGE = 2 * NBP;
  // float tables (window, three norm tables) rounded to 16 bytes so the complex arrays after
  // them stay 8-byte aligned (at L = 2 the tables are 5 floats)
  static constexpr int FLT = (PL::L + 3 * H + 3) & ~3;
  static constexpr size_t SMEM = size_t(FLT) * 4 + size_t(PL::TW) * 8 +
                                 size_t(TEAMS) * PL::BUF * 8 + size_t(TEAMS) * STAGE * 8;
};

__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(
                   static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst))),
               "l"(gsrc)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

template <class PL>
__device__ __forceinline__ void istft_load_pair(float2 (&v)[PL::E], const float2* za,
                                                const float2* zb, bool two, int nbins_in, int t) {
  constexpr int L = PL::L;
  // conj of the Hermitian-extended pair spectrum Z = X_s + i X_{s+1}, DC/Nyquist real
  static_for<0, PL::E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    const int k = slot_elem<PL, e>(t);
    const bool upper = k > L / 2;
    const int kk = upper ? L - k : k;
    float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
    if (kk < nbins_in) {
      a = __ldg(za + kk);
      if (two) b = __ldg(zb + kk);
    }
    if (kk == 0 || 2 * kk == L) {
      a.y = 0.f;
      b.y = 0.f;
    }
    if (upper) {
      a.y = -a.y;
      b.y = -b.y;
    }
    v[e] = make_float2(a.x - b.y, -(a.y + b.x));
  });
}

// istft_load_pair from a staged pair (sa, sb: one-sided bins of frames s, s+1 in shared memory)
template <class PL>
__device__ __forceinline__ void istft_stage_pair(float2 (&v)[PL::E], const float2* sa,
                                                 const float2* sb, bool two, int nbins_in, int t) {
  constexpr int L = PL::L;
  static_for<0, PL::E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    const int k = slot_elem<PL, e>(t);
    const bool upper = k > L / 2;
    const int kk = upper ? L - k : k;
    float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
    if (kk < nbins_in) {
      a = sa[kk];
      if (two) b = sb[kk];
    }
    if (kk == 0 || 2 * kk == L) {
      a.y = 0.f;
      b.y = 0.f;
    }
    if (upper) {
      a.y = -a.y;
      b.y = -b.y;
    }
    v[e] = make_float2(a.x - b.y, -(a.y + b.x));
  });
}

template <int LOG_L, int LOG_E>
__global__ void __launch_bounds__(IstftHalfCfg<LOG_L, LOG_E>::THREADS)
    k_istft_half(IstftParams pr) {
  using CFG = IstftHalfCfg<LOG_L, LOG_E>;
  using PL = typename CFG::PL;
  constexpr int L = PL::L, E = PL::E, P = PL::P, H = CFG::H, EH = E / 2;
  static_assert(E >= 2, "half-overlap istft needs at least two points per thread");
  extern __shared__ float4 smem[];
  float* weff = reinterpret_cast<float*>(smem);  // win * scale / L
  float* inv_mid = weff + L;                     // 1 / (w^2[n] + w^2[n+H]) or 1
  float* inv_first = inv_mid + H;                // 1 / w^2[n]      (block 0)
  float* inv_last = inv_first + H;               // 1 / w^2[n + H]  (block nseg)
  float2* tw = reinterpret_cast<float2*>(weff + CFG::FLT);
  float2* sbuf = tw + PL::TW;
  float2* stage_all = sbuf + CFG::TEAMS * PL::BUF;
  const float fs = pr.scale / float(L);
  for (int i = threadIdx.x; i < L; i += blockDim.x) weff[i] = pr.win[i] * fs;
  for (int i = threadIdx.x; i < H; i += blockDim.x) {
    const float a = pr.win[i], b = pr.win[i + H];
    const float m = fmaf(a, a, b * b), f = a * a, l = b * b;
    inv_mid[i] = m > 1e-10f ? 1.0f / m : 1.0f;
    inv_first[i] = f > 1e-10f ? 1.0f / f : 1.0f;
    inv_last[i] = l > 1e-10f ? 1.0f / l : 1.0f;
  }
  build_twiddles<PL>(tw, threadIdx.x, blockDim.x);
  __syncthreads();
  const int team = threadIdx.x / P, t = threadIdx.x - team * P;
  const unsigned mask = team_mask<P>();
  float2* buf = sbuf + team * PL::BUF;
  float2* stage = stage_all + team * CFG::STAGE;  // [frame s | frame s+1][NBP]
  const int nb_stage = pr.nbins_in < CFG::NBP ? pr.nbins_in : CFG::NBP;
  const int64_t tau = int64_t(blockIdx.x) * CFG::TEAMS + team;
  int64_t g = tau * pr.G;
  const int64_t gend = min(g + pr.G, pr.total);
  while (g < gend) {
    const int64_t r = g / pr.nseg;
    const int f0 = int(g - r * pr.nseg);
    const int64_t lim = int64_t(f0) + (gend - g);
    const int f1 = int(lim < pr.nseg ? lim : int64_t(pr.nseg));
    const float2* zr = pr.z + r * pr.ld_row;
    float* orow = pr.out + r * pr.outlen;
    float carry[EH];
#pragma unroll
    for (int e = 0; e < EH; ++e) carry[e] = 0.f;
    if (f0 > 0) {  // second half of frame f0-1
      float2 v[E];
      istft_load_pair<PL>(v, zr + int64_t(f0 - 1) * pr.ldf, nullptr, false, pr.nbins_in, t);
      team_pass0<PL>(v);
      team_passes<PL>(v, buf, tw, t, mask);
#pragma unroll
      for (int e = 0; e < EH; ++e) carry[e] = v[e + EH].x * weff[t + e * P + H];
      team_sync<P>(mask);
    }
    // the pair's one-sided spectra are copied into the team's stage asynchronously (each bin
    // once, coalesced), one pair ahead of the transform that reads them
    auto issue = [&](int s) {
      const float2* za = zr + int64_t(s) * pr.ldf;
      const bool two = s + 1 < f1;
      for (int i = t; i < nb_stage; i += P) {
        cp_async8(stage + i, za + i);
        if (two) cp_async8(stage + CFG::NBP + i, za + pr.ldf + i);
      }
      cp_async_commit();
    };
    if (f0 < f1) issue(f0);
    for (int s = f0; s < f1; s += 2) {
      const bool two = s + 1 < f1;
      const float2* za = zr + int64_t(s) * pr.ldf;
      if (s + 5 < f1) {  // warm L2 with the pair after the one being staged next
        const char* nx = reinterpret_cast<const char*>(za + 4 * int64_t(pr.ldf));
        const int bytes = 2 * pr.ldf * 8;
        for (int o = t * 128; o < bytes; o += P * 128)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(nx + o));
      }
      cp_async_wait_all();
      team_sync<P>(mask);
      float2 v[E];
      istft_stage_pair<PL>(v, stage, stage + CFG::NBP, two, nb_stage, t);
      team_sync<P>(mask);  // every lane has read the stage: the next pair may overwrite it
      if (s + 2 < f1) issue(s + 2);
      team_pass0<PL>(v);
      team_passes<PL>(v, buf, tw, t, mask);
      float* ob = orow + int64_t(s) * H;
      const float* inv0 = s == 0 ? inv_first : inv_mid;
#pragma unroll
      for (int e = 0; e < EH; ++e) {
        const int n = t + e * P;
        ob[n] = fmaf(v[e].x, weff[n], carry[e]) * inv0[n];
      }
      if (two) {
        const float* inv1 = inv_mid;  // block s+1 <= nseg-1 is interior
#pragma unroll
        for (int e = 0; e < EH; ++e) {
          const int n = t + e * P;
          const float val = fmaf(v[e + EH].x, weff[n + H], -v[e].y * weff[n]);
          ob[H + n] = val * inv1[n];
          carry[e] = -v[e + EH].y * weff[n + H];
        }
      } else {
#pragma unroll
        for (int e = 0; e < EH; ++e) carry[e] = v[e + EH].x * weff[t + e * P + H];
      }
      team_sync<P>(mask);
    }
    if (f1 == pr.nseg) {  // block nseg: the lone second half of the last frame
      float* ob = orow + int64_t(pr.nseg) * H;
#pragma unroll
      for (int e = 0; e < EH; ++e) {
        const int n = t + e * P;
        ob[n] = carry[e] * inv_last[n];
      }
    }
    g += f1 - f0;
  }
}

}  // namespace b2s
