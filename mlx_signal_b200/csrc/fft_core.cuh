// Register/shared-memory FFT engine for the framed-spectral kernels (sm_100a).
//
// A length-L complex FFT is computed by a "team" of P = L/E threads, each holding E complex
// points in registers. The transform is a Stockham autosort factorisation (the public
// formulation of Govindaraju et al., "High performance discrete Fourier transforms on graphics
// processors", SC'08): every pass performs radix-R DFTs entirely in registers, multiplies by the
// inter-pass twiddles read from a shared-memory table, and exchanges data through a padded
// shared-memory buffer. Only one exchange is needed for L = E*E (e.g. 1024 = 32 x 32).
//
// Numerics: every twiddle is generated in FP64 and rounded to FP32 exactly once -- register DFT
// constants at compile time (constexpr Taylor series on an exactly reduced dyadic angle), table
// twiddles at kernel start with sincospi() in double. Radix-2 butterflies use the
// cosine-normalised FMA form (a +/- s*(c + i*tn*c)), six FMAs per twiddled butterfly. (Packed
// .f32x2 adds/FMAs were measured slower here than scalar FP32 for these butterflies.)
//
// This replaces the radix-2 threadgroup Stockham of the reference
// (src/mlx_signal_processing/_stft_metal.py:124-144, _PAIR_FFT :227-252), which runs log2(M)
// barrier-separated stages over threadgroup memory with twiddles read from a device table.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>

namespace b2s {

// ------------------------------------------------------------------------------------------
// compile-time helpers
// ------------------------------------------------------------------------------------------

template <int I, int N, typename F>
__device__ __forceinline__ void static_for(F&& f) {
  if constexpr (I < N) {
    f(std::integral_constant<int, I>{});
    static_for<I + 1, N>(f);
  }
}

constexpr int ilog2(int v) { return v <= 1 ? 0 : 1 + ilog2(v >> 1); }

constexpr int bitrev(int v, int bits) {
  int r = 0;
  for (int i = 0; i < bits; ++i) r |= ((v >> i) & 1) << (bits - 1 - i);
  return r;
}

constexpr double kPi = 3.141592653589793238462643383279502884;

constexpr double taylor_sin(double x) {
  double term = x, sum = x;
  for (int k = 1; k < 16; ++k) {
    term *= -x * x / double((2 * k) * (2 * k + 1));
    sum += term;
  }
  return sum;
}

constexpr double taylor_cos(double x) {
  double term = 1.0, sum = 1.0;
  for (int k = 1; k < 16; ++k) {
    term *= -x * x / double((2 * k - 1) * (2 * k));
    sum += term;
  }
  return sum;
}

struct CS {
  double c, s;
};

// (cos, sin) of 2*pi*f for a fraction of a turn f in [0, 1); the octant folding is exact for
// the dyadic fractions used here, so only the final Taylor evaluation (|x| <= pi/4) rounds.
constexpr CS turn_cs(double f) {
  if (f >= 0.5) {
    CS h = turn_cs(f - 0.5);
    return CS{-h.c, -h.s};
  }
  if (f >= 0.25) {
    CS h = turn_cs(f - 0.25);
    return CS{-h.s, h.c};
  }
  if (f > 0.125) {
    double g = 0.25 - f;
    double x = 2.0 * kPi * g;
    return CS{taylor_sin(x), taylor_cos(x)};
  }
  double x = 2.0 * kPi * f;
  return CS{taylor_cos(x), taylor_sin(x)};
}

// W_M^k = exp(-2*pi*i*k/M)
constexpr CS twiddle(long long k, long long M) {
  long long m = k % M;
  if (m < 0) m += M;
  CS v = turn_cs(double(m) / double(M));
  return CS{v.c, -v.s};
}

constexpr double dabs(double v) { return v < 0 ? -v : v; }

// ------------------------------------------------------------------------------------------
// complex arithmetic on float2 (x = re, y = im)
// ------------------------------------------------------------------------------------------

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float cnorm(float2 a) { return fmaf(a.x, a.x, a.y * a.y); }

// One radix-2 DIT butterfly with compile-time twiddle W_M^I:  (a, c) -> (a + w c, a - w c).
template <int I, int M>
__device__ __forceinline__ void bfly(float2& a, float2& c) {
  constexpr int i = I % M;
  if constexpr (i == 0) {
    const float2 t = a;
    a = cadd(t, c);
    c = csub(t, c);
  } else if constexpr (4 * i == M) {  // w = -i  ->  w c = (c.y, -c.x)
    const float ax = a.x, ay = a.y;
    a = make_float2(ax + c.y, ay - c.x);
    c = make_float2(ax - c.y, ay + c.x);
  } else if constexpr (4 * i == 3 * M) {  // w = +i  ->  w c = (-c.y, c.x)
    const float ax = a.x, ay = a.y;
    a = make_float2(ax - c.y, ay + c.x);
    c = make_float2(ax + c.y, ay - c.x);
  } else {
    constexpr CS w = twiddle(i, M);
    constexpr bool rmaj = dabs(w.c) >= dabs(w.s);
    constexpr float sc = float(rmaj ? w.c : w.s);
    constexpr float tn = float(rmaj ? w.s / w.c : w.c / w.s);
    float2 u;
    if constexpr (rmaj) {  // w = sc * (1 + i tn)
      u = make_float2(fmaf(-tn, c.y, c.x), fmaf(tn, c.x, c.y));
    } else {  // w = sc * (tn + i)
      u = make_float2(fmaf(tn, c.x, -c.y), fmaf(tn, c.y, c.x));
    }
    const float2 t = a;
    a = make_float2(fmaf(sc, u.x, t.x), fmaf(sc, u.y, t.y));
    c = make_float2(fmaf(-sc, u.x, t.x), fmaf(-sc, u.y, t.y));
  }
}

// In-place radix-2 DIT DFT of R points held at v[OFF .. OFF+R): input q must sit at
// v[OFF + bitrev(q)], output k ends at v[OFF + k] (natural order).
template <int R, int OFF, int H = 1, int N>
__device__ __forceinline__ void dft_dit(float2 (&v)[N]) {
  if constexpr (H < R) {
    static_for<0, R / (2 * H)>([&](auto gc) {
      constexpr int g = decltype(gc)::value * 2 * H;
      static_for<0, H>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        bfly<i, 2 * H>(v[OFF + g + i], v[OFF + g + i + H]);
      });
    });
    dft_dit<R, OFF, H * 2>(v);
  }
}

// ------------------------------------------------------------------------------------------
// Stockham team FFT
// ------------------------------------------------------------------------------------------

// Team FFT plan: L = 2^LOG_L complex points, E = 2^LOG_E per thread, P = L/E threads.
// Radix sequence: an optional first pass of radix RL = 2^(LOG_L mod LOG_E) (E/RL butterflies
// per thread, no twiddles), then passes of radix E (one butterfly per thread).
template <int LOG_L, int LOG_E>
struct Plan {
  static constexpr int L = 1 << LOG_L;
  static constexpr int E = 1 << LOG_E;
  static constexpr int P = L / E;
  static constexpr int LOG_RL = LOG_E ? LOG_L % LOG_E : 0;
  static constexpr int NFULL = LOG_E ? LOG_L / LOG_E : 1;
  static constexpr int NPASS = NFULL + (LOG_RL ? 1 : 0);
  static constexpr int radix(int p) { return (LOG_RL && p == 0) ? (1 << LOG_RL) : E; }
  static constexpr int span(int p) {  // product of radices before pass p
    int s = 1;
    for (int i = 0; i < p; ++i) s *= radix(i);
    return s;
  }
  // shared-memory padding: one complex every 2^PADSH keeps the strided Stockham writes and
  // the contiguous reads bank-conflict free for 8-byte elements. (Two complex per 2^PADSH,
  // which would allow 128-bit stores of the first exchange, measured slower.)
  static constexpr int PADSH = LOG_E < 4 ? 4 : LOG_E;
  static constexpr int BUF = L + (L >> PADSH);
  __host__ __device__ static constexpr int pad(int a) { return a + (a >> PADSH); }
  // twiddle table offsets: pass p >= 1 uses R_p * S_p entries W_{S R}^{k q} stored [q][k]
  static constexpr int tw_off(int p) {
    int o = 0;
    for (int i = 1; i < p; ++i) o += radix(i) * span(i);
    return o;
  }
  static constexpr int TW = tw_off(NPASS);
  // output bin held in register e after the last pass (radix E, span P): k = t + e*P
};

// Master table W_4096^j, j in [0, 4096): every inter-pass twiddle of a plan with L <= 4096 is one
// of its entries (W_N^m = W_4096^(m 4096/N)). Evaluated at compile time by the same FP64 series
// as the register constants and rounded to FP32 once, so a CTA fills its tables with a gather
// from L2 instead of evaluating FP64 sines per entry.
constexpr int kTwMasterLog = 12;
constexpr int kTwMasterN = 1 << kTwMasterLog;
struct TwMaster {
  float2 v[kTwMasterN];
};
constexpr TwMaster make_tw_master() {
  TwMaster t{};
  for (int j = 0; j < kTwMasterN; ++j) {
    const CS w = twiddle(j, kTwMasterN);
    t.v[j] = float2{float(w.c), float(w.s)};
  }
  return t;
}
static __device__ const TwMaster g_tw_master = make_tw_master();

// Fill the twiddle tables of a plan (all passes) into shared memory: passes whose twiddles are
// all entries of the master table gather them from it; a longer pass (L = 8192) evaluates its
// entries with FP64 sincospi of the exactly reduced integer phase, rounded to FP32 once.
template <class PL>
__device__ void build_twiddles(float2* tw, int tid, int nthreads) {
  static_for<1, PL::NPASS>([&](auto pc) {
    constexpr int p = decltype(pc)::value;
    constexpr int R = PL::radix(p), S = PL::span(p), SR = S * R;
    float2* t = tw + PL::tw_off(p);
    if constexpr (SR <= kTwMasterN) {
      constexpr int step = kTwMasterN / SR;
      for (int e = tid; e < R * S; e += nthreads) {
        const int q = e / S, k = e - q * S;
        t[e] = g_tw_master.v[((k * q) & (SR - 1)) * step];
      }
    } else {
      for (int e = tid; e < R * S; e += nthreads) {
        const int q = e / S, k = e - q * S;
        double sn, cs;
        sincospi(-2.0 * double((k * q) & (SR - 1)) / double(SR), &sn, &cs);
        t[e] = make_float2(float(cs), float(sn));
      }
    }
  });
}

// Team synchronisation: teams of <= 32 threads live inside one warp; larger teams are the
// whole CTA.
template <int P>
__device__ __forceinline__ void team_sync(unsigned mask) {
  if constexpr (P <= 32) {
    __syncwarp(mask);
  } else {
    __syncthreads();
  }
}

// Run passes 1..NPASS-1 given that pass 0 outputs are already in v (natural order per butterfly,
// v[b*R0 + r]). Writes pass outputs to the exchange buffer, reads the next pass inputs. On return
// v[e] holds bin k = t + e*P.
template <class PL>
__device__ __forceinline__ void team_passes(float2 (&v)[PL::E], float2* buf, const float2* tw,
                                            int t, unsigned mask) {
  constexpr int L = PL::L, P = PL::P;
  static_for<0, PL::NPASS - 1>([&](auto pc) {
    constexpr int p = decltype(pc)::value;  // pass whose outputs are being stored
    constexpr int R = PL::radix(p), S = PL::span(p), B = PL::E / R;
    // store pass-p outputs in Stockham order. The padded index pad(base + r S) is pad(base)
    // plus a compile-time offset whenever adding r S cannot carry into the padding shift: S a
    // multiple of 2^PADSH, or the R S-aligned block holding base inside one 2^PADSH block.
    constexpr int PB = 1 << PL::PADSH;
    static_for<0, B>([&](auto bc) {
      constexpr int b = decltype(bc)::value;
      const int j = t + P * b;
      const int jm = j % S;
      const int base = (j - jm) * R + jm;
      if constexpr (S % PB == 0 || R * S <= PB) {
        float2* pb = buf + PL::pad(base);
        static_for<0, R>([&](auto rc) {
          constexpr int r = decltype(rc)::value;
          constexpr int off = (S % PB == 0) ? r * S + ((r * S) >> PL::PADSH) : r * S;
          pb[off] = v[b * R + r];
        });
      } else {
        static_for<0, R>([&](auto rc) {
          constexpr int r = decltype(rc)::value;
          buf[PL::pad(base + r * S)] = v[b * R + r];
        });
      }
    });
    team_sync<P>(mask);
    // load pass-(p+1) inputs, apply twiddles, bit-reverse into the register DFT order
    constexpr int pn = p + 1;
    constexpr int Rn = PL::radix(pn), Sn = PL::span(pn), Bn = PL::E / Rn;
    const float2* twp = tw + PL::tw_off(pn);
    // Radix-16 passes of transforms of 2048 points and more (exchange- and twiddle-read-bound
    // in shared memory) read the twiddle anchors w, w^2, w^4, w^8 of the butterfly and form the
    // other eleven powers by complex products in registers (each within ~2 ulp), a quarter of
    // the twiddle reads.
    constexpr bool kAnchors = L >= 2048 && Rn == 16;
    static_for<0, Bn>([&](auto bc) {
      constexpr int b = decltype(bc)::value;
      const int j = t + P * b;
      const int jm = j % Sn;
      // j < L / Rn: with L / Rn a multiple of 2^PADSH the q-th input sits at a compile-time
      // offset from pad(j)
      constexpr int QS = L / Rn;
      const float2* pj = buf + PL::pad(j);
      [[maybe_unused]] float2 w1, w2, w3, w4, w5, w6, w7, w8;  // set only with kAnchors
      if constexpr (kAnchors) {
        w1 = twp[Sn + jm];
        w2 = twp[2 * Sn + jm];
        w4 = twp[4 * Sn + jm];
        w8 = twp[8 * Sn + jm];
        w3 = cmul(w1, w2);
        w5 = cmul(w4, w1);
        w6 = cmul(w4, w2);
        w7 = cmul(w4, w3);
      }
      static_for<0, Rn>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        float2 val;
        if constexpr (QS % PB == 0) {
          val = pj[q * QS + ((q * QS) >> PL::PADSH)];
        } else {
          val = buf[PL::pad(j + q * QS)];
        }
        if constexpr (q > 0) {
          if constexpr (kAnchors) {
            constexpr int lo = q & 7;
            const float2 wl = lo == 1 ? w1 : lo == 2 ? w2 : lo == 3 ? w3 : lo == 4 ? w4
                            : lo == 5 ? w5 : lo == 6 ? w6 : w7;
            const float2 wq = q == 8 ? w8 : (q > 8 ? cmul(w8, wl) : wl);
            val = cmul(val, wq);
          } else {
            val = cmul(val, twp[q * Sn + jm]);
          }
        }
        v[b * Rn + bitrev(q, ilog2(Rn))] = val;
      });
    });
    team_sync<P>(mask);
    static_for<0, Bn>([&](auto bc) {
      constexpr int b = decltype(bc)::value;
      dft_dit<Rn, b * Rn>(v);
    });
  });
}

// Pass 0 DFTs (inputs already placed at v[b*R0 + bitrev(q)] for butterfly j = t + P*b, input
// element j + q*L/R0).
template <class PL>
__device__ __forceinline__ void team_pass0(float2 (&v)[PL::E]) {
  constexpr int R0 = PL::radix(0), B0 = PL::E / R0;
  static_for<0, B0>([&](auto bc) {
    constexpr int b = decltype(bc)::value;
    dft_dit<R0, b * R0>(v);
  });
}

}  // namespace b2s
