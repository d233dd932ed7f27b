// 50%-overlap welch for nfft == nperseg == 1024, hop == 512, on packed f32x2 arithmetic.
//
// Same mathematics as k_welch_half (two consecutive segments per complex FFT, z = x_s +
// i x_{s+1}, accumulating |Z_k|^2; half-blocks A | B | C loaded once with C carried; window
// fused into the first radix-2 stage; constant detrend as the low-bin spectral correction), with
// the 32 complex points of each thread held as structure-of-arrays PAIRS: register pair j keeps
// the real parts of register positions j and j + 16 (re[j] = (re_j, re_{j+16})) and another
// keeps their imaginary parts. Every radix-2 stage of the in-register 32-point DFT whose
// butterflies join positions p and p + H with H <= 8 then runs on both halves at once with one
// packed instruction (FADD2 / FMUL2 / FFMA2) per operation, and both halves use the same
// twiddle, so trivial (1, -i) and general twiddles never mix inside an instruction. Only the
// H = 16 stage (positions p and p + 16: the two halves of one pair) stays scalar. The inter-pass
// twiddle multiply and the |Z|^2 accumulation are packed too. The B200 FP32 pipe is 32 lanes
// per sub-partition, so packing does not add FP32 throughput: it halves the issue slots the
// FP32 work takes, which leaves the loads, exchange and address work room to issue beside it.
//
// Exchange between the two radix-32 passes (32 x 32 transpose through shared memory): real and
// imaginary planes of 32 rows x 34 floats; row r (the writer thread) keeps output q at float
// 2 (q mod 16) + q / 16, so a pair (q, q + 16) is one 64-bit store and a column read (one float
// per row) is bank-conflict free.
//
// Segment sums: the |Z_k|^2 terms of each block of kFoldPairs pairs are summed in registers,
// then added into a per-team FP32 shared-memory total (two-level blocked summation: the
// rounding error grows with kFoldPairs + pairs / kFoldPairs instead of with the pair count);
// the cross-team sum is FP64 (k_reduce_mean).
//
// Reference behaviour replaced: _stft_metal.rfft_power_mean (src/mlx_signal_processing/
// _stft_metal.py:530-557, kernel _SUM_SRC :458-505, group reduction _reduce_groups :443-455).
#pragma once

#include "mean_kernels.cuh"

namespace b2s {
namespace pk {

constexpr int kRowStride = 34;  // floats per exchange row
constexpr int kPlane = 32 * kRowStride;  // floats per exchange plane

__device__ __forceinline__ float2 bc(float c) { return make_float2(c, c); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, neg2(b)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// Packed radix-2 DIT butterfly with the same compile-time twiddle W_M^I in both halves:
// (a, c) -> (a + w c, a - w c), complex values given as (re, im) pairs of packed registers.
template <int I, int M>
__device__ __forceinline__ void bfly2(float2& ar, float2& ai, float2& cr, float2& ci) {
  constexpr int i = I % M;
  const float2 tr = ar, ti = ai;
  if constexpr (i == 0) {
    ar = add2(tr, cr);
    ai = add2(ti, ci);
    cr = sub2(tr, cr);
    ci = sub2(ti, ci);
  } else if constexpr (4 * i == M) {  // w = -i: w c = (ci, -cr)
    ar = add2(tr, ci);
    ai = sub2(ti, cr);
    const float2 ncr = cr;
    cr = sub2(tr, ci);
    ci = add2(ti, ncr);
  } else if constexpr (4 * i == 3 * M) {  // w = +i: w c = (-ci, cr)
    ar = sub2(tr, ci);
    ai = add2(ti, cr);
    const float2 ncr = cr;
    cr = add2(tr, ci);
    ci = sub2(ti, ncr);
  } else {
    constexpr CS w = twiddle(i, M);
    constexpr bool rmaj = dabs(w.c) >= dabs(w.s);
    constexpr float sc = float(rmaj ? w.c : w.s);
    constexpr float tn = float(rmaj ? w.s / w.c : w.c / w.s);
    float2 ur, ui;
    if constexpr (rmaj) {  // w = sc (1 + i tn)
      ur = fma2(bc(-tn), ci, cr);
      ui = fma2(bc(tn), cr, ci);
    } else {  // w = sc (tn + i)
      ur = fma2(bc(tn), cr, neg2(ci));
      ui = fma2(bc(tn), ci, cr);
    }
    ar = fma2(bc(sc), ur, tr);
    ai = fma2(bc(sc), ui, ti);
    cr = fma2(bc(-sc), ur, tr);
    ci = fma2(bc(-sc), ui, ti);
  }
}

// 32-point DIT DFT on the packed layout (position p < 16 in the .x half of pair p, p >= 16 in
// the .y half of pair p - 16; inputs in bit-reversed position order, outputs natural). Stages
// with span H0 .. 8 are packed; the span-16 stage joins the two halves of each pair (scalar).
template <int H0>
__device__ __forceinline__ void dft32(float2 (&re)[16], float2 (&im)[16]) {
  static_for<0, 4>([&](auto sc_) {
    constexpr int H = 1 << decltype(sc_)::value;
    if constexpr (H >= H0) {
      static_for<0, 16 / (2 * H)>([&](auto gc) {
        constexpr int g = decltype(gc)::value * 2 * H;
        static_for<0, H>([&](auto ic) {
          constexpr int i = decltype(ic)::value;
          bfly2<i, 2 * H>(re[g + i], im[g + i], re[g + i + H], im[g + i + H]);
        });
      });
    }
  });
  static_for<0, 16>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    float2 a = make_float2(re[i].x, im[i].x);
    float2 c = make_float2(re[i].y, im[i].y);
    bfly<i, 32>(a, c);
    re[i] = make_float2(a.x, c.x);
    im[i] = make_float2(a.y, c.y);
  });
}

// Shared-memory layout per CTA: scratch | window table | low-bin window spectrum | pass-1
// twiddles | per team: exchange planes (re, im) and the blocked-sum totals.
template <class CFG>
struct Smem {
  using PL = typename CFG::PL;
  static constexpr int P = PL::P;                    // 32
  static constexpr int WIN4 = 8 * P;                 // float4 window entries
  static constexpr int TW4 = 16 * P;                 // float4 twiddle entries
  static constexpr int TEAM_FLOATS = 2 * kPlane + 32 * P;  // planes + totals (16 float2 x P)
  static constexpr size_t BYTES = size_t(CFG::TEAMS) * 16 + size_t(WIN4) * 16 +
                                  size_t(2 * P) * 8 + size_t(TW4) * 16 +
                                  size_t(CFG::TEAMS) * TEAM_FLOATS * 4;
};

struct Ctx {
  const float4* wt;    // window: wt[g * 32 + t] = (w[n], w[n + 32], w[n + 512], w[n + 544])
  const float2* wlo;   // DFT(win)_t, t < 32 (zero beyond n_low)
  const float2* whi;   // DFT(win)_{L - 32 + t}
  const float4* tw;    // pass-1 twiddles: tw[m * 32 + t] = (Re W^(2m t), Re W^((2m+1) t),
                       //                                    Im W^(2m t), Im W^((2m+1) t))
  float* xre;          // exchange planes (re at xre, im at xre + kPlane)
  float2* tot;         // blocked-sum totals: tot[j * 32 + t]
  float4* scratch;
  int t;
};

// Element offset of register pair g's first lane in the pass-0 load pattern: position 2g holds
// element t + 32 bitrev5(2g) = t + 64 bitrev3(g), position 2g + 16 the element 32 later.
template <int G>
__device__ __forceinline__ int load_off(int t) {
  return t + 64 * bitrev(G, 3);
}

// Welch over the pairs of segments [s0, s1) of one row; writes the row's mirror-combined
// partial slot (dst[k] = Q_k + Q_{L-k}, k <= 512) at the end.
template <int DET>
__device__ __forceinline__ void welch_range(const Ctx& c, const float* __restrict__ xr, int s0,
                                            int s1, float* dst) {
  constexpr int L = 1024, H = 512, P = 32;
  const int t = c.t;
  const unsigned mask = 0xffffffffu;
  const float inv_n = 1.0f / float(L);
  float2 A[8], B[8], C[8];
  float2 acc[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    acc[j] = make_float2(0.f, 0.f);
    c.tot[j * P + t] = make_float2(0.f, 0.f);
  }
  bool carry = false;
  float sum_c = 0.f;
  int npairs = 0;
  auto step = [&](int s, auto two_c) {
    constexpr bool TWO = decltype(two_c)::value;
    const float* base = xr + int64_t(s) * H;
    if (s + 3 < s1) {  // warm L2 with the next pair's two new half-blocks
      for (int o = t * 32; o < 2 * H; o += P * 32)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(base + 3 * H + o));
    }
    static_for<0, 8>([&](auto gc) {
      constexpr int g = decltype(gc)::value;
      const int n = load_off<g>(t);
      if (!carry) A[g] = make_float2(__ldg(base + n), __ldg(base + n + 32));
      B[g] = make_float2(__ldg(base + H + n), __ldg(base + H + n + 32));
      C[g] = TWO ? make_float2(__ldg(base + 2 * H + n), __ldg(base + 2 * H + n + 32))
                 : make_float2(0.f, 0.f);
    });
    float ma = 0.f, mb = 0.f;
    if constexpr (DET != kDetrendNone) {
      auto tsum = [](const float2(&v)[8]) {
        const float2 s = add2(add2(add2(v[0], v[1]), add2(v[2], v[3])),
                              add2(add2(v[4], v[5]), add2(v[6], v[7])));
        return s.x + s.y;
      };
      float sa = sum_c;
      if (!carry) {
        float sums[1] = {tsum(A)};
        team_sum<P, 1>(sums, c.scratch, mask);
        sa = sums[0];
      }
      float sums[2] = {tsum(B), TWO ? tsum(C) : 0.f};
      team_sum<P, 2>(sums, c.scratch, mask);
      ma = (sa + sums[0]) * inv_n;
      mb = TWO ? (sums[0] + sums[1]) * inv_n : 0.f;
      sum_c = sums[1];
    }
    float2 re[16], im[16];
    // window + first radix-2 stage (positions 2g, 2g + 1 pair elements n and n + 512)
    static_for<0, 8>([&](auto gc) {
      constexpr int g = decltype(gc)::value;
      const float4 w4 = c.wt[g * P + t];
      const float2 wl = make_float2(w4.x, w4.y), wh = make_float2(w4.z, w4.w);
      float2 al = A[g], bl = TWO ? B[g] : make_float2(0.f, 0.f);
      float2 ah = B[g], bh = C[g];
      if constexpr (DET == kDetrendConstant) {
        al = sub2(al, bc(ma));
        ah = sub2(ah, bc(ma));
        if constexpr (TWO) {
          bl = sub2(bl, bc(mb));
          bh = sub2(bh, bc(mb));
        }
      }
      const float2 ar = mul2(wl, al), ai = mul2(wl, bl);
      re[2 * g] = fma2(wh, ah, ar);
      re[2 * g + 1] = fma2(neg2(wh), ah, ar);
      im[2 * g] = fma2(wh, bh, ai);
      im[2 * g + 1] = fma2(neg2(wh), bh, ai);
    });
    dft32<2>(re, im);
    // exchange: row t keeps pass-0 output q at 2 (q mod 16) + q / 16
    __syncwarp(mask);
    {
      float2* wr = reinterpret_cast<float2*>(c.xre + t * kRowStride);
      float2* wi = reinterpret_cast<float2*>(c.xre + kPlane + t * kRowStride);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        wr[j] = re[j];
        wi[j] = im[j];
      }
    }
    __syncwarp(mask);
    {
      const int col = 2 * (t & 15) + (t >> 4);
      const float* rr = c.xre + col;
      const float* ri = c.xre + kPlane + col;
      static_for<0, 16>([&](auto jc) {
        constexpr int j = decltype(jc)::value;
        constexpr int q = bitrev(j, 5);  // rows q, q + 1 -> positions j, j + 16
        const float2 zr = make_float2(rr[q * kRowStride], rr[(q + 1) * kRowStride]);
        const float2 zi = make_float2(ri[q * kRowStride], ri[(q + 1) * kRowStride]);
        const float4 w4 = c.tw[(q / 2) * P + t];
        const float2 wr = make_float2(w4.x, w4.y), wi = make_float2(w4.z, w4.w);
        re[j] = fma2(zr, wr, neg2(mul2(zi, wi)));
        im[j] = fma2(zr, wi, mul2(zi, wr));
      });
    }
    __syncwarp(mask);
    dft32<1>(re, im);
    if constexpr (DET == kDetrendConstantSpectral) {
      const float2 m = make_float2(ma, mb);
      const float2 cl = cmul(m, c.wlo[t]);
      const float2 ch = cmul(m, c.whi[t]);
      re[0].x -= cl.x;
      im[0].x -= cl.y;
      re[15].y -= ch.x;
      im[15].y -= ch.y;
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      acc[j] = fma2(re[j], re[j], acc[j]);
      acc[j] = fma2(im[j], im[j], acc[j]);
    }
#pragma unroll
    for (int g = 0; g < 8; ++g) A[g] = C[g];
    carry = true;
    if (++npairs == kFoldPairs) {  // fold the register block into the team total
      npairs = 0;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        c.tot[j * P + t] = add2(c.tot[j * P + t], acc[j]);
        acc[j] = make_float2(0.f, 0.f);
      }
    }
  };
  int s = s0;
  for (; s + 1 < s1; s += 2) step(s, std::true_type{});
  if (s < s1) step(s, std::false_type{});
  // total of the range: bin t + 32 j in .x, bin t + 32 j + 512 in .y; mirror-combine through the
  // exchange plane (dst[k] = Q_k + Q_{L-k})
  float* sq = c.xre;
  __syncwarp(mask);
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const float2 v = add2(c.tot[j * P + t], acc[j]);
    sq[t + 32 * j] = v.x;
    sq[t + 32 * j + 512] = v.y;
  }
  __syncwarp(mask);
  for (int k = t; k <= L / 2; k += P) dst[k] = sq[k] + sq[(L - k) & (L - 1)];
  __syncwarp(mask);
}

}  // namespace pk

// Packed 50%-overlap welch, nfft == nperseg == 1024, hop 512: one 32-thread team per warp,
// teams walk balanced (row, segment) ranges as k_welch_half does and write the same partial
// slots (mirror-combined |Z|^2 sums) for k_reduce_mean.
template <int DET>
__global__ void __launch_bounds__(MeanCfg<10, 5>::THREADS, MeanCfg<10, 5>::MIN_CTAS)
    k_welch_half_packed(MeanParams pr) {
  using CFG = MeanCfg<10, 5>;
  using SM = pk::Smem<CFG>;
  constexpr int P = 32, L = 1024;
  extern __shared__ float4 smem[];
  float4* scratch = smem;                                     // TEAMS float4
  float4* wt = smem + CFG::TEAMS;                             // 8 x 32 float4
  float2* wlo = reinterpret_cast<float2*>(wt + SM::WIN4);     // 32
  float2* whi = wlo + P;                                      // 32
  float4* tw = reinterpret_cast<float4*>(whi + P);            // 16 x 32 float4
  float* teamf = reinterpret_cast<float*>(tw + SM::TW4);      // TEAMS x TEAM_FLOATS
  // window table: wt[g * 32 + t] = (w[n], w[n + 32], w[n + 512], w[n + 544]), n = t + 64 bitrev3(g)
  for (int i = threadIdx.x; i < SM::WIN4; i += blockDim.x) {
    const int g = i / P, t = i - g * P;
    const int n = t + 64 * bitrev(g, 3);
    wt[i] = make_float4(pr.win[n], pr.win[n + 32], pr.win[n + 512], pr.win[n + 544]);
  }
  if constexpr (DET == kDetrendConstantSpectral)
    load_window_lowbins<P>(wlo, whi, pr.wdft, pr.n_low, threadIdx.x, blockDim.x);
  // pass-1 twiddles W_1024^(q t) for the row pair q = 2m, 2m + 1 (from the FP64-built master)
  for (int i = threadIdx.x; i < SM::TW4; i += blockDim.x) {
    const int m = i / P, t = i - m * P;
    const float2 a = g_tw_master.v[((2 * m * t) & (L - 1)) * (kTwMasterN / L)];
    const float2 b = g_tw_master.v[(((2 * m + 1) * t) & (L - 1)) * (kTwMasterN / L)];
    tw[i] = make_float4(a.x, b.x, a.y, b.y);
  }
  __syncthreads();
  pdl_trigger();
  const int team = threadIdx.x / P;
  pk::Ctx c;
  c.wt = wt;
  c.wlo = wlo;
  c.whi = whi;
  c.tw = tw;
  c.xre = teamf + team * SM::TEAM_FLOATS;
  c.tot = reinterpret_cast<float2*>(c.xre + 2 * pk::kPlane);
  c.scratch = scratch + team;
  c.t = threadIdx.x - team * P;
  const int64_t tau = int64_t(blockIdx.x) * CFG::TEAMS + team;
  int64_t g = tau * pr.G;
  const int64_t gend = min(g + pr.G, pr.total);
  while (g < gend) {
    const int64_t r = g / pr.nseg;
    const int s0 = int(g - r * pr.nseg);
    const int64_t lim = int64_t(s0) + (gend - g);
    const int s1 = int(lim < pr.nseg ? lim : int64_t(pr.nseg));
    const int64_t slot = tau - first_team(r, pr.nseg, pr.G);
    pk::welch_range<DET>(c, pr.x + r * pr.ld_x, s0, s1,
                         pr.partial + (r * pr.cmax + slot) * int64_t(welch_slot_floats(L)));
    g += s1 - s0;
  }
}

}  // namespace b2s
