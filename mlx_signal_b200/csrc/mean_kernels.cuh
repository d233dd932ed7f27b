// Fused segment-mean spectral kernels: welch (|X|^2), csd (conj(X) Y) and coherence
// (Pxx, Pyy, Pxy) for power-of-two nfft, real float32 input.
//
// Reference behaviour replaced: _stft_metal.rfft_power_mean (src/mlx_signal_processing/
// _stft_metal.py:530-557, kernel source _SUM_SRC :458-505), csd_mean / coherence_mean
// (:739-746, _PAIR_SUM_SRC :620-667) and their host-side group reduction (_reduce_groups
// :443-455). Differences by design:
//  * welch packs TWO real segments of a row into one complex FFT (z = x_s + i x_{s+1}); the sum
//    of both power spectra is (|Z_k|^2 + |Z_{L-k}|^2)/2, so no per-segment untangle is needed and
//    the mirror combination happens once, in the final reduction;
//  * csd/coherence pack x and y of the same segment (z = x_s + i y_s); the per-bin products
//    Z_k Z_{L-k} and |Z_k|^2 carry all three cross/auto spectra;
//  * the flattened (row, segment) space is split evenly over all resident teams, each team
//    accumulating in registers and writing one partial row per row it touches; the final
//    reduction sums partials in a fixed order in FP64 (deterministic, blocked summation).
#pragma once

#include "fft_core.cuh"
#include "spectral_params.h"
#include "team_util.cuh"

namespace b2s {

template <int LOG_L, int LOG_E>
struct MeanCfg {
  using PL = Plan<LOG_L, LOG_E>;
  static constexpr int TEAMS = PL::P >= 64 ? 1 : 128 / PL::P;
  static constexpr int THREADS = TEAMS * PL::P;
  // 128-thread CTAs held to 3 per SM (<= 168 registers); measured faster for the generic welch
  // and the frame kernels, whose unbounded builds took ~208-254 registers (2 CTAs per SM)
  static constexpr int MIN_CTAS = THREADS == 128 ? 3 : 1;
  static constexpr int SCRATCH = PL::P >= 64 ? PL::P / 32 : 1;   // float4 per team
  static constexpr int WIN = (PL::L + 3) & ~3;                     // window floats (16 B multiple)
  static constexpr size_t SMEM = size_t(TEAMS) * SCRATCH * 16      // team scratch
                                 + size_t(WIN) * 4                 // window
                                 + size_t(PL::TW) * 8              // twiddle tables
                                 + size_t(TEAMS) * PL::BUF * 8;    // exchange buffers
};

// k_welch_mean's shared memory: the MeanCfg layout plus one L-float blocked-sum total per team.
template <class CFG>
constexpr size_t welch_mean_smem() {
  return CFG::SMEM + size_t(CFG::TEAMS) * CFG::PL::L * 4;
}

struct MeanSmem {
  float4* scratch;
  float* win;
  float2* tw;
  float2* buf;
};

template <class CFG>
__device__ __forceinline__ MeanSmem mean_smem_setup(const float* win, int nperseg) {
  using PL = typename CFG::PL;
  extern __shared__ float4 smem[];
  MeanSmem s;
  s.scratch = smem;
  s.win = reinterpret_cast<float*>(smem + CFG::TEAMS * CFG::SCRATCH);
  s.tw = reinterpret_cast<float2*>(s.win + CFG::WIN);
  s.buf = s.tw + PL::TW;
  for (int i = threadIdx.x; i < PL::L; i += blockDim.x) s.win[i] = i < nperseg ? win[i] : 0.f;
  build_twiddles<PL>(s.tw, threadIdx.x, blockDim.x);
  __syncthreads();
  return s;
}

// Load two real segments into (re, im) in the pass-0 element pattern (zero beyond nperseg or
// when the second segment is absent).
template <class PL>
__device__ __forceinline__ void load_pair(float2 (&v)[PL::E], const float* __restrict__ a,
                                          const float* __restrict__ b, bool has_b, int t,
                                          int nperseg) {
  if (nperseg == PL::L) {
    static_for<0, PL::E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const int n = slot_elem<PL, e>(t);
      v[e].x = __ldg(a + n);
      v[e].y = has_b ? __ldg(b + n) : 0.f;
    });
  } else {
    static_for<0, PL::E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const int n = slot_elem<PL, e>(t);
      const bool ok = n < nperseg;
      v[e].x = ok ? __ldg(a + n) : 0.f;
      v[e].y = (ok && has_b) ? __ldg(b + n) : 0.f;
    });
  }
}

// Welch partial slot: P2_k = Q_k + Q_{L-k} for k in [0, L/2] (the mirror-combined |Z|^2 sums;
// 0.5 * P2_k is the sum of |X_s[k]|^2 over both segments of every pair).
__host__ __device__ constexpr int welch_slot_floats(int L) { return L / 2 + 1; }

// Two-level blocked summation of the welch kernels' per-bin sums: each thread sums the |Z|^2
// terms of kFoldPairs pairs of segments in registers, then adds that block into a team total in
// shared memory (tot[e * P + t], FP32). The rounding error of a team's sum then grows with
// kFoldPairs + pairs / kFoldPairs instead of with the number of pairs; the cross-team sum of the
// partial slots is FP64 (k_reduce_mean).
constexpr int kFoldPairs = 8;
// From nfft 2048 up the 50%-overlap welch kernel keeps plain FP32 register sums while a team's
// range holds at most kDirectPairs pairs (relative rounding error <= kDirectPairs * 2^-24 ~
// 3.8e-6) and adds the shared-memory block totals only beyond that (the BLOCKED instantiation,
// chosen by the host from the segments per team): the totals cost 3-5 % of the kernel's time at
// nperseg 4096 and 8192 on 64 x 2^20, whose teams sum ~110 segments.
constexpr int kDirectPairs = 64;
constexpr int kDirectSegs = 2 * kDirectPairs;  // host switch: block totals when G > kDirectSegs

template <int E, int P>
__device__ __forceinline__ void fold_block(float (&acc)[E], float* tot, int t) {
#pragma unroll
  for (int e = 0; e < E; ++e) {
    tot[e * P + t] += acc[e];
    acc[e] = 0.f;
  }
}

template <int E, int P>
__device__ __forceinline__ void zero_total(float* tot, int t) {
#pragma unroll
  for (int e = 0; e < E; ++e) tot[e * P + t] = 0.f;
}

// Write a team's per-bin accumulators (bin k = t + e*P in acc[e]) as mirror-combined partials
// dst[k] = acc_k + acc_{L-k}, k in [0, L/2], staging through the (free) exchange buffer; resets
// acc.
template <class PL>
__device__ __forceinline__ void flush_mirror(float (&acc)[PL::E], float* dst, float2* buf, int t,
                                             unsigned mask) {
  constexpr int L = PL::L, E = PL::E, P = PL::P;
  float* sq = reinterpret_cast<float*>(buf);
  team_sync<P>(mask);
#pragma unroll
  for (int e = 0; e < E; ++e) {
    sq[t + e * P] = acc[e];
    acc[e] = 0.f;
  }
  team_sync<P>(mask);
  for (int k = t; k <= L / 2; k += P) dst[k] = sq[k] + sq[(L - k) & (L - 1)];
  team_sync<P>(mask);
}

// Welch: partial[r][slot][k] = sum over the team's segments of |Z_k|^2, z = x_s + i x_{s+1}.
template <int LOG_L, int LOG_E, int DET>
__global__ void __launch_bounds__(MeanCfg<LOG_L, LOG_E>::THREADS, MeanCfg<LOG_L, LOG_E>::MIN_CTAS)
    k_welch_mean(MeanParams pr) {
  using CFG = MeanCfg<LOG_L, LOG_E>;
  using PL = typename CFG::PL;
  constexpr int L = PL::L, E = PL::E, P = PL::P;
  const MeanSmem sm = mean_smem_setup<CFG>(pr.win, pr.nperseg);
  const int team = threadIdx.x / P, t = threadIdx.x - team * P;
  const unsigned mask = team_mask<P>();
  float4* scratch = sm.scratch + team * CFG::SCRATCH;
  float2* buf = sm.buf + team * PL::BUF;
  const int64_t tau = int64_t(blockIdx.x) * CFG::TEAMS + team;
  int64_t g = tau * pr.G;
  const int64_t gend = min(g + pr.G, pr.total);
  float* tot = reinterpret_cast<float*>(sm.buf + CFG::TEAMS * PL::BUF) + team * L;
  float acc[E];
#pragma unroll
  for (int e = 0; e < E; ++e) acc[e] = 0.f;
  while (g < gend) {
    const int64_t r = g / pr.nseg;
    const int s0 = int(g - r * pr.nseg);
    const int64_t lim = int64_t(s0) + (gend - g);
    const int s1 = int(lim < pr.nseg ? lim : int64_t(pr.nseg));
    const float* xr = pr.x + r * pr.ld_x;
    zero_total<E, P>(tot, t);
    int npairs = 0;
    for (int s = s0; s < s1; s += 2) {
      const bool two = s + 1 < s1;
      const float* xa = xr + int64_t(s) * pr.hop;
      float2 v[E];
      load_pair<PL>(v, xa, xa + pr.hop, two, t, pr.nperseg);
      detrend_window<PL, DET>(v, sm.win, t, pr.nperseg, scratch, mask);
      team_pass0<PL>(v);
      team_passes<PL>(v, buf, sm.tw, t, mask);
#pragma unroll
      for (int e = 0; e < E; ++e) {
        acc[e] = fmaf(v[e].x, v[e].x, acc[e]);
        acc[e] = fmaf(v[e].y, v[e].y, acc[e]);
      }
      if (++npairs == kFoldPairs) {
        npairs = 0;
        fold_block<E, P>(acc, tot, t);
      }
    }
#pragma unroll
    for (int e = 0; e < E; ++e) acc[e] += tot[e * P + t];
    const int64_t slot = tau - first_team(r, pr.nseg, pr.G);
    flush_mirror<PL>(acc, pr.partial + (r * pr.cmax + slot) * int64_t(welch_slot_floats(L)), buf,
                     t, mask);
    g += s1 - s0;
  }
}

// Programmatic dependent launch: let the dependent reduction grid be scheduled as soon as every
// CTA of this grid has started (it waits for our completion before reading partials).
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Launch a 50%-overlap kernel as a programmatic dependent of the stream's previous kernel: its
// CTAs become resident and build their constant tables while that kernel (typically the previous
// call's reduction) finishes; they read the caller's buffers only after griddepcontrol.wait.
template <class K>
inline void launch_half(K kernel, dim3 g, int threads, size_t smem, cudaStream_t s,
                        const MeanParams& p) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = g;
  cfg.blockDim = dim3(unsigned(threads));
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  (void)cudaLaunchKernelEx(&cfg, kernel, p);  // errors surface through cudaGetLastError
}

// Shared-memory tables and team coordinates used by the half-overlap pair loop.
template <class PL>
struct HalfCtx {
  const float* win;    // L window values (read when the transposed table is not used)
  const float4* wt;    // this thread's transposed window row: (w[n_g], w[n_g+H], w[n_g+1], ...)
  const float2* wlo;   // DFT(win)_t for t < P (zero beyond n_low)
  const float2* whi;   // DFT(win)_{L-P+t}
  const float2* tw;    // inter-pass twiddles
  float2* buf;         // team exchange buffer
  float4* scratch;     // team reduction scratch
  int t;
  unsigned mask;
};

// Transposed window table of the half-overlap kernel: row t (team-local thread) holds, for its
// register pairs g < E/2, w[n_g] and w[n_g + L/2] with n_g = slot_elem<2g>(t), so a thread reads
// its whole window with E/4 128-bit loads. Row stride E + 4 floats keeps rows 16-byte aligned and
// the 8-thread phases of a 128-bit load on disjoint banks.
template <class PL>
struct HalfWinT {
  static constexpr int WS = PL::E + 4;
  static constexpr int FLOATS = PL::P * WS;
  static constexpr bool USE = PL::E >= 4;
};

template <class PL>
__device__ __forceinline__ void build_half_wint(float* wt, const float* win, int tid) {
  constexpr int H = PL::L / 2, WS = HalfWinT<PL>::WS;
  if (tid < PL::P) {
    float* row = wt + tid * WS;
    static_for<0, PL::E / 2>([&](auto gc) {
      constexpr int gi = decltype(gc)::value;
      const int n = slot_elem<PL, 2 * gi>(tid);
      row[2 * gi] = win[n];
      row[2 * gi + 1] = win[n + H];
    });
  }
}

// Shared-memory layout of the half-overlap kernel: scratch | window (transposed table or L floats) |
// low-bin window
// spectrum (2P complex: DFT_L(win)_t and DFT_L(win)_{L-P+t}) | twiddles | exchange buffers.
template <class CFG>
struct HalfSmem {
  using PL = typename CFG::PL;
  // window region: the transposed table (E >= 4) or the plain window, in floats (16-byte multiple)
  static constexpr int WINF = ((HalfWinT<PL>::USE ? HalfWinT<PL>::FLOATS : PL::L) + 3) & ~3;
  static constexpr size_t BYTES = size_t(CFG::TEAMS) * CFG::SCRATCH * 16 + size_t(WINF) * 4 +
                                  size_t(2 * PL::P) * 8 + size_t(PL::TW) * 8 +
                                  size_t(CFG::TEAMS) * PL::BUF * 8;
};

// k_welch_half's shared memory: the HalfSmem layout plus one L-float blocked-sum total per team.
template <class CFG>
constexpr size_t welch_half_smem() {
  return HalfSmem<CFG>::BYTES + size_t(CFG::TEAMS) * CFG::PL::L * 4;
}

// Welch for the 50%-overlap case nperseg == nfft == L, hop == L/2 (the reference's default
// noverlap = nperseg/2). A pair of segments (s, s+1) spans three half-blocks A | B | C of the row:
// x_s = A|B, x_{s+1} = B|C, and the next pair's A is this pair's C. Each half-block is loaded once
// (C is carried in registers), the segment sums come from the three block sums, and the window
// multiply is fused into the first radix-2 butterfly stage, which pairs elements n and n + L/2:
// out = a +/- c with a = z_n w_n, c = z_{n+L/2} w_{n+L/2}.
// Constant detrend: DET == kDetrendConstant subtracts the means before the window (time domain);
// DET == kDetrendConstantSpectral subtracts (m_s + i m_{s+1}) DFT(win)_k after the FFT on the
// low bins k < n_low and k > L - n_low (the only non-zero window-spectrum bins), which keeps the
// mean reduction off the FFT's critical path.
//
// welch_half_range accumulates sum |Z_k|^2 over the pairs of segments [s0, s1) of one row into
// acc (bin k = t + e*P in acc[e]). Full pairs run a step without the lone-segment selects; an odd
// last segment runs the same step with the second segment zero. WT: window from the transposed
// table (HalfWinT) instead of the plain one. SPLIT = false keeps one loop with a runtime
// lone-segment flag (less code, for kernels that already run near their register limit).
// tot: optional blocked-sum team total (tot[e * P + t]); when given, acc is folded into it every
// kFoldPairs pairs (the caller zeroes it and adds it back at the end of the range).
template <class PL, int DET, bool WT = false, bool SPLIT = true>
__device__ __forceinline__ void welch_half_range(const HalfCtx<PL>& c, const float* __restrict__ xr,
                                                 int s0, int s1, float (&acc)[PL::E],
                                                 float* tot = nullptr) {
  constexpr int L = PL::L, E = PL::E, P = PL::P, H = L / 2, EH = E / 2;
  constexpr int R0 = PL::radix(0), B0 = E / R0;
  static_assert(!WT || HalfWinT<PL>::USE, "transposed window needs E >= 4");
  const int t = c.t;
  const float inv_n = 1.0f / float(L);
  float A[EH], B[EH], C[EH];
  bool carry = false;
  int npairs = 0;
  float sum_c = 0.f;  // team total of the carried half-block (this pair's A)
  auto step = [&](int s, auto two_c) {
    const bool TWO = bool(two_c);  // a compile-time constant for std::true_type / false_type
    const float* base = xr + int64_t(s) * H;
    if (s + 3 < s1) {  // warm L2 with the next pair's two new half-blocks
      for (int o = t * 32; o < 2 * H; o += P * 32)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(base + 3 * H + o));
    }
    static_for<0, EH>([&](auto gc) {
      constexpr int gi = decltype(gc)::value;
      const int n = slot_elem<PL, 2 * gi>(t);
      if (!carry) A[gi] = __ldg(base + n);
      B[gi] = __ldg(base + H + n);
      C[gi] = TWO ? __ldg(base + 2 * H + n) : 0.f;
    });
    [[maybe_unused]] float ma = 0.f, mb = 0.f;  // segment means (constant detrend only)
    if constexpr (DET == kDetrendConstant || DET == kDetrendConstantSpectral) {
      // block totals: A's comes from the previous pair (its C), so only B and C are reduced
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
      const float2 cl = cmul(m, c.wlo[t]);
      const float2 ch = cmul(m, c.whi[t]);
      v[0] = csub(v[0], cl);
      v[E - 1] = csub(v[E - 1], ch);
    }
#pragma unroll
    for (int e = 0; e < E; ++e) {
      acc[e] = fmaf(v[e].x, v[e].x, acc[e]);
      acc[e] = fmaf(v[e].y, v[e].y, acc[e]);
    }
#pragma unroll
    for (int i = 0; i < EH; ++i) A[i] = C[i];
    carry = true;
    if (tot != nullptr && ++npairs == kFoldPairs) {
      npairs = 0;
      fold_block<E, P>(acc, tot, t);
    }
  };
  if constexpr (SPLIT) {
    int s = s0;
    for (; s + 1 < s1; s += 2) step(s, std::true_type{});
    if (s < s1) step(s, std::false_type{});
  } else {
    for (int s = s0; s < s1; s += 2) step(s, s + 1 < s1);
  }
}

// Load the low-bin window spectrum for the spectral detrend: lo[i] = DFT(win)_i and
// hi[i] = DFT(win)_{L-P+i} = conj(DFT(win)_{P-i}) (real window), zero at and beyond n_low.
template <int P>
__device__ __forceinline__ void load_window_lowbins(float2* lo, float2* hi, const float2* wdft,
                                                    int n_low, int tid, int nthreads) {
  for (int i = tid; i < P; i += nthreads) {
    lo[i] = (wdft != nullptr && i < n_low) ? wdft[i] : make_float2(0.f, 0.f);
    const int km = P - i;
    hi[i] = (wdft != nullptr && km < n_low) ? cconj(wdft[km]) : make_float2(0.f, 0.f);
  }
}

template <int LOG_L, int LOG_E, int DET, bool BLOCKED>
__global__ void __launch_bounds__(MeanCfg<LOG_L, LOG_E>::THREADS, MeanCfg<LOG_L, LOG_E>::MIN_CTAS)
    k_welch_half(MeanParams pr) {
  using CFG = MeanCfg<LOG_L, LOG_E>;
  using PL = typename CFG::PL;
  constexpr int L = PL::L, E = PL::E, P = PL::P;
  constexpr bool WT = HalfWinT<PL>::USE;
  extern __shared__ float4 smem[];
  float* win1 = reinterpret_cast<float*>(smem + CFG::TEAMS * CFG::SCRATCH);
  float2* wlo = reinterpret_cast<float2*>(win1 + HalfSmem<CFG>::WINF);  // DFT(win)_t, t < P
  float2* whi = wlo + P;                                              // DFT(win)_{L-P+t}
  float2* tw = whi + P;
  float2* sbuf = tw + PL::TW;
  // the twiddles come from a constant table; everything the caller passes (window, window
  // spectrum, signal) is read only after the stream's previous kernel has completed: the kernel
  // may be launched as a programmatic dependent of it (launch_half)
  build_twiddles<PL>(tw, threadIdx.x, blockDim.x);
  pdl_wait();
  if constexpr (WT) {
    build_half_wint<PL>(win1, pr.win, threadIdx.x);
  } else {
    for (int i = threadIdx.x; i < L; i += blockDim.x) win1[i] = pr.win[i];
  }
  if constexpr (DET == kDetrendConstantSpectral)
    load_window_lowbins<P>(wlo, whi, pr.wdft, pr.n_low, threadIdx.x, blockDim.x);
  __syncthreads();
  pdl_trigger();
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
  int64_t g = tau * pr.G;
  const int64_t gend = min(g + pr.G, pr.total);
  // block totals (BLOCKED: ranges longer than kDirectPairs pairs)
  float* tot = BLOCKED ? reinterpret_cast<float*>(sbuf + CFG::TEAMS * PL::BUF) + team * L : nullptr;
  float acc[E];
#pragma unroll
  for (int e = 0; e < E; ++e) acc[e] = 0.f;
  while (g < gend) {
    const int64_t r = g / pr.nseg;
    const int s0 = int(g - r * pr.nseg);
    const int64_t lim = int64_t(s0) + (gend - g);
    const int s1 = int(lim < pr.nseg ? lim : int64_t(pr.nseg));
    if constexpr (BLOCKED) zero_total<E, P>(tot, c.t);
    welch_half_range<PL, DET, WT>(c, pr.x + r * pr.ld_x, s0, s1, acc, tot);
    if constexpr (BLOCKED) {
#pragma unroll
      for (int e = 0; e < E; ++e) acc[e] += tot[e * P + c.t];
    }
    const int64_t slot = tau - first_team(r, pr.nseg, pr.G);
    flush_mirror<PL>(acc, pr.partial + (r * pr.cmax + slot) * int64_t(welch_slot_floats(L)),
                     c.buf, c.t, c.mask);
    g += s1 - s0;
  }
}

// Partial-slot layout of the cross kernel: Q[cross_q_floats(L)] (|Z_k|^2, padded to an even
// count so the complex section stays 8-byte aligned) then C[L/2+1] complex.
__host__ __device__ constexpr int cross_q_floats(int L) { return L + (L & 1); }
__host__ __device__ constexpr int cross_slot_floats(int L) {
  return cross_q_floats(L) + 2 * (L / 2 + 1);
}

// Blocked summation of the cross kernels: each thread sums kFoldSegs segments' terms in FP32
// registers, then the team adds that block into its FP64 partial slot (a plain store for the
// first block of a row range, fire-and-forget FP64 reductions after it; only the owning team
// writes a slot). A team's sum then rounds in FP32 over at most kFoldSegs terms
// and in FP64 across blocks, whatever the number of segments; k_reduce_mean sums the FP64 slots.
// (The welch kernels keep their block totals in shared memory; the cross kernels' Q and C
// accumulators would need about 2 L floats per team there, which would cost a CTA per SM.)
constexpr int kFoldSegs = 32;

// The block is staged in the team's exchange buffer (free between segments; it holds the
// slot's 2 L + 2 floats) and added from there by a strided loop, which keeps the FP64 work off
// the registers of the segment loop.
template <class PL, int EH1>
__device__ __forceinline__ void flush_cross_f64(float (&q)[PL::E], float (&cr)[EH1],
                                                float (&ci)[EH1], double* slot, float2* buf, int t,
                                                unsigned mask, bool first) {
  constexpr int L = PL::L, E = PL::E, P = PL::P, CQ = cross_q_floats(L);
  if constexpr (PL::BUF * 2 < cross_slot_floats(L)) {
    // short transforms (L < 16: no padding in the exchange buffer): each thread adds its own
    // elements directly
#pragma unroll
    for (int e = 0; e < E; ++e) {
      double* d = slot + t + e * P;
      if (first) *d = double(q[e]);
      else atomicAdd(d, double(q[e]));
      q[e] = 0.f;
    }
#pragma unroll
    for (int e = 0; e < EH1; ++e) {
      if (e < E / 2 || t == 0) {
        double* d = slot + CQ + 2 * (t + e * P);
        if (first) {
          d[0] = double(cr[e]);
          d[1] = double(ci[e]);
        } else {
          atomicAdd(d, double(cr[e]));
          atomicAdd(d + 1, double(ci[e]));
        }
      }
      cr[e] = ci[e] = 0.f;
    }
    if ((L & 1) && t == 0 && first) slot[L] = 0.0;
    return;
  }
  float* sq = reinterpret_cast<float*>(buf);
#pragma unroll
  for (int e = 0; e < E; ++e) {
    sq[t + e * P] = q[e];
    q[e] = 0.f;
  }
#pragma unroll
  for (int e = 0; e < EH1; ++e) {
    if (e < E / 2 || t == 0) {
      sq[CQ + 2 * (t + e * P)] = cr[e];
      sq[CQ + 2 * (t + e * P) + 1] = ci[e];
    }
    cr[e] = ci[e] = 0.f;
  }
  if (L & 1) sq[L] = 0.f;  // the padding float of Q
  team_sync<P>(mask);
  if (first) {
    for (int i = t; i < cross_slot_floats(L); i += P) slot[i] = double(sq[i]);
  } else {
    for (int i = t; i < cross_slot_floats(L); i += P) atomicAdd(slot + i, double(sq[i]));
  }
  team_sync<P>(mask);
}

// csd / coherence: z = x_s + i y_s. Accumulates Q_k = sum |Z_k|^2 (all k) and
// C_k = sum Z_k Z_{L-k} for k in [0, L/2] (C is symmetric in k <-> L-k), blocked into FP64
// partial slots (flush_cross_f64).
template <int LOG_L, int LOG_E, int DET>
__global__ void __launch_bounds__(MeanCfg<LOG_L, LOG_E>::THREADS)
    k_cross_mean(MeanParams pr) {
  using CFG = MeanCfg<LOG_L, LOG_E>;
  using PL = typename CFG::PL;
  constexpr int L = PL::L, E = PL::E, P = PL::P, EH = E / 2 + 1;
  const MeanSmem sm = mean_smem_setup<CFG>(pr.win, pr.nperseg);
  const int team = threadIdx.x / P, t = threadIdx.x - team * P;
  const unsigned mask = team_mask<P>();
  float4* scratch = sm.scratch + team * CFG::SCRATCH;
  float2* buf = sm.buf + team * PL::BUF;
  const int64_t tau = int64_t(blockIdx.x) * CFG::TEAMS + team;
  int64_t g = tau * pr.G;
  const int64_t gend = min(g + pr.G, pr.total);
  float q[E];
  float cr[EH], ci[EH];
#pragma unroll
  for (int e = 0; e < E; ++e) q[e] = 0.f;
#pragma unroll
  for (int e = 0; e < EH; ++e) cr[e] = ci[e] = 0.f;
  while (g < gend) {
    const int64_t r = g / pr.nseg;
    const int s0 = int(g - r * pr.nseg);
    const int64_t lim = int64_t(s0) + (gend - g);
    const int s1 = int(lim < pr.nseg ? lim : int64_t(pr.nseg));
    const float* xr = pr.x + r * pr.ld_x;
    const float* yr = pr.y + r * pr.ld_y;
    const int64_t slot = tau - first_team(r, pr.nseg, pr.G);
    double* dslot = reinterpret_cast<double*>(pr.partial) +
                    (r * pr.cmax + slot) * int64_t(cross_slot_floats(L));
    bool first = true;
    int nblk = 0;
    for (int s = s0; s < s1; ++s) {
      float2 v[E];
      load_pair<PL>(v, xr + int64_t(s) * pr.hop, yr + int64_t(s) * pr.hop, true, t, pr.nperseg);
      detrend_window<PL, DET>(v, sm.win, t, pr.nperseg, scratch, mask);
      team_pass0<PL>(v);
      team_passes<PL>(v, buf, sm.tw, t, mask);
      // mirror exchange through the (now free) buffer: the mirrors L - k of the bins k <= L/2
      // read below sit in registers e >= E/2 (bin 0 is its own mirror)
#pragma unroll
      for (int e = 0; e < E; ++e) {
        q[e] = fmaf(v[e].x, v[e].x, q[e]);
        q[e] = fmaf(v[e].y, v[e].y, q[e]);
      }
#pragma unroll
      for (int e = E / 2; e < E; ++e) buf[PL::pad(t + e * P)] = v[e];
      if (t == 0) buf[0] = v[0];
      team_sync<P>(mask);
#pragma unroll
      for (int e = 0; e < EH; ++e) {
        if (e < E / 2 || t == 0) {
          const int k = t + e * P;
          const float2 m = buf[PL::pad((L - k) & (L - 1))];
          cr[e] = fmaf(v[e].x, m.x, fmaf(-v[e].y, m.y, cr[e]));
          ci[e] = fmaf(v[e].x, m.y, fmaf(v[e].y, m.x, ci[e]));
        }
      }
      team_sync<P>(mask);
      if (++nblk == kFoldSegs) {
        flush_cross_f64<PL, EH>(q, cr, ci, dslot, buf, t, mask, first);
        first = false;
        nblk = 0;
      }
    }
    if (first || nblk) flush_cross_f64<PL, EH>(q, cr, ci, dslot, buf, t, mask, first);
    g += s1 - s0;
  }
}

// 50%-overlap csd / coherence (nperseg == nfft == L, hop == L/2), z = x_s + i y_s per segment:
// segment s = A | B where A is the previous segment's B. The window multiply is fused into the
// first radix-2 stage (which pairs n with n + L/2, i.e. A with B), from the transposed window
// table; the segment means come from the carried half-block sum plus the new one; the constant
// detrend runs inside the fused stage (DET == kDetrendConstant) or as the low-bin spectral
// correction Z_k -= (m_x + i m_y) DFT(win)_k (DET == kDetrendConstantSpectral); the next
// half-block is prefetched into L2. Partial slots are those of k_cross_mean (FP64 Q_k for all k,
// C_k = Z_k Z_{L-k} for k <= L/2, blocked every kFoldSegs segments); CSD accumulates only Im C
// (its real part stays zero: csd does not read it).
template <int LOG_L, int LOG_E, int DET, bool CSD>
__global__ void __launch_bounds__(MeanCfg<LOG_L, LOG_E>::THREADS, MeanCfg<LOG_L, LOG_E>::MIN_CTAS)
    k_cross_half(MeanParams pr) {
  using CFG = MeanCfg<LOG_L, LOG_E>;
  using PL = typename CFG::PL;
  constexpr int L = PL::L, E = PL::E, P = PL::P, H = L / 2, EH = E / 2, EH1 = E / 2 + 1;
  constexpr int R0 = PL::radix(0), B0 = E / R0;
  constexpr bool WT = HalfWinT<PL>::USE;
  extern __shared__ float4 smem[];
  float* win1 = reinterpret_cast<float*>(smem + CFG::TEAMS * CFG::SCRATCH);
  float2* wlo = reinterpret_cast<float2*>(win1 + HalfSmem<CFG>::WINF);
  float2* whi = wlo + P;
  float2* tw = whi + P;
  float2* sbuf = tw + PL::TW;
  // the twiddles come from a constant table; everything the caller passes (window, window
  // spectrum, signal) is read only after the stream's previous kernel has completed: the kernel
  // may be launched as a programmatic dependent of it (launch_half)
  build_twiddles<PL>(tw, threadIdx.x, blockDim.x);
  pdl_wait();
  if constexpr (WT) {
    build_half_wint<PL>(win1, pr.win, threadIdx.x);
  } else {
    for (int i = threadIdx.x; i < L; i += blockDim.x) win1[i] = pr.win[i];
  }
  if constexpr (DET == kDetrendConstantSpectral)
    load_window_lowbins<P>(wlo, whi, pr.wdft, pr.n_low, threadIdx.x, blockDim.x);
  __syncthreads();
  pdl_trigger();
  const int team = threadIdx.x / P, t = threadIdx.x - team * P;
  const unsigned mask = team_mask<P>();
  float4* scratch = smem + team * CFG::SCRATCH;
  float2* buf = sbuf + team * PL::BUF;
  const float4* wt = reinterpret_cast<const float4*>(win1) + t * (HalfWinT<PL>::WS / 4);
  const int64_t tau = int64_t(blockIdx.x) * CFG::TEAMS + team;
  int64_t g = tau * pr.G;
  const int64_t gend = min(g + pr.G, pr.total);
  const float inv_n = 1.0f / float(L);
  float q[E];
  float cr[EH1], ci[EH1];
#pragma unroll
  for (int e = 0; e < E; ++e) q[e] = 0.f;
#pragma unroll
  for (int e = 0; e < EH1; ++e) cr[e] = ci[e] = 0.f;
  while (g < gend) {
    const int64_t r = g / pr.nseg;
    const int s0 = int(g - r * pr.nseg);
    const int64_t lim = int64_t(s0) + (gend - g);
    const int s1 = int(lim < pr.nseg ? lim : int64_t(pr.nseg));
    const float* xr = pr.x + r * pr.ld_x;
    const float* yr = pr.y + r * pr.ld_y;
    const int64_t slot = tau - first_team(r, pr.nseg, pr.G);
    double* dslot = reinterpret_cast<double*>(pr.partial) +
                    (r * pr.cmax + slot) * int64_t(cross_slot_floats(L));
    bool first = true;
    int nblk = 0;
    float sax = 0.f, say = 0.f;  // sums of this segment's A half (the previous B)
    bool have_a = false;
    for (int s = s0; s < s1; ++s) {
      const float* ax = xr + int64_t(s) * H;
      const float* ay = yr + int64_t(s) * H;
      if (s + 2 < s1) {  // warm L2 with the next segment's new half-block
        for (int o = t * 32; o < H; o += P * 32) {
          asm volatile("prefetch.global.L2 [%0];" ::"l"(ax + 2 * H + o));
          asm volatile("prefetch.global.L2 [%0];" ::"l"(ay + 2 * H + o));
        }
      }
      float Ax[EH], Ay[EH], Bx[EH], By[EH];
      static_for<0, EH>([&](auto gc) {
        constexpr int gi = decltype(gc)::value;
        const int n = slot_elem<PL, 2 * gi>(t);
        Ax[gi] = __ldg(ax + n);
        Ay[gi] = __ldg(ay + n);
        Bx[gi] = __ldg(ax + H + n);
        By[gi] = __ldg(ay + H + n);
      });
      float mx = 0.f, my = 0.f;
      if constexpr (DET == kDetrendConstant || DET == kDetrendConstantSpectral) {
        float sb[2] = {tree_sum<EH>([&](auto gc) { return Bx[decltype(gc)::value]; }),
                       tree_sum<EH>([&](auto gc) { return By[decltype(gc)::value]; })};
        if (!have_a) {
          float s4[4] = {tree_sum<EH>([&](auto gc) { return Ax[decltype(gc)::value]; }),
                         tree_sum<EH>([&](auto gc) { return Ay[decltype(gc)::value]; }), sb[0],
                         sb[1]};
          team_sum<P, 4>(s4, scratch, mask);
          sax = s4[0];
          say = s4[1];
          sb[0] = s4[2];
          sb[1] = s4[3];
        } else {
          team_sum<P, 2>(sb, scratch, mask);
        }
        mx = (sax + sb[0]) * inv_n;
        my = (say + sb[1]) * inv_n;
        sax = sb[0];
        say = sb[1];
        have_a = true;
      }
      float2 v[E];
      auto fuse = [&](auto gc, float wl, float wh) {
        constexpr int gi = decltype(gc)::value;
        float2 zl = make_float2(Ax[gi], Ay[gi]);
        float2 zh = make_float2(Bx[gi], By[gi]);
        if constexpr (DET == kDetrendConstant) {
          zl = make_float2(zl.x - mx, zl.y - my);
          zh = make_float2(zh.x - mx, zh.y - my);
        }
        const float2 a = make_float2(zl.x * wl, zl.y * wl);
        v[2 * gi] = make_float2(fmaf(zh.x, wh, a.x), fmaf(zh.y, wh, a.y));
        v[2 * gi + 1] = make_float2(fmaf(-zh.x, wh, a.x), fmaf(-zh.y, wh, a.y));
      };
      if constexpr (WT) {
        static_for<0, EH / 2>([&](auto pc) {
          constexpr int gp = decltype(pc)::value;
          const float4 w4 = wt[gp];
          fuse(std::integral_constant<int, 2 * gp>{}, w4.x, w4.y);
          fuse(std::integral_constant<int, 2 * gp + 1>{}, w4.z, w4.w);
        });
      } else {
        static_for<0, EH>([&](auto gc) {
          constexpr int gi = decltype(gc)::value;
          const int n = slot_elem<PL, 2 * gi>(t);
          fuse(gc, win1[n], win1[n + H]);
        });
      }
      static_for<0, B0>([&](auto bc) {
        constexpr int b = decltype(bc)::value;
        dft_dit<R0, b * R0, 2>(v);
      });
      team_passes<PL>(v, buf, tw, t, mask);
      if constexpr (DET == kDetrendConstantSpectral) {
        const float2 m = make_float2(mx, my);
        v[0] = csub(v[0], cmul(m, wlo[t]));
        v[E - 1] = csub(v[E - 1], cmul(m, whi[t]));
      }
      // |Z_k|^2 for every bin; Z_k Z_{L-k} for k <= L/2 through a mirror exchange
#pragma unroll
      for (int e = 0; e < E; ++e) {
        q[e] = fmaf(v[e].x, v[e].x, q[e]);
        q[e] = fmaf(v[e].y, v[e].y, q[e]);
      }
      // mirrors L - k of the bins k <= L/2 read below: registers e >= E/2, and bin 0 itself
#pragma unroll
      for (int e = E / 2; e < E; ++e) buf[PL::pad(t + e * P)] = v[e];
      if (t == 0) buf[0] = v[0];
      team_sync<P>(mask);
#pragma unroll
      for (int e = 0; e < EH1; ++e) {
        if (e < E / 2 || t == 0) {
          const int k = t + e * P;
          const float2 m = buf[PL::pad((L - k) & (L - 1))];
          if constexpr (!CSD) cr[e] = fmaf(v[e].x, m.x, fmaf(-v[e].y, m.y, cr[e]));
          ci[e] = fmaf(v[e].x, m.y, fmaf(v[e].y, m.x, ci[e]));
        }
      }
      team_sync<P>(mask);
      if (++nblk == kFoldSegs) {
        flush_cross_f64<PL, EH1>(q, cr, ci, dslot, buf, t, mask, first);
        first = false;
        nblk = 0;
      }
    }
    if (first || nblk) flush_cross_f64<PL, EH1>(q, cr, ci, dslot, buf, t, mask, first);
    g += s1 - s0;
  }
}

// Final reduction over partial slots (fixed order, FP64), mirror combination, one-sided
// doubling and 1/nseg. mode: 0 welch (float out), 1 csd (complex out), 2 coherence (float out).
struct ReduceParams {
  const float* partial;
  int64_t rows;
  int L;
  int nout;          // output bins per row
  int onesided;      // apply one-sided doubling (welch/csd)
  int nseg;
  int64_t G;
  int cmax;
  int64_t nteams;
  int mode;
  int f64;           // modes 1/2: FP64 partial slots (k_cross_mean / k_cross_half)
  float* out;
};

}  // namespace b2s
