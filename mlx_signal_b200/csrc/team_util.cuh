// Shared helpers for the framed-spectral kernels: team reductions, pairwise register sums,
// detrend of a register-resident segment, and the balanced segment-range work split.
#pragma once

#include "fft_core.cuh"

namespace b2s {

// Pairwise (tree) sum of a compile-time register range: error grows with log2(N), not N.
template <int N, int OFF = 0, class F>
__device__ __forceinline__ float tree_sum(F&& f) {
  if constexpr (N == 1) {
    return f(std::integral_constant<int, OFF>{});
  } else {
    return tree_sum<N / 2, OFF>(f) + tree_sum<N - N / 2, OFF + N / 2>(f);
  }
}

// Sum four floats across the P threads of a team. Teams of <= 32 threads are aligned lane
// groups of one warp (xor shuffles stay inside the team); larger teams are the whole CTA and
// go through `scratch` (>= P/32 float4, team-private).
template <int P>
__device__ __forceinline__ float4 team_sum4(float4 v, float4* scratch, unsigned mask) {
  if constexpr (P <= 32) {
#pragma unroll
    for (int off = P / 2; off > 0; off >>= 1) {
      v.x += __shfl_xor_sync(mask, v.x, off);
      v.y += __shfl_xor_sync(mask, v.y, off);
      v.z += __shfl_xor_sync(mask, v.z, off);
      v.w += __shfl_xor_sync(mask, v.w, off);
    }
    return v;
  } else {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      v.x += __shfl_xor_sync(0xffffffffu, v.x, off);
      v.y += __shfl_xor_sync(0xffffffffu, v.y, off);
      v.z += __shfl_xor_sync(0xffffffffu, v.z, off);
      v.w += __shfl_xor_sync(0xffffffffu, v.w, off);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) scratch[w] = v;
    __syncthreads();
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int i = 0; i < P / 32; ++i) {
      const float4 u = scratch[i];
      s.x += u.x; s.y += u.y; s.z += u.z; s.w += u.w;
    }
    __syncthreads();
    return s;
  }
}

// Sum NV floats (in place) across the P threads of a team; same layout rules as team_sum4.
template <int P, int NV>
__device__ __forceinline__ void team_sum(float (&v)[NV], float4* scratch, unsigned mask) {
  static_assert(NV <= 4, "at most four values per reduction");
  if constexpr (P <= 32) {
#pragma unroll
    for (int off = P / 2; off > 0; off >>= 1) {
#pragma unroll
      for (int i = 0; i < NV; ++i) v[i] += __shfl_xor_sync(mask, v[i], off);
    }
  } else {
    float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
    if constexpr (NV > 0) f.x = v[0];
    if constexpr (NV > 1) f.y = v[1];
    if constexpr (NV > 2) f.z = v[2];
    if constexpr (NV > 3) f.w = v[3];
    f = team_sum4<P>(f, scratch, mask);
    if constexpr (NV > 0) v[0] = f.x;
    if constexpr (NV > 1) v[1] = f.y;
    if constexpr (NV > 2) v[2] = f.z;
    if constexpr (NV > 3) v[3] = f.w;
  }
}

// Lane mask of the team containing this thread (teams of P <= 32 lanes are aligned groups).
template <int P>
__device__ __forceinline__ unsigned team_mask() {
  if constexpr (P >= 32) {
    return 0xffffffffu;
  } else {
    const unsigned base = (threadIdx.x & 31) & ~(unsigned)(P - 1);
    return ((1u << P) - 1u) << base;
  }
}

// Detrend kinds (scipy.signal.detrend semantics per segment). kDetrendConstantSpectral is the
// constant detrend applied after the FFT as Z_k -= m * DFT(win)_k, valid when the window's DFT
// vanishes outside a few low bins (hann, hamming, blackman, boxcar, ...).
enum : int {
  kDetrendNone = 0,
  kDetrendConstant = 1,
  kDetrendLinear = 2,
  kDetrendConstantSpectral = 3
};

// Element index of register slot `slot` in the pass-0 load pattern: slot = b*R0 + bitrev(q)
// holds element t + P*b + q*(L/R0).
template <class PL, int SLOT>
__device__ __forceinline__ int slot_elem(int t) {
  constexpr int R0 = PL::radix(0);
  constexpr int b = SLOT / R0;
  constexpr int q = bitrev(SLOT % R0, ilog2(R0));
  return t + PL::P * b + q * (PL::L / R0);
}

// Detrend and window two real segments packed as (re, im) = (segment a, segment b) in v,
// elements laid out in the pass-0 load pattern. `win` is the window zero-padded to L.
// Segment sums use pairwise register sums plus a team reduction; linear detrend subtracts the
// least-squares line over indices 0..nperseg-1 (scipy.signal.detrend type='linear').
template <class PL, int DET>
__device__ __forceinline__ void detrend_window(float2 (&v)[PL::E], const float* win, int t,
                                               int nperseg, float4* scratch, unsigned mask) {
  constexpr int E = PL::E;
  if constexpr (DET == kDetrendNone) {
    static_for<0, E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const float w = win[slot_elem<PL, e>(t)];
      v[e] = make_float2(v[e].x * w, v[e].y * w);
    });
  } else if constexpr (DET == kDetrendConstant) {
    const float sa = tree_sum<E>([&](auto ec) { return v[decltype(ec)::value].x; });
    const float sb = tree_sum<E>([&](auto ec) { return v[decltype(ec)::value].y; });
    const float4 s = team_sum4<PL::P>(make_float4(sa, sb, 0.f, 0.f), scratch, mask);
    const float inv = 1.0f / float(nperseg);
    const float ma = s.x * inv, mb = s.y * inv;
    static_for<0, E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const float w = win[slot_elem<PL, e>(t)];  // zero beyond nperseg
      v[e] = make_float2((v[e].x - ma) * w, (v[e].y - mb) * w);
    });
  } else {
    // linear: x - mean - slope*(n - c), c = (N-1)/2, slope = sum((n-c) x) / (N (N^2-1)/12)
    const float c = 0.5f * float(nperseg - 1);
    const float sa = tree_sum<E>([&](auto ec) { return v[decltype(ec)::value].x; });
    const float sb = tree_sum<E>([&](auto ec) { return v[decltype(ec)::value].y; });
    const float ta = tree_sum<E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const int n = slot_elem<PL, e>(t);
      return n < nperseg ? (float(n) - c) * v[e].x : 0.f;
    });
    const float tb = tree_sum<E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const int n = slot_elem<PL, e>(t);
      return n < nperseg ? (float(n) - c) * v[e].y : 0.f;
    });
    const float4 s = team_sum4<PL::P>(make_float4(sa, sb, ta, tb), scratch, mask);
    const double N = double(nperseg);
    const double denom = N * (N * N - 1.0) / 12.0;
    const float inv = 1.0f / float(nperseg);
    const float ka = denom > 0.0 ? float(double(s.z) / denom) : 0.f;
    const float kb = denom > 0.0 ? float(double(s.w) / denom) : 0.f;
    const float ma = s.x * inv, mb = s.y * inv;
    static_for<0, E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const int n = slot_elem<PL, e>(t);
      const float w = win[n];
      const float d = float(n) - c;
      v[e] = make_float2((v[e].x - ma - ka * d) * w, (v[e].y - mb - kb * d) * w);
    });
  }
}

// Balanced split of the flattened (row, segment) space over `nteams` teams: team tau owns
// global segments [tau*G, min((tau+1)*G, total)). A row r is touched by teams
// first_team(r) .. last_team(r); team tau writes its partial sums of row r into slot
// tau - first_team(r).
__host__ __device__ __forceinline__ int64_t first_team(int64_t r, int64_t nseg, int64_t G) {
  return (r * nseg) / G;
}
__host__ __device__ __forceinline__ int64_t last_team(int64_t r, int64_t nseg, int64_t G) {
  return ((r + 1) * nseg - 1) / G;
}

}  // namespace b2s
