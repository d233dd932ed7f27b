// Real transforms of length n = C * M (C odd in [3, 15], M = 2m, the packed length m a power of
// two in the three-pass range) by decimation in time around the power-of-two kernels:
//   forward:  D_s[q] = x[C q + s]                                   (k_mixed_deinterleave)
//             R_s = rfft_M(D_s) through the packed m-point three-pass transform
//             X_k = sum_s W_n^(s k) R_s[k mod M],  k in [0, n/2]     (k_mixed_combine: the
//             packed-transform untangle and the radix-C combine in one kernel)
//   inverse:  U_s[k1] = (1/C) W_n^(-s k1) sum_k2 W_C^(-s k2) Y[k1 + M k2],  k1 in [0, m]
//             (Y the Hermitian extension of the one-sided input), packed for the m-point
//             inverse with the irfft pretwist                         (k_mixed_fold_pretwist)
//             D_s = irfft_M(U_s) through the inverse three-pass transform
//             y[C q + s] = D_s[q]                                      (k_mixed_interleave)
// U_s is Hermitian because y is real, so each branch s needs only its one-sided half.
//
// Reference behaviour replaced: the reference's long transforms of a composite length split it
// into a divisor pair and run the four-step identity over MLX's own mixed-radix FFT
// (src/mlx_signal_processing/_fourstep.py:55-72 _choose_split, :177-231 fft_large/rfft_large,
// :372-408 irfft_large); here the odd factor C becomes one radix-C step fused into the
// untangle / pretwist kernels that the power-of-two path already runs.
//
// Twiddles: every W_n^k and W_C^t is formed in FP64 (sincospi of an exactly reduced phase, or an
// FP64 product of such values) and rounded to FP32 once; the radix-C sums run in FP32.
#pragma once

#include "fft3_kernels.cuh"

namespace b2s {

constexpr int kMaxMixC = 15;   // largest odd factor
constexpr int kMixQ = 512;     // samples per branch handled by one (de)interleave block
constexpr int kMixB = 256;     // threads per (de)interleave block

__device__ __forceinline__ float2 f2(double2 v) { return make_float2(float(v.x), float(v.y)); }
__device__ __forceinline__ double2 dconj(double2 v) { return make_double2(v.x, -v.y); }
__device__ __forceinline__ float2 fconj(float2 v) { return make_float2(v.x, -v.y); }

// D[(b C + s) M + q] = x[b C M + C q + s]: one block per (row, kMixQ-sample chunk); the chunk's
// C kMixQ contiguous samples are read as float4 into shared memory and written out as C
// coalesced branch rows (shared-memory stride C is odd: no bank conflicts).
__global__ void __launch_bounds__(kMixB) k_mixed_deinterleave(const float* __restrict__ x,
                                                              float* __restrict__ D, int C,
                                                              int64_t M) {
  __shared__ __align__(16) float sm[kMaxMixC * kMixQ];
  fft_pdl_wait();
  fft_pdl_trigger();
  const int64_t chunks = M / kMixQ;
  const int64_t b = blockIdx.x / chunks;
  const int64_t q0 = (blockIdx.x - b * chunks) * kMixQ;
  const float4* src = reinterpret_cast<const float4*>(x + b * C * M + C * q0);
  float4* sm4 = reinterpret_cast<float4*>(sm);
  for (int i = threadIdx.x; i < C * kMixQ / 4; i += kMixB) sm4[i] = src[i];
  __syncthreads();
  for (int s = 0; s < C; ++s) {
    float* dst = D + (b * C + s) * M + q0;
    for (int q = threadIdx.x; q < kMixQ; q += kMixB) dst[q] = sm[q * C + s];
  }
}

// y[b C M + C q + s] = D[(b C + s) M + q]: the inverse of k_mixed_deinterleave.
__global__ void __launch_bounds__(kMixB) k_mixed_interleave(const float* __restrict__ D,
                                                            float* __restrict__ y, int C,
                                                            int64_t M) {
  __shared__ __align__(16) float sm[kMaxMixC * kMixQ];
  fft_pdl_wait();
  fft_pdl_trigger();
  const int64_t chunks = M / kMixQ;
  const int64_t b = blockIdx.x / chunks;
  const int64_t q0 = (blockIdx.x - b * chunks) * kMixQ;
  for (int s = 0; s < C; ++s) {
    const float* src = D + (b * C + s) * M + q0;
    for (int q = threadIdx.x; q < kMixQ; q += kMixB) sm[q * C + s] = src[q];
  }
  __syncthreads();
  float4* dst = reinterpret_cast<float4*>(y + b * C * M + C * q0);
  const float4* sm4 = reinterpret_cast<const float4*>(sm);
  for (int i = threadIdx.x; i < C * kMixQ / 4; i += kMixB) dst[i] = sm4[i];
}

// FP64 W_C^t = exp(-2 pi i t / C), t in [0, C), into a shared table.
template <int C>
__device__ __forceinline__ void radix_table(double2* wc) {
  if (threadIdx.x < C) {
    double sn, cs;
    sincospi(-2.0 * double(threadIdx.x) / double(C), &sn, &cs);
    wc[threadIdx.x] = make_double2(cs, sn);
  }
}

// Untangle of the C packed branch transforms and the radix-C combine. Thread j in [0, m/2] of
// row b reads Z_s[j], Z_s[m-j] (s < C), forms R_s[j], R_s[m-j] (packed-real untangle,
// w_j = exp(-i pi j/m)) and their mirrors R_s[M-j] = conj R_s[j], R_s[m+j] = conj R_s[m-j], and
// writes every output k = rho + M k2 (k < nout) of the residues rho in {j, m-j, m+j, 2m-j} as
//   X_k = sum_s omega^s R_s[rho],  omega = W_n^k = W_n^rho W_C^k2  (Horner in FP32).
// a = W_n^m (FP64) relates the residues' twiddles: W_n^(m-j) = a conj(W_n^j), W_n^(m+j) =
// a W_n^j, W_n^(2m-j) = a^2 conj(W_n^j).
template <int C>
__global__ void __launch_bounds__(kUntB) k_mixed_combine(const float2* __restrict__ Z,
                                                         float2* __restrict__ X, int64_t m,
                                                         int64_t ldx, int64_t nout, double2 a) {
  __shared__ double2 wc[C];
  radix_table<C>(wc);
  __syncthreads();
  fft_pdl_wait();
  fft_pdl_trigger();
  const int64_t half = m / 2 + 1;
  const int64_t per_row = (half + kUntB - 1) / kUntB;
  const int64_t b = blockIdx.x / per_row;
  const int64_t j = (blockIdx.x - b * per_row) * kUntB + threadIdx.x;
  if (j >= half) return;
  const int64_t M = 2 * m;
  float2 rj[C], rmj[C];  // R_s[j], R_s[m - j]
  {
    float2 zk[C], zm[C];
#pragma unroll
    for (int s = 0; s < C; ++s) {  // every read first: 2C loads in flight
      const float2* z = Z + (b * C + s) * m;
      zk[s] = z[j];
      zm[s] = j ? z[m - j] : zk[s];
    }
    double sn, cs;
    sincospi(-double(j) / double(m), &sn, &cs);
    const float2 w = make_float2(float(cs), float(sn));
#pragma unroll
    for (int s = 0; s < C; ++s) {
      if (j == 0) {
        rj[s] = make_float2(zk[s].x + zk[s].y, 0.f);   // R_s[0]
        rmj[s] = make_float2(zk[s].x - zk[s].y, 0.f);  // R_s[m]
      } else {
        const float2 ze = make_float2(0.5f * (zk[s].x + zm[s].x), 0.5f * (zk[s].y - zm[s].y));
        const float2 zo = make_float2(0.5f * (zk[s].x - zm[s].x), 0.5f * (zk[s].y + zm[s].y));
        const float2 wz = cmul(w, zo);
        rj[s] = make_float2(ze.x + wz.y, ze.y - wz.x);
        rmj[s] = make_float2(ze.x - wz.y, -ze.y - wz.x);  // conj(ze) - i conj(w zo)
      }
    }
  }
  double sn, cs;
  sincospi(-2.0 * double(j) / double(C * M), &sn, &cs);
  const double2 wn = make_double2(cs, sn);  // W_n^j
  float2* x = X + b * ldx;
  // residue r: 0 -> j, 1 -> m-j, 2 -> m+j, 3 -> 2m-j (duplicates skipped at j = 0 and 2j = m)
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    if (j == 0 && r >= 2) break;
    if (2 * j == m && (r == 1 || r == 3)) continue;
    const int64_t rho = r == 0 ? j : r == 1 ? m - j : r == 2 ? m + j : 2 * m - j;
    const double2 wr = r == 0 ? wn : r == 1 ? zmul(a, dconj(wn))
                               : r == 2 ? zmul(a, wn) : zmul(zmul(a, a), dconj(wn));
    for (int k2 = 0; k2 < C; ++k2) {
      const int64_t k = rho + M * k2;
      if (k >= nout) continue;
      const float2 om = f2(zmul(wr, wc[k2]));
      float2 acc = r == 0 ? rj[C - 1] : r == 1 ? rmj[C - 1]
                          : r == 2 ? fconj(rmj[C - 1]) : fconj(rj[C - 1]);
#pragma unroll
      for (int s = C - 2; s >= 0; --s) {
        const float2 v = r == 0 ? rj[s] : r == 1 ? rmj[s] : r == 2 ? fconj(rmj[s]) : fconj(rj[s]);
        acc = make_float2(fmaf(acc.x, om.x, fmaf(-acc.y, om.y, v.x)),
                          fmaf(acc.x, om.y, fmaf(acc.y, om.x, v.y)));
      }
      x[k] = acc;
    }
  }
}

// Radix-C fold of the one-sided input and the packed irfft pretwist of each branch. Thread j in
// [0, m/2] of row b builds, for k1 in {j, m-j}, the C values Y[k1 + M k2] of the Hermitian
// extension of X (bins >= nbins are zero, the imaginary parts of bins 0 and n/2 are dropped,
// bin kfix is multiplied by ffix, everything by scale), their radix-C inverse DFT
//   U_s[k1] = (scale/C) W_n^(-s k1) sum_k2 W_C^(-s k2) Y[k1 + M k2],
// and then, per branch s, the pretwist of (U_s[j], U_s[m-j]) into row b C + s of Yp (the input
// of the m-point inverse transform; the packed result interleaves irfft_M(U_s)).
template <int C>
__global__ void __launch_bounds__(kUntB) k_mixed_fold_pretwist(
    const float2* __restrict__ X, int64_t ldx, int64_t nbins, float2* __restrict__ Yp, int64_t m,
    double2 a, float scale, int64_t kfix, float ffix) {
  __shared__ double2 wc[C];
  __shared__ float2 wci[C];  // W_C^(-t) in FP32
  radix_table<C>(wc);
  __syncthreads();
  if (threadIdx.x < C) wci[threadIdx.x] = f2(dconj(wc[threadIdx.x]));
  __syncthreads();
  fft_pdl_wait();
  fft_pdl_trigger();
  const int64_t half = m / 2 + 1;
  const int64_t per_row = (half + kUntB - 1) / kUntB;
  const int64_t b = blockIdx.x / per_row;
  const int64_t j = (blockIdx.x - b * per_row) * kUntB + threadIdx.x;
  if (j >= half) return;
  const int64_t M = 2 * m, n = C * M, nh = C * m;
  const float2* x = X + b * ldx;
  auto getx = [&](int64_t k) -> float2 {  // k in [0, n/2]
    if (k >= nbins) return make_float2(0.f, 0.f);
    float2 v = x[k];
    if (k == 0 || k == nh) v.y = 0.f;
    if (k == kfix) v = make_float2(v.x * ffix, v.y * ffix);
    return v;
  };
  auto gety = [&](int64_t k) -> float2 { return k <= nh ? getx(k) : fconj(getx(n - k)); };
  double sn, cs;
  sincospi(-2.0 * double(j) / double(n), &sn, &cs);
  const double2 wn = make_double2(cs, sn);  // W_n^j
  const float sc = scale / float(C);
  float2 u0[C], u1[C];  // U_s[j], U_s[m - j]
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int64_t k1 = h == 0 ? j : m - j;
    float2 yv[C];
#pragma unroll
    for (int k2 = 0; k2 < C; ++k2) yv[k2] = gety(k1 + M * k2);
    // W_n^(-k1): conj(W_n^j) for k1 = j; conj(a conj(W_n^j)) = conj(a) W_n^j for k1 = m - j
    const double2 base = h == 0 ? dconj(wn) : zmul(dconj(a), wn);
    double2 p = make_double2(1.0, 0.0);
#pragma unroll
    for (int s = 0; s < C; ++s) {
      float2 v = make_float2(0.f, 0.f);
#pragma unroll
      for (int k2 = 0; k2 < C; ++k2) {
        const float2 t = wci[(s * k2) % C];
        v = make_float2(fmaf(yv[k2].x, t.x, fmaf(-yv[k2].y, t.y, v.x)),
                        fmaf(yv[k2].x, t.y, fmaf(yv[k2].y, t.x, v.y)));
      }
      float2 u = cmul(f2(p), v);
      u = make_float2(u.x * sc, u.y * sc);
      if (h == 0) u0[s] = u; else u1[s] = u;
      p = zmul(p, base);
    }
  }
  // pretwist per branch (w_j = exp(-i pi j/m)); U_s[0] and U_s[m] are real
  sincospi(-double(j) / double(m), &sn, &cs);
  const float c = float(cs), sf = float(sn);
#pragma unroll
  for (int s = 0; s < C; ++s) {
    float2 xk = u0[s], xm = u1[s];
    if (j == 0) {
      xk.y = 0.f;
      xm.y = 0.f;
    }
    float2* y = Yp + (b * C + s) * m;
    const float2 wcj = make_float2(c, -sf);
    const float2 e1 = make_float2(0.5f * (xk.x + xm.x), 0.5f * (xk.y - xm.y));
    const float2 o1 = make_float2(0.5f * (xk.x - xm.x), 0.5f * (xk.y + xm.y));
    const float2 t1 = cmul(wcj, o1);
    y[j] = make_float2(e1.x - t1.y, e1.y + t1.x);
    if (j != 0 && 2 * j != m) {
      const float2 e2 = make_float2(e1.x, -e1.y);
      const float2 o2 = make_float2(-o1.x, o1.y);
      const float2 t2 = cmul(make_float2(-c, -sf), o2);
      y[m - j] = make_float2(e2.x - t2.y, e2.y + t2.x);
    }
  }
}

}  // namespace b2s
