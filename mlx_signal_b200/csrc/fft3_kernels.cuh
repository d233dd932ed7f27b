// Three-pass (Bailey) power-of-two complex FFT for long transforms, N = R3 * R2 * R1, plus the
// packed real-input untangle and its inverse.
//
// Reference behaviour replaced: _fourstep_metal.fft3_last (src/mlx_signal_processing/
// _fourstep_metal.py:272-303, kernel sources _P1/_P2/_P3_SRC :90-185) and the large real
// transforms of _fourstep.py (rfft_large :213-231 with _rfft_untangle :195-210, irfft_large
// :372-408). Same index maps (the four-step identity applied twice):
//     n = (m3 R2 + m2) R1 + r,   k = kr (R2 R3) + km2 R3 + km3
//     x[m3][m2][r] -> S1[m2][r][km3] -> S2[km2][r][km3] -> X[kr][km2][km3]
//     pass 1: DFT_R3 over m3, twiddle W_N^(R1 m2 km3)      (= W_{R2 R3}^(m2 km3))
//     pass 2: DFT_R2 over m2, twiddle W_N^(r (km2 R3 + km3))
//     pass 3: DFT_R1 over r
// Differences by design:
//  * every pass stages a 16-column x L-row tile into shared memory with TMA bulk tensor copies
//    (cp.async.bulk.tensor, 128B swizzle, mbarrier completion, no multicast), so the strided
//    column walk of the reference's per-thread gather becomes one coalesced bulk transfer;
//  * each tile column is an L-point team FFT in registers (the spectral kernels' engine);
//  * inter-pass twiddles are formed in FP64 and rounded to FP32 once: pass 1 from a per-tile
//    shared-memory table (an FP64 sincospi of the exactly reduced integer phase per output row,
//    filled while the tile's copy is in flight), pass 2 per thread from an FP64 anchor and step
//    (sincospi of exact integer phases) and an FP64 recurrence over the thread's rows -- no
//    twiddle table in global memory;
//  * the inverse transform is conj(FFT(conj(x))) / N with 1/N folded into pass 1.
// Every mbarrier wait is bounded; on timeout the CTA records SP_ERR_TIMEOUT in the error word,
// waits (bounded) for its own copies and returns without touching the data; the code is also
// stored in a process-wide word in mapped pinned host memory (sp_fft_sticky_error). The limit of
// the wait for each tile is a launch parameter (sp_fft_set_wait_limit), so a host watchdog test
// can make it run out.
#pragma once

#include <cuda.h>

#include "b200signal.h"
#include "fft_core.cuh"
#include "team_util.cuh"

namespace b2s {

struct Fft3Params {
  const float2* in;    // pass input (pass 1: the signal)
  float2* out;         // pass output
  int R1, R2, R3;      // digits, N = R3 * R2 * R1
  int log_n;
  int64_t N;
  int batch;
  int inverse;         // 1: conj on load (pass 1) and on store (pass 3), scale 1/N in pass 1
  int* err;            // device error word (0 = ok)
  int* sticky;         // process-wide word in mapped pinned host memory (or null): a timeout
                       // also lands here, so a host watchdog reads it without a copy
  int ntiles;          // tiles of this pass (a persistent CTA walks tile, tile + gridDim.x, ...)
  uint32_t wait_polls; // poll limit of the wait for each tile's copy (kMbarSpinLimit by default)
};

// Programmatic dependent launch: the passes and the untangle kernels are launched as dependents
// of the stream's previous kernel; each builds what needs no input, waits for the previous grid
// to complete, then lets its own dependent start its prologue.
__device__ __forceinline__ void fft_pdl_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}
__device__ __forceinline__ void fft_pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

constexpr int kTileCols = 16;                  // columns per tile: 16 complex = 128 B rows
constexpr uint32_t kMbarSpinLimit = 1u << 22;  // bounded mbarrier polling

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// true when the phase with parity `parity` has completed; at most `polls` polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          uint32_t polls = kMbarSpinLimit) {
  uint32_t done = 0;
  for (uint32_t it = 0; it < polls; ++it) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 3-D tiled TMA load of one box at coordinates {c0, c1, c2} (no multicast).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

// 3-D tiled TMA store of one box from shared memory at coordinates {c0, c1, c2} (bulk group).
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* src, int c0,
                                             int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
          reinterpret_cast<uint64_t>(map)),
      "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

// Element (row, col) of a tile whose 128-byte rows were written with the 128B swizzle: the
// 16-byte chunk index is XORed with (row mod 8).
__device__ __forceinline__ int swz(int row, int col) {
  return row * kTileCols + ((((col >> 1) ^ (row & 7)) << 1) | (col & 1));
}

// FP64 W_N^p = exp(-2 pi i p / N) from the exactly reduced integer phase.
__device__ __forceinline__ double2 w_exact(int64_t p, int64_t N) {
  p %= N;
  double s, c;
  sincospi(-2.0 * double(p) / double(N), &s, &c);
  return make_double2(c, s);
}

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

template <int LOG_L, int LOG_E>
struct Fft3Cfg {
  using PL = Plan<LOG_L, LOG_E>;
  static constexpr int L = PL::L;
  static constexpr int THREADS = kTileCols * PL::P;
  static constexpr int TILE_BYTES = L * kTileCols * 8;
  static constexpr int XBUF_BYTES = kTileCols * PL::BUF * 8;
  // A slot holds a TMA tile and, once every team has its column in registers, the teams'
  // exchange buffers: sized for the larger of the two, in whole 1024-byte swizzle units.
  static constexpr int SLOT_BYTES =
      ((TILE_BYTES > XBUF_BYTES ? TILE_BYTES : XBUF_BYTES) + 1023) / 1024 * 1024;
  // alignment slack | two slots (1024-byte aligned for the swizzle) | team twiddles |
  // per-tile inter-pass twiddles (L + kTileCols float2; passes 1 and 2) | 2 mbarriers
  static constexpr size_t smem(int pass) {
    return 1024 + 2 * size_t(SLOT_BYTES) + size_t(PL::TW) * 8 +
           (pass == 3 ? 0 : size_t(L + kTileCols) * 8) + 16;
  }
  // CTAs per SM that the shared memory allows (228 KB per SM, 1 KB reserved per CTA, at most
  // 2048 threads), asked of the register allocator for columns of 128 points and more; shorter
  // columns (whose pass-2 code would spill under that bound) keep the default.
  static constexpr int min_blocks(int pass) {
    const int by_smem = int((228u * 1024u) / (smem(pass) + 1024));
    const int by_threads = 2048 / THREADS;
    const int b = by_smem < by_threads ? by_smem : by_threads;
    return (L < 128 || b < 1) ? 1 : b;
  }
};

// One pass of the three-pass FFT. PASS 1: tile rows m3 (L = R3), columns r; PASS 2: rows m2
// (L = R2), columns km3; PASS 3: rows r (L = R1), columns km3.
// Persistent and double-buffered: a CTA walks tiles blockIdx.x, blockIdx.x + gridDim.x, ...;
// before waiting for tile i it issues the TMA load of tile i+1 into the other buffer, so the
// copy overlaps the FFT of tile i. The u-th completion of buffer j's mbarrier is phase u & 1.
template <int PASS>
__device__ __forceinline__ void fft3_tile_coords(int tile, int R1, int R2, int R3, int* cg,
                                                 int* slab, int* b) {
  const int colgroups = (PASS == 1 ? R1 : R3) / kTileCols;
  const int slabs = PASS == 1 ? R2 : (PASS == 2 ? R1 : R2);
  *cg = tile % colgroups;
  tile /= colgroups;
  *slab = tile % slabs;
  *b = tile / slabs;
}

template <int LOG_L, int LOG_E, int PASS>
__global__ void __launch_bounds__(Fft3Cfg<LOG_L, LOG_E>::THREADS,
                                  Fft3Cfg<LOG_L, LOG_E>::min_blocks(PASS))
    k_fft3_pass(const __grid_constant__ CUtensorMap src, const __grid_constant__ CUtensorMap dst,
                Fft3Params pr) {
  using CFG = Fft3Cfg<LOG_L, LOG_E>;
  using PL = typename CFG::PL;
  constexpr int L = PL::L, E = PL::E, P = PL::P;
  static_assert(CFG::SLOT_BYTES >= CFG::TILE_BYTES && CFG::SLOT_BYTES >= CFG::XBUF_BYTES &&
                    CFG::SLOT_BYTES % 1024 == 0,
                "a slot holds the TMA tile and every team's exchange buffer, swizzle-aligned");
  static_assert(CFG::smem(PASS) <= 227u * 1024u, "pass exceeds the shared memory of one CTA");
  extern __shared__ __align__(16) unsigned char smraw[];
  // 1024-byte alignment for the swizzle, as an offset into the shared array (so every pointer
  // below stays in the shared address space: LDS/STS, not generic loads)
  const uint32_t pad = (1024u - (smem_u32(smraw) & 1023u)) & 1023u;
  constexpr int SLOT = CFG::SLOT_BYTES / 8;                 // float2 per slot
  float2* tiles = reinterpret_cast<float2*>(smraw + pad);  // two slots
  float2* tw = tiles + 2 * SLOT;
  float2* ttw = tw + PL::TW;  // this tile's inter-pass twiddles
  uint64_t* bar = reinterpret_cast<uint64_t*>(ttw + (PASS == 3 ? 0 : L + kTileCols));
  const int R1 = pr.R1, R2 = pr.R2, R3 = pr.R3;
  const int64_t N = pr.N;
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_init(bar + 1, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  build_twiddles<PL>(tw, threadIdx.x, blockDim.x);
  __syncthreads();
  fft_pdl_wait();  // the previous pass (or kernel) has completed: its output may be read
  fft_pdl_trigger();
  auto issue = [&](int tl, int j) {  // thread 0: TMA load of tile tl into buffer j
    int cg_, slab_, b_;
    fft3_tile_coords<PASS>(tl, R1, R2, R3, &cg_, &slab_, &b_);
    float2* dst = tiles + j * SLOT;
    mbar_expect_tx(bar + j, uint32_t(CFG::TILE_BYTES));
    for (int r0 = 0; r0 < L; r0 += 256) {
      // box rows run along dim 2 for passes 1/2 ({2 col, slab, b L + row}) and along dim 1
      // for pass 3 ({2 col, row, b R2 + slab})
      if constexpr (PASS == 3) {
        tma_load_3d(dst + r0 * kTileCols, &src, bar + j, 2 * cg_ * kTileCols, r0,
                    b_ * R2 + slab_);
      } else {
        tma_load_3d(dst + r0 * kTileCols, &src, bar + j, 2 * cg_ * kTileCols, slab_,
                    b_ * L + r0);
      }
    }
  };
  int tl = blockIdx.x;
  if (threadIdx.x == 0 && tl < pr.ntiles) issue(tl, 0);
  for (int it = 0; tl < pr.ntiles; ++it, tl += gridDim.x) {
    const int j = it & 1;
    const uint32_t par = uint32_t(it >> 1) & 1u;
    const int nxt = tl + int(gridDim.x);
    if (threadIdx.x == 0 && nxt < pr.ntiles) {
      // passes 2 and 3: the previous tile's TMA store must have read buffer j ^ 1 first
      if constexpr (PASS != 1) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
      issue(nxt, j ^ 1);
    }
    // This tile's inter-pass twiddles, computed while its copy is in flight (the previous
    // tile's readers finished at the last barrier; the wait below publishes them). Each is an
    // independent FP64 sincospi of an exactly reduced integer phase, rounded once to FP32:
    //   pass 1: W_N^(R1 m2 km3) (times 1/N for the inverse), one per output row km3, shared by
    //           every column of the tile;
    //   pass 2: W_N^(r km2 R3) per row km2 and W_N^(r km3) per column km3, multiplied per
    //           element in FP32 (about one ulp more than a product rounded once; no FP64 work
    //           per element).
    if constexpr (PASS == 1) {
      int cg_, slab_, b_;
      fft3_tile_coords<PASS>(tl, R1, R2, R3, &cg_, &slab_, &b_);
      const double sc = pr.inverse ? 1.0 / double(N) : 1.0;
      for (int i = threadIdx.x; i < L; i += blockDim.x) {
        const double2 w = w_exact(int64_t(R1) * slab_ * i, N);
        ttw[i] = make_float2(float(w.x * sc), float(w.y * sc));
      }
    }
    const bool ok = __syncthreads_and(mbar_wait(bar + j, par, pr.wait_polls) ? 1 : 0) != 0;
    if (!ok) {
      if (threadIdx.x == 0) {
        atomicExch(pr.err, SP_ERR_TIMEOUT);
        if (pr.sticky) {
          *reinterpret_cast<volatile int*>(pr.sticky) = SP_ERR_TIMEOUT;
          __threadfence_system();
        }
        // bounded second waits (full limit) for the copies still in flight, so that no TMA
        // write lands in this CTA's shared memory after it exits
        (void)mbar_wait(bar + j, par);
        if (nxt < pr.ntiles) (void)mbar_wait(bar + (j ^ 1), uint32_t((it + 1) >> 1) & 1u);
        if constexpr (PASS != 1) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
      }
      return;
    }
    float2* tile = tiles + j * SLOT;
    int cg, slab, b;
    fft3_tile_coords<PASS>(tl, R1, R2, R3, &cg, &slab, &b);
    const int col0 = cg * kTileCols;
    const int team = threadIdx.x / P, t = threadIdx.x - team * P;
    const unsigned mask = team_mask<P>();
    float2* buf = tile + team * PL::BUF;  // exchange buffer inside this tile's slot
    const int c = team;  // this team's column in the tile
    float2 v[E];
    static_for<0, E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const int row = slot_elem<PL, e>(t);
      float2 z = tile[swz(row, c)];
      if (PASS == 1 && pr.inverse) z.y = -z.y;
      v[e] = z;
    });
    __syncthreads();  // every column is in registers: the slot becomes exchange space
    team_pass0<PL>(v);
    team_passes<PL>(v, buf, tw, t, mask);
    // output k = t + e*P of this column
    if constexpr (PASS == 1) {
      // twiddle W_N^(R1 m2 km3) of output row km3 = t + e P, from the tile table
      const int m2 = slab, r = col0 + c;
      float2* dst = pr.out + int64_t(b) * N + (int64_t(m2) * R1 + r) * R3;
#pragma unroll
      for (int e = 0; e < E; ++e) dst[t + e * P] = cmul(v[e], ttw[t + e * P]);
    } else {
      if constexpr (PASS == 2) {
        // twiddle W_N^(r (km2 R3 + km3)), km2 = t + e P, km3 = col0 + c: an FP64 anchor
        // W_N^(r (t R3 + km3)) and step W_N^(r R3 P), an FP64 recurrence over e, each factor
        // rounded to FP32 once
        const int64_t r = slab, km3 = col0 + c;
        double2 w = w_exact(r * (int64_t(t) * R3 + km3), N);
        const double2 st = w_exact(r * R3 * P, N);
#pragma unroll
        for (int e = 0; e < E; ++e) {
          v[e] = cmul(v[e], make_float2(float(w.x), float(w.y)));
          w = zmul(w, st);
        }
      }
      __syncthreads();  // every team has read its column: the tile can be overwritten
  #pragma unroll
      for (int e = 0; e < E; ++e) {
        float2 z = v[e];
        if (PASS == 3 && pr.inverse) z.y = -z.y;
        tile[swz(t + e * P, c)] = z;
      }
      // the staged tile (128-byte rows in the load's swizzle) goes out as TMA tensor stores:
      //   PASS 2: S2[b][km2 = row][r = slab][km3 = col0 ..] at {2 col0, slab, b R2 + row},
      //   PASS 3: X[b][kr = row][km2 = slab][km3 = col0 ..] at {2 col0, slab, b R1 + row}
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (threadIdx.x == 0) {
        for (int r0 = 0; r0 < L; r0 += 256)
          tma_store_3d(&dst, tile + r0 * kTileCols, 2 * col0, slab, b * L + r0);
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
      }
    }
    // The slot was written through the generic proxy (exchange, output staging); order those
    // accesses before the TMA (async proxy) that refills it with tile it + 2.
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();  // slot j is free for the load of tile it + 2
  }
  // the last TMA stores complete before the CTA (and its shared memory) goes away
  if constexpr (PASS != 1) {
    if (threadIdx.x == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
  }
}

// Twiddles w_k = exp(-i pi k / m) of the real-FFT untangle and its inverse. A thread handles
// kUntT indices k = k0 + j * kUntB (j < kUntT): one FP64 sincospi anchor at k0, then an FP64
// rotation by the launch's step d = exp(-i pi kUntB / m) per index, each rounded to FP32 once.
constexpr int kUntB = 256;  // threads per block
constexpr int kUntT = 4;    // indices per thread (8 and 16 measured slower at 2^22)

// Packed real FFT untangle (n = 2m real samples viewed as m complex z, Z = FFT_m(z)):
//   X_k = (Z_k + conj Z_{m-k})/2 - i w_k (Z_k - conj Z_{m-k})/2, w_k = exp(-i pi k/m), k < m;
//   X_m = Re Z_0 - Im Z_0. Index k in [0, m/2] produces X_k and X_{m-k}; only bins below nout
//   are written (nout = m + 1 for the whole one-sided spectrum).
__global__ void __launch_bounds__(kUntB) k_rfft_untangle(const float2* __restrict__ Z,
                                                         float2* __restrict__ X, int64_t m,
                                                         int64_t ldx, int64_t nout, double2 d) {
  fft_pdl_wait();
  fft_pdl_trigger();
  const int64_t half = m / 2 + 1;
  const int64_t per_row = (half + kUntB * kUntT - 1) / (kUntB * kUntT);
  const int64_t b = blockIdx.x / per_row;
  const int64_t k0 = (blockIdx.x - b * per_row) * (kUntB * kUntT) + threadIdx.x;
  const float2* z = Z + b * m;
  float2* x = X + b * ldx;
  // Every read of the thread first, so that its 2 kUntT loads are in flight together: the
  // kernel waits on the latency of these (L2-resident) reads, not on bandwidth.
  float2 zks[kUntT], zms[kUntT];
#pragma unroll
  for (int j = 0; j < kUntT; ++j) {
    const int64_t k = k0 + int64_t(j) * kUntB;
    zks[j] = k < half ? z[k] : make_float2(0.f, 0.f);
    zms[j] = (k < half && k != 0) ? z[m - k] : make_float2(0.f, 0.f);
  }
  double sn, cs;
  sincospi(-double(k0) / double(m), &sn, &cs);
  double2 w = make_double2(cs, sn);
#pragma unroll
  for (int j = 0; j < kUntT; ++j) {
    const int64_t k = k0 + int64_t(j) * kUntB;
    if (k < half) {
      if (k == 0) {
        const float2 z0 = zks[j];
        x[0] = make_float2(z0.x + z0.y, 0.f);
        if (m < nout) x[m] = make_float2(z0.x - z0.y, 0.f);
      } else {
        const float2 zk = zks[j], zm = zms[j];
        const float2 wf = make_float2(float(w.x), float(w.y));
        // X_{m-k} shares zk, zm: ze' = conj(ze), zo' = -conj(zo), w_{m-k} = -conj(w_k)
        const float2 ze = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        const float2 zo = make_float2(0.5f * (zk.x - zm.x), 0.5f * (zk.y + zm.y));
        const float2 wz = cmul(wf, zo);
        if (k < nout) x[k] = make_float2(ze.x + wz.y, ze.y - wz.x);
        if (2 * k != m && m - k < nout) {
          const float2 wz2 = make_float2(wz.x, -wz.y);  // w' zo' = conj(w zo)
          x[m - k] = make_float2(ze.x + wz2.y, -ze.y - wz2.x);
        }
      }
    }
    w = zmul(w, d);
  }
}

// Analytic-signal spectrum of n = 2m real samples from the packed transform Z = FFT_m(z)
// (scipy.signal.hilbert's mask h for even n): the untangle above gives X_k for k <= m, and
//   Y_0 = X_0, Y_k = 2 X_k (0 < k < m), Y_m = X_m, Y_k = 0 (m < k < 2m)
// is written as the input of the n-point inverse FFT (row stride 2m complex). Index k in
// [0, m/2] writes Y_k, Y_{m-k} and the zeros Y_{m+k}, Y_{2m-k}.
__global__ void __launch_bounds__(kUntB) k_hilbert_spectrum(const float2* __restrict__ Z,
                                                            float2* __restrict__ Y, int64_t m,
                                                            double2 d) {
  fft_pdl_wait();
  fft_pdl_trigger();
  const int64_t half = m / 2 + 1;
  const int64_t per_row = (half + kUntB * kUntT - 1) / (kUntB * kUntT);
  const int64_t b = blockIdx.x / per_row;
  const int64_t k0 = (blockIdx.x - b * per_row) * (kUntB * kUntT) + threadIdx.x;
  const float2* z = Z + b * m;
  float2* y = Y + b * 2 * m;
  float2 zks[kUntT], zms[kUntT];
#pragma unroll
  for (int j = 0; j < kUntT; ++j) {
    const int64_t k = k0 + int64_t(j) * kUntB;
    zks[j] = k < half ? z[k] : make_float2(0.f, 0.f);
    zms[j] = (k < half && k != 0) ? z[m - k] : make_float2(0.f, 0.f);
  }
  double sn, cs;
  sincospi(-double(k0) / double(m), &sn, &cs);
  double2 w = make_double2(cs, sn);
  const float2 zero = make_float2(0.f, 0.f);
#pragma unroll
  for (int j = 0; j < kUntT; ++j) {
    const int64_t k = k0 + int64_t(j) * kUntB;
    if (k < half) {
      if (k == 0) {
        const float2 z0 = zks[j];
        y[0] = make_float2(z0.x + z0.y, 0.f);
        y[m] = make_float2(z0.x - z0.y, 0.f);
      } else {
        const float2 zk = zks[j], zm = zms[j];
        const float2 wf = make_float2(float(w.x), float(w.y));
        const float2 ze = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        const float2 zo = make_float2(0.5f * (zk.x - zm.x), 0.5f * (zk.y + zm.y));
        const float2 wz = cmul(wf, zo);
        y[k] = make_float2(2.f * (ze.x + wz.y), 2.f * (ze.y - wz.x));
        y[m + k] = zero;
        if (2 * k != m) {
          const float2 wz2 = make_float2(wz.x, -wz.y);
          y[m - k] = make_float2(2.f * (ze.x + wz2.y), 2.f * (-ze.y - wz2.x));
          y[2 * m - k] = zero;
        }
      }
    }
    w = zmul(w, d);
  }
}

// Inverse of the untangle (irfft pre-twist): from X_0..X_m build the packed spectrum
//   Y_k = E_k + i conj(w_k) O_k, E = (X_k + conj X_{m-k})/2, O = (X_k - conj X_{m-k})/2,
// with X_0, X_m taken as real; then z = IFFT_m(Y) interleaves the n real samples. Every bin is
// multiplied by `scale`, and bin kfix (if any) also by ffix (the resample's unpaired bin).
__global__ void __launch_bounds__(kUntB) k_irfft_pretwist(const float2* __restrict__ X,
                                                          int64_t ldx, int64_t nbins,
                                                          float2* __restrict__ Y, int64_t m,
                                                          double2 d, float scale, int64_t kfix,
                                                          float ffix) {
  fft_pdl_wait();
  fft_pdl_trigger();
  const int64_t half = m / 2 + 1;
  const int64_t per_row = (half + kUntB * kUntT - 1) / (kUntB * kUntT);
  const int64_t b = blockIdx.x / per_row;
  const int64_t k0 = (blockIdx.x - b * per_row) * (kUntB * kUntT) + threadIdx.x;
  const float2* x = X + b * ldx;
  float2* y = Y + b * m;
  auto get = [&](int64_t j) -> float2 {
    if (j >= nbins) return make_float2(0.f, 0.f);
    float2 v = x[j];
    if (j == 0 || j == m) v.y = 0.f;
    const float f = j == kfix ? scale * ffix : scale;
    return make_float2(v.x * f, v.y * f);
  };
  float2 xks[kUntT], xms[kUntT];  // every read first, as in the untangle
#pragma unroll
  for (int j = 0; j < kUntT; ++j) {
    const int64_t k = k0 + int64_t(j) * kUntB;
    xks[j] = k < half ? get(k) : make_float2(0.f, 0.f);
    xms[j] = k < half ? get(m - k) : make_float2(0.f, 0.f);
  }
  double sn, cs;
  sincospi(-double(k0) / double(m), &sn, &cs);
  double2 w = make_double2(cs, sn);
#pragma unroll
  for (int j = 0; j < kUntT; ++j) {
    const int64_t k = k0 + int64_t(j) * kUntB;
    if (k < half) {
      const float2 xk = xks[j], xm = xms[j];
      const float c = float(w.x), sf = float(w.y);
      const float2 wc = make_float2(c, -sf);  // conj(w_k)
      const float2 e1 = make_float2(0.5f * (xk.x + xm.x), 0.5f * (xk.y - xm.y));
      const float2 o1 = make_float2(0.5f * (xk.x - xm.x), 0.5f * (xk.y + xm.y));
      const float2 t1 = cmul(wc, o1);
      y[k % m] = make_float2(e1.x - t1.y, e1.y + t1.x);
      if (k != 0 && 2 * k != m) {
        // index m-k: E' = conj(E), O' = -conj(O), conj(w_{m-k}) = -w_k
        const float2 e2 = make_float2(e1.x, -e1.y);
        const float2 o2 = make_float2(-o1.x, o1.y);
        const float2 wc2 = make_float2(-c, -sf);
        const float2 t2 = cmul(wc2, o2);
        y[m - k] = make_float2(e2.x - t2.y, e2.y + t2.x);
      }
    }
    w = zmul(w, d);
  }
}

}  // namespace b2s
