// C-ABI: segment-mean spectral estimates (welch / csd / coherence).
#include <cuda.h>

#include <mutex>
#include <utility>

#include "capi_common.h"
#include "dispatch.cuh"

namespace b2s {
namespace {

constexpr int kMaxLog = kMaxLogL;

}  // namespace

// One CTA of kRedGroups warps per (row, 32 consecutive output bins): warp g sums the row's
// partial slots c = g, g + kRedGroups, ... in FP64 for its 32 bins (loads coalesced over the
// bins), then warp 0 adds the group sums in group order. The order is fixed by the launch
// geometry alone, so results are deterministic; a row spread over hundreds of teams (few rows)
// is summed by kRedGroups warps per bin instead of one thread.
constexpr int kRedGroups = 8;

__global__ void __launch_bounds__(32 * kRedGroups) k_reduce_mean(ReduceParams p) {
  pdl_wait();  // launched as a programmatic dependent of the segment kernel
  // the next kernel in the stream (e.g. the next call's segment kernel, which waits for this
  // grid to complete before reading anything the caller passes) may start its prologue now
  pdl_trigger();
  __shared__ double4 red[kRedGroups][32];
  const int lane = threadIdx.x & 31, grp = threadIdx.x >> 5;
  const int64_t chunks = (p.nout + 31) / 32;
  const int64_t r = blockIdx.x / chunks;
  const int k = int(blockIdx.x - r * chunks) * 32 + lane;
  const bool live = k < p.nout;
  const int L = p.L;
  const int kk = k == 0 ? 0 : L - k;  // mirror bin of the L-periodic spectrum (any L)
  const int kc = k <= kk ? k : kk;
  const int64_t t0 = first_team(r, p.nseg, p.G);
  int64_t t1 = last_team(r, p.nseg, p.G);
  if (t1 > p.nteams - 1) t1 = p.nteams - 1;
  const int nsl = int(t1 - t0 + 1);
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  if (live) {
    if (p.mode == 4) {
      const int stride = 2 * L;
      const float* q = p.partial + r * p.cmax * int64_t(stride) + 2 * k;
#pragma unroll 2
      for (int c = grp; c < nsl; c += kRedGroups) {
        a0 += double(q[int64_t(c) * stride]);
        a1 += double(q[int64_t(c) * stride + 1]);
      }
    } else if (p.mode == 3) {
      const int stride = cross_q_floats(L);
      const float* q = p.partial + r * p.cmax * int64_t(stride) + k;
#pragma unroll 4
      for (int c = grp; c < nsl; c += kRedGroups) a0 += double(q[int64_t(c) * stride]);
    } else if (p.mode == 0) {
      const int stride = welch_slot_floats(L);
      const float* q = p.partial + r * p.cmax * int64_t(stride) + kc;
#pragma unroll 4
      for (int c = grp; c < nsl; c += kRedGroups) a0 += double(q[int64_t(c) * stride]);
    } else if (p.f64) {
      const int stride = cross_slot_floats(L);
      const int cq = cross_q_floats(L);
      const double* base = reinterpret_cast<const double*>(p.partial) + r * p.cmax * int64_t(stride);
#pragma unroll 2
      for (int c = grp; c < nsl; c += kRedGroups) {
        const double* q = base + int64_t(c) * stride;
        a0 += q[k];
        a1 += q[kk];
        a2 += q[cq + 2 * kc];
        a3 += q[cq + 2 * kc + 1];
      }
    } else {
      const int stride = cross_slot_floats(L);
      const int cq = cross_q_floats(L);
      const float* base = p.partial + r * p.cmax * int64_t(stride);
#pragma unroll 2
      for (int c = grp; c < nsl; c += kRedGroups) {
        const float* q = base + int64_t(c) * stride;
        a0 += double(q[k]);
        a1 += double(q[kk]);
        a2 += double(q[cq + 2 * kc]);
        a3 += double(q[cq + 2 * kc + 1]);
      }
    }
  }
  red[grp][lane] = make_double4(a0, a1, a2, a3);
  __syncthreads();
  if (grp != 0 || !live) return;
  a0 = a1 = a2 = a3 = 0.0;
#pragma unroll
  for (int g = 0; g < kRedGroups; ++g) {
    const double4 v = red[g][lane];
    a0 += v.x;
    a1 += v.y;
    a2 += v.z;
    a3 += v.w;
  }
  const int64_t idx = r * p.nout + k;
  double fac = 1.0 / double(p.nseg);
  if (p.onesided && k != 0 && 2 * k != L) fac *= 2.0;
  if (p.mode == 0) {
    p.out[idx] = float(0.5 * a0 * fac);
    return;
  }
  if (p.mode == 3) {  // complex input: two-sided, no mirror
    p.out[idx] = float(a0 * fac);
    return;
  }
  if (p.mode == 4) {  // csd of complex inputs: mean conj(X) Y, two-sided
    p.out[2 * idx] = float(a0 * fac);
    p.out[2 * idx + 1] = float(a1 * fac);
    return;
  }
  const double qk = a0, qm = a1, cr = a2, ci = a3;
  const double pxy_re = 0.5 * ci, pxy_im = 0.25 * (qm - qk);
  if (p.mode == 1) {
    p.out[2 * idx] = float(pxy_re * fac);
    p.out[2 * idx + 1] = float(pxy_im * fac);
    return;
  }
  const double sxx = 0.25 * (qk + qm + 2.0 * cr);
  const double syy = 0.25 * (qk + qm - 2.0 * cr);
  const double num = pxy_re * pxy_re + pxy_im * pxy_im;
  const double den = sxx * syy;
  double coh = den > 0.0 ? num / den : 0.0;
  if (!(coh >= 0.0)) coh = 0.0;
  if (coh > 1.0) coh = 1.0;
  p.out[idx] = float(coh);
}


namespace {

struct MeanPlanInfo {
  MeanInfo k;
  int log_l = 0;
  int nseg = 0;
  int64_t total = 0, G = 0, nteams = 0, blocks = 0;
  int cmax = 0;
  bool f64 = false;  // FP64 partial slots (k_cross_mean / k_cross_half)
  int64_t slot_floats = 0;
  int64_t ws_bytes = 0;
};

// Largest count of low window-spectrum bins the spectral detrend correction can apply: the
// bins k < P and k > L - P are the first and last register of every team thread.
int spectral_bins(int log_l) { return (1 << log_l) >> team_log_e_rt(log_l); }

// CTA waves of the 50%-overlap welch and csd / coherence grids at short segments. With one team
// range per resident team, the SMs of the 64 x 2^20 welch at nperseg 256 finished between 57 %
// and 100 % of the kernel's time (identical team ranges; ncu sm__cycles_active min/max); shorter
// ranges over several waves let the block scheduler even that out. Measured on 64 x 2^20 (welch,
// 1 / 2 / 4 / 8 waves, us): nperseg 32 315 / 330 / 369 / 423, 64 182 / 164 / 161 / 175,
// 128 186 / 162 / 164 / 173, 256 151 / 133 / 127 / 137, 512 144 / 144 / 147 / 155 (1024 and up
// lose to the extra per-CTA setup); csd pairs with this rule at nperseg 64 / 128 / 256:
// 498 / 452 / 381 -> 463 / 408 / 317 us.
int half_waves(int log_l) { return log_l == 8 ? 4 : (log_l == 6 || log_l == 7) ? 2 : 1; }

// mode: 0 welch, 1 csd, 2 coherence. The segments-per-team split (and so the workspace size)
// comes from one canonical kernel per family (the time-domain-detrend variant, coherence for the
// cross family), so sp_mean_workspace_size, which knows neither the detrend form nor csd vs
// coherence, sizes every variant's launch.
// fine = false keeps one wave (the smallest workspace; the no-allocation entry point falls back
// to it when the finer split's partial slots would not fit its fixed scratch).
int make_plan(int mode, int64_t rows, int64_t n, int nperseg, int nfft, int hop, int detrend,
              MeanPlanInfo* pl, bool spectral = false, bool fine = true) {
  // mode 3: welch of complex rows (one segment per transform, two-sided); mode 4: csd of two
  // complex signals (two transforms per segment, two-sided)
  const bool cplx = mode == 3 || mode == 4;
  const bool cross = mode == 1 || mode == 2;
  if (rows < 0 || n < 1 || nperseg < 1 || nperseg > n || hop < 1 || hop > nperseg ||
      nfft < nperseg || detrend < 0 || detrend > 2 || n >= (int64_t(1) << 31)) {
    set_error("invalid spectral-mean arguments (rows=%lld n=%lld nperseg=%d nfft=%d hop=%d)",
              (long long)rows, (long long)n, nperseg, nfft, hop);
    return SP_ERR_ARG;
  }
  int log_l = ilog2_exact(nfft);
  // welch with a non-power-of-two nfft: the Bluestein kernel on a power-of-two transform
  const bool blue = log_l < 0 && !cplx && nfft >= 3 && nfft <= kBlueMaxN;
  const int max_log = cplx ? kMaxLog : kMaxLogLReal;
  if (!blue && (log_l < 0 || log_l > max_log)) {
    set_error("nfft=%d: fused kernels need a power of two <= %d (or any nfft <= %d)",
              nfft, 1 << max_log, kBlueMaxN);
    return SP_ERR_UNSUPPORTED;
  }
  if (blue) log_l = blue_log_m(nfft);
  const bool half = !blue && !cplx && log_l >= 1 && nperseg == nfft && 2 * hop == nperseg &&
                    detrend <= 1;
  const int hdet = (spectral && detrend == 1) ? 2 : detrend;  // lookup index: 2 = spectral
  MeanInfo canon;
  if (cplx) {
    pl->k = canon = mode == 4 ? cplx_lookup_csd(log_l, detrend) : cplx_lookup_welch(log_l, detrend);
  } else if (blue) {
    pl->k = canon = cross ? blue_lookup_cross(log_l, detrend) : blue_lookup_welch(log_l, detrend);
  } else if (cross && half) {
    pl->k = mean_lookup_cross_half(log_l, hdet, mode == 1);
    canon = mean_lookup_cross_half(log_l, detrend, false);
  } else if (cross) {
    pl->k = canon = mean_lookup_cross(log_l, detrend);
  } else if (half) {
    pl->k = mean_lookup_welch_half(log_l, hdet, false);
    canon = mean_lookup_welch_half(log_l, detrend, false);
  } else {
    pl->k = canon = mean_lookup_welch(log_l, detrend);
  }
  pl->log_l = log_l;
  pl->nseg = int((n - nperseg) / hop + 1);
  pl->total = rows * pl->nseg;
  int sms = 0;
  const int nb = resident_ctas(canon.fn, canon.threads, canon.smem, &sms);
  if (resident_ctas(pl->k.fn, pl->k.threads, pl->k.smem, &sms) <= 0) {
    set_error("no resident CTA for spectral-mean kernel (nfft=%d, smem=%zu)", nfft, pl->k.smem);
    return SP_ERR_UNSUPPORTED;
  }
  if (nb <= 0) {
    set_error("no resident CTA for spectral-mean kernel (nfft=%d, smem=%zu)", nfft, pl->k.smem);
    return SP_ERR_UNSUPPORTED;
  }
  const int64_t cap = int64_t(nb) * sms * canon.teams;
  const int64_t total = pl->total > 0 ? pl->total : 1;
  const int waves = (fine && half) ? half_waves(log_l) : 1;
  pl->G = cplx    ? cdiv(total, cap)
          : cross ? cdiv(total, int64_t(waves) * cap)
                  : 2 * cdiv(total, 2 * int64_t(waves) * cap);
  if (pl->G < 1) pl->G = 1;
  // long team ranges sum through shared-memory block totals (same shape, threads and smem; the
  // residency query also opts the kernel in to its dynamic shared memory)
  if (half && !cross && !cplx && !blue && pl->G > kDirectSegs) {
    pl->k = mean_lookup_welch_half(log_l, hdet, true);
    if (resident_ctas(pl->k.fn, pl->k.threads, pl->k.smem, &sms) <= 0) {
      set_error("no resident CTA for spectral-mean kernel (nfft=%d, smem=%zu)", nfft, pl->k.smem);
      return SP_ERR_UNSUPPORTED;
    }
  }
  pl->nteams = cdiv(total, pl->G);
  pl->blocks = cdiv(pl->nteams, pl->k.teams);
  int64_t cm = cdiv(pl->nseg, pl->G) + 1;
  if (cm > pl->nteams) cm = pl->nteams;
  pl->cmax = int(cm);
  pl->f64 = cross && !blue;
  pl->slot_floats = cross ? (pl->f64 ? 2 : 1) * int64_t(cross_slot_floats(nfft))
                          : (mode == 4 ? 2 * int64_t(nfft)
                                       : (cplx ? cross_q_floats(nfft) : welch_slot_floats(nfft)));
  pl->ws_bytes = rows * pl->cmax * pl->slot_floats * int64_t(sizeof(float));
  return SP_OK;
}

int run_mean(int mode, const float* x, const float* y, int64_t rows, int64_t n, int64_t ldx,
             int64_t ldy, const float* win, int nperseg, int nfft, int hop, int detrend,
             int onesided, float* out, void* ws, size_t ws_bytes, void* stream,
             const float* wdft = nullptr, int n_low = 0, bool fine = true) {
  const bool cross = mode == 1 || mode == 2 || mode == 4;  // two input signals
  if (!x || !win || !out || (cross && !y) || ldx < n || (cross && ldy < n)) {
    set_error("null pointer or row stride smaller than n");
    return SP_ERR_ARG;
  }
  const int log_l_in = ilog2_exact(nfft);
  const bool spectral = wdft != nullptr && n_low >= 1 && log_l_in >= 1 &&
                        n_low <= spectral_bins(log_l_in);
  MeanPlanInfo pl;
  int st = make_plan(mode, rows, n, nperseg, nfft, hop, detrend, &pl, spectral, fine);
  if (st != SP_OK) return st;
  if (rows == 0) return SP_OK;
  if (ws_bytes < size_t(pl.ws_bytes) || (pl.ws_bytes > 0 && !ws)) {
    set_error("workspace too small: need %lld bytes, got %zu", (long long)pl.ws_bytes, ws_bytes);
    return SP_ERR_WORKSPACE;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  MeanParams p;
  p.x = x;
  p.y = y;
  p.ld_x = ldx;
  p.ld_y = cross ? ldy : 0;
  p.rows = rows;
  p.nperseg = nperseg;
  p.hop = hop;
  p.nseg = pl.nseg;
  p.detrend = detrend;
  p.win = win;
  p.G = pl.G;
  p.cmax = pl.cmax;
  p.total = pl.total;
  p.partial = static_cast<float*>(ws);
  // the spectral tables are read only by the 50%-overlap kernels' spectral variants
  p.wdft = spectral ? reinterpret_cast<const float2*>(wdft) : nullptr;
  p.n_low = spectral ? n_low : 0;
  p.nfft = nfft;
  pl.k.launch(dim3(unsigned(pl.blocks)), pl.k.threads, pl.k.smem, s, p);
  B2S_CHECK_CUDA(cudaGetLastError(), "spectral-mean kernel launch");
  ReduceParams rp;
  rp.partial = p.partial;
  rp.rows = rows;
  rp.L = nfft;
  rp.nout = (mode == 2 || onesided) ? nfft / 2 + 1 : nfft;
  rp.onesided = (mode != 2 && onesided) ? 1 : 0;
  rp.nseg = pl.nseg;
  rp.G = pl.G;
  rp.cmax = pl.cmax;
  rp.nteams = pl.nteams;
  rp.mode = mode;
  rp.f64 = pl.f64 ? 1 : 0;
  rp.out = out;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(rows * cdiv(rp.nout, 32)));
  cfg.blockDim = dim3(32 * kRedGroups);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  B2S_CHECK_CUDA(cudaLaunchKernelEx(&cfg, k_reduce_mean, rp), "spectral-mean reduce launch");
  return SP_OK;
}

// ---------------------------------------------------------------------------------------------
// Fixed scratch for sp_welch_f32_noalloc. Some callers cannot allocate device memory at call
// time: plugin hosts that only hand over input/output pointers owned by another framework, and
// latency-critical loops that must not take cudaMalloc's implicit device synchronisation or
// grow their footprint after start-up. For them the partial-sum workspace lives in this
// file-scope array. A device holds it from the first use of this file's kernels there (the
// module is loaded lazily by default) until the process exits.
// ---------------------------------------------------------------------------------------------
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;  // 16 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
struct NoAllocSlot {
  CUcontext ctx = nullptr;  // context the address was resolved in
  void* addr = nullptr;
};
NoAllocSlot g_noalloc_slot[kNoAllocMaxDevices];

// cuCtxGetCurrent through the runtime's driver entry-point query (no link-time libcuda
// dependency, so the library still loads on machines without a driver).
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(p);
  }();
  return fn;
}

// Device address of the scratch array on the current device. In host code the array's name is
// only a host-side stand-in, so the address comes from cudaGetSymbolAddress, resolved with the
// device current and cached per device together with the context it was resolved in: after a
// cudaDeviceReset the device gets a new primary context (and a freshly loaded module), so the
// cached address is resolved again instead of being reused.
int noalloc_scratch(void** out) {
  int dev = 0;
  B2S_CHECK_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    set_error("sp_welch_f32_noalloc: device index %d beyond the supported %d", dev,
              kNoAllocMaxDevices);
    return SP_ERR_ARG;
  }
  // the plan query before this call (occupancy) has made the device's context current
  CUcontext ctx = nullptr;
  const CtxGetCurrentFn get = ctx_get_current();
  if (get == nullptr || get(&ctx) != CUDA_SUCCESS) ctx = nullptr;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  NoAllocSlot& slot = g_noalloc_slot[dev];
  // without a context handle to compare, resolve the address on every call
  if (slot.addr == nullptr || ctx == nullptr || slot.ctx != ctx) {
    void* p = nullptr;
    B2S_CHECK_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress");
    slot.ctx = ctx;
    slot.addr = p;
  }
  *out = slot.addr;
  return SP_OK;
}

}  // namespace
}  // namespace b2s

extern "C" {

int sp_welch_f32_noalloc(const float* x, int64_t rows, int64_t n, int64_t ld, const float* win,
                         int nperseg, int nfft, int hop, int detrend, int onesided, float* out,
                         void* stream) {
  b2s::MeanPlanInfo pl;
  int st = b2s::make_plan(0, rows, n, nperseg, nfft, hop, detrend, &pl);
  if (st != SP_OK) return st;
  bool fine = true;
  if (size_t(pl.ws_bytes) > b2s::kNoAllocScratchBytes) {  // one wave needs the least scratch
    fine = false;
    st = b2s::make_plan(0, rows, n, nperseg, nfft, hop, detrend, &pl, false, false);
    if (st != SP_OK) return st;
  }
  if (size_t(pl.ws_bytes) > b2s::kNoAllocScratchBytes) {
    b2s::set_error(
        "sp_welch_f32_noalloc: this shape needs %lld bytes of scratch but the built-in scratch "
        "holds %zu bytes; use sp_welch_f32 with a caller-provided workspace",
        (long long)pl.ws_bytes, b2s::kNoAllocScratchBytes);
    return SP_ERR_WORKSPACE;
  }
  void* ws = nullptr;
  const int sst = b2s::noalloc_scratch(&ws);
  if (sst != SP_OK) return sst;
  return b2s::run_mean(0, x, nullptr, rows, n, ld, 0, win, nperseg, nfft, hop, detrend, onesided,
                       out, ws, b2s::kNoAllocScratchBytes, stream, nullptr, 0, fine);
}

int64_t sp_mean_workspace_size(int kind, int64_t rows, int64_t n, int nperseg, int nfft, int hop,
                               int detrend) {
  b2s::MeanPlanInfo pl;
  const int mode = (kind == 3 || kind == 4) ? kind : (kind != 0 ? 2 : 0);
  const int st = b2s::make_plan(mode, rows, n, nperseg, nfft, hop, detrend, &pl);
  return st == SP_OK ? pl.ws_bytes : int64_t(st);
}

int sp_welch_f32(const float* x, int64_t rows, int64_t n, int64_t ld, const float* win,
                 int nperseg, int nfft, int hop, int detrend, int onesided, float* out,
                 void* workspace, size_t workspace_bytes, void* stream) {
  return b2s::run_mean(0, x, nullptr, rows, n, ld, 0, win, nperseg, nfft, hop, detrend, onesided,
                       out, workspace, workspace_bytes, stream);
}

int sp_welch_c64(const float* x, int64_t rows, int64_t n, int64_t ld, const float* win,
                 int nperseg, int nfft, int hop, int detrend, float* out, void* workspace,
                 size_t workspace_bytes, void* stream) {
  return b2s::run_mean(3, x, nullptr, rows, n, ld, 0, win, nperseg, nfft, hop, detrend, 0, out,
                       workspace, workspace_bytes, stream);
}

int sp_csd_cplx(const float* x, const float* y, int64_t rows, int64_t n, int64_t ldx,
                int64_t ldy, const float* win, int nperseg, int nfft, int hop, int detrend,
                float* out, void* workspace, size_t workspace_bytes, void* stream) {
  return b2s::run_mean(4, x, y, rows, n, ldx, ldy, win, nperseg, nfft, hop, detrend, 0, out,
                       workspace, workspace_bytes, stream);
}

int sp_welch_spectral_bins(int nfft) {
  const int log_l = b2s::ilog2_exact(nfft);
  if (log_l < 1 || log_l > b2s::kMaxLogLReal) return 0;
  return b2s::spectral_bins(log_l);
}

int sp_welch_f32_ex(const float* x, int64_t rows, int64_t n, int64_t ld, const float* win,
                    const float* win_dft_low, int n_low, int nperseg, int nfft, int hop,
                    int detrend, int onesided, float* out, void* workspace,
                    size_t workspace_bytes, void* stream) {
  return b2s::run_mean(0, x, nullptr, rows, n, ld, 0, win, nperseg, nfft, hop, detrend, onesided,
                       out, workspace, workspace_bytes, stream, win_dft_low, n_low);
}

int sp_csd_c64(const float* x, const float* y, int64_t rows, int64_t n, int64_t ldx,
               int64_t ldy, const float* win, int nperseg, int nfft, int hop, int detrend,
               int onesided, float* out, void* workspace, size_t workspace_bytes, void* stream) {
  return b2s::run_mean(1, x, y, rows, n, ldx, ldy, win, nperseg, nfft, hop, detrend, onesided,
                       out, workspace, workspace_bytes, stream);
}

int sp_csd_c64_ex(const float* x, const float* y, int64_t rows, int64_t n, int64_t ldx,
                  int64_t ldy, const float* win, const float* win_dft_low, int n_low, int nperseg,
                  int nfft, int hop, int detrend, int onesided, float* out, void* workspace,
                  size_t workspace_bytes, void* stream) {
  return b2s::run_mean(1, x, y, rows, n, ldx, ldy, win, nperseg, nfft, hop, detrend, onesided,
                       out, workspace, workspace_bytes, stream, win_dft_low, n_low);
}

int sp_coherence_f32_ex(const float* x, const float* y, int64_t rows, int64_t n, int64_t ldx,
                        int64_t ldy, const float* win, const float* win_dft_low, int n_low,
                        int nperseg, int nfft, int hop, int detrend, float* out, void* workspace,
                        size_t workspace_bytes, void* stream) {
  return b2s::run_mean(2, x, y, rows, n, ldx, ldy, win, nperseg, nfft, hop, detrend, 1, out,
                       workspace, workspace_bytes, stream, win_dft_low, n_low);
}

int sp_coherence_f32(const float* x, const float* y, int64_t rows, int64_t n, int64_t ldx,
                     int64_t ldy, const float* win, int nperseg, int nfft, int hop, int detrend,
                     float* out, void* workspace, size_t workspace_bytes, void* stream) {
  return b2s::run_mean(2, x, y, rows, n, ldx, ldy, win, nperseg, nfft, hop, detrend, 1, out,
                       workspace, workspace_bytes, stream);
}

}
