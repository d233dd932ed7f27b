// C-ABI: long power-of-two FFTs (three TMA-staged passes) and the packed real transforms.
#include <cmath>
#include <cudaTypedefs.h>

#include <atomic>
#include <mutex>

#include "capi_common.h"
#include "fft3_kernels.cuh"
#include "fft_mixed.cuh"

namespace b2s {
namespace {

constexpr int kMinLogN = 12, kMaxLogN = 26;

// poll limit of the per-tile copy waits (sp_fft_set_wait_limit)
std::atomic<uint32_t> g_wait_polls{kMbarSpinLimit};

// Process-wide sticky error word in mapped, portable pinned host memory: the passes store a
// timeout there as well as in the workspace word, so a watchdog reads it with a plain load (no
// copy, no event). Allocated on first use; null if the allocation fails (the workspace word
// still reports).
int* sticky_word() {
  static int* host = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    if (cudaHostAlloc(&p, sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable) ==
        cudaSuccess) {
      *static_cast<volatile int*>(p) = 0;
      host = static_cast<int*>(p);
    } else {
      (void)cudaGetLastError();
    }
  });
  return host;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// digits (R3, R2, R1) of N = 2^e, as balanced as possible (each in [16, 512] for e in [12, 26]);
// a larger digit goes to pass 1 (R3) first, then pass 2: pass 1 writes its output with direct
// stores, so its longer columns cost no staging (measured 2^23 rfft 55.8 -> 54.1 us against
// the longer column in pass 3)
void digits(int e, int* R3, int* R2, int* R1) {
  const int a = e / 3, rem = e % 3;
  *R3 = 1 << (a + (rem > 0 ? 1 : 0));
  *R2 = 1 << (a + (rem > 1 ? 1 : 0));
  *R1 = 1 << a;
}

// 3-D float32 tensor map over rows of 2*d0 floats: dims {2 d0, d1, d2}, box {32, b1, b2},
// 128B swizzle (the box's 128-byte rows land bank-conflict free for column reads).
int make_map(CUtensorMap* map, const void* base, int64_t d0, int64_t d1, int64_t d2, int b1,
             int b2) {
  auto fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled is unavailable from the driver");
    return SP_ERR_CUDA;
  }
  cuuint64_t dims[3] = {cuuint64_t(2 * d0), cuuint64_t(d1), cuuint64_t(d2)};
  cuuint64_t strides[2] = {cuuint64_t(2 * d0 * 4), cuuint64_t(2 * d0 * d1 * 4)};
  cuuint32_t box[3] = {32u, cuuint32_t(b1), cuuint32_t(b2)};
  cuuint32_t estr[3] = {1u, 1u, 1u};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(base), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d)", int(r));
    return SP_ERR_CUDA;
  }
  return SP_OK;
}

// Launch as a programmatic dependent of the stream's previous kernel (the kernels call
// griddepcontrol.wait before reading anything that kernel may write).
template <class K, class... Args>
cudaError_t launch_pdl(K kernel, dim3 grid, int threads, size_t smem, cudaStream_t s,
                       Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(unsigned(threads));
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// points per thread of the tile-column FFT of length 2^LOG_L
template <int LOG_L>
constexpr int fft3_log_e() {
  return LOG_L <= 8 ? 4 : 5;
}

// Persistent launch: at most the resident CTAs (occupancy x SMs), each walking its share of
// the pass's `tiles` (resident_ctas also raises the kernel's shared-memory limit per device).
template <int PASS, int LL>
int launch_one(const CUtensorMap& map, const CUtensorMap& omap, Fft3Params p, int tiles,
               cudaStream_t s) {
  using CFG = Fft3Cfg<LL, fft3_log_e<LL>()>;
  auto k = &k_fft3_pass<LL, fft3_log_e<LL>(), PASS>;
  constexpr size_t kSmem = CFG::smem(PASS);
  int sms = 0;
  const int nb = resident_ctas(reinterpret_cast<const void*>(k), CFG::THREADS, kSmem, &sms);
  if (nb <= 0) {
    set_error("no resident CTA for the fft3 pass (2^%d points per column)", LL);
    return SP_ERR_UNSUPPORTED;
  }
  p.ntiles = tiles;
  const int grid = tiles < nb * sms ? tiles : nb * sms;
  B2S_CHECK_CUDA(launch_pdl(k, dim3(unsigned(grid)), CFG::THREADS, kSmem, s, map, omap, p),
                 "fft3 pass launch");
  return SP_OK;
}

template <int PASS>
int launch_pass(int log_l, const CUtensorMap& map, const CUtensorMap& omap, const Fft3Params& p,
                int blocks,
                cudaStream_t s) {  // blocks = tiles of the pass
  switch (log_l) {
    case 4: return launch_one<PASS, 4>(map, omap, p, blocks, s);
    case 5: return launch_one<PASS, 5>(map, omap, p, blocks, s);
    case 6: return launch_one<PASS, 6>(map, omap, p, blocks, s);
    case 7: return launch_one<PASS, 7>(map, omap, p, blocks, s);
    case 8: return launch_one<PASS, 8>(map, omap, p, blocks, s);
    case 9: return launch_one<PASS, 9>(map, omap, p, blocks, s);
    default:
      set_error("unsupported pass length 2^%d", log_l);
      return SP_ERR_UNSUPPORTED;
  }
}

// N-point complex FFT of `batch` rows: in -> s1 -> s2 -> out.
int fft3(const float2* in, float2* s1, float2* s2, float2* out, int batch, int e, int inverse,
         int* err, cudaStream_t s) {
  int R3, R2, R1;
  digits(e, &R3, &R2, &R1);
  Fft3Params p;
  p.R1 = R1;
  p.R2 = R2;
  p.R3 = R3;
  p.log_n = e;
  p.N = int64_t(1) << e;
  p.batch = batch;
  p.inverse = inverse;
  p.err = err;
  p.sticky = sticky_word();  // unified addressing: the host pointer is the device pointer
  p.ntiles = 0;
  p.wait_polls = g_wait_polls.load(std::memory_order_relaxed);
  const int l3 = ilog2_exact(R3), l2 = ilog2_exact(R2), l1 = ilog2_exact(R1);
  CUtensorMap m1, m2, m3, o2, o3;
  int st;
  // pass 1 source x[b][m3][m2][r]: dims {2 R1, R2, batch R3}, box {32, 1, min(R3, 256)}
  if ((st = make_map(&m1, in, R1, R2, int64_t(batch) * R3, 1, R3 < 256 ? R3 : 256))) return st;
  // pass 2 source S1[b][m2][r][km3]: dims {2 R3, R1, batch R2}, box {32, 1, min(R2, 256)}
  if ((st = make_map(&m2, s1, R3, R1, int64_t(batch) * R2, 1, R2 < 256 ? R2 : 256))) return st;
  // pass 3 source S2[b][km2][r][km3]: dims {2 R3, R1, batch R2}, box {32, min(R1, 256), 1}
  if ((st = make_map(&m3, s2, R3, R1, int64_t(batch) * R2, R1 < 256 ? R1 : 256, 1))) return st;
  // pass 2 destination S2 (TMA stores of row tiles): dims {2 R3, R1, batch R2},
  // box {32, 1, min(R2, 256)}; pass 3 destination X[b][kr][km2][km3]: dims {2 R3, R2, batch R1},
  // box {32, 1, min(R1, 256)}
  if ((st = make_map(&o2, s2, R3, R1, int64_t(batch) * R2, 1, R2 < 256 ? R2 : 256))) return st;
  if ((st = make_map(&o3, out, R3, R2, int64_t(batch) * R1, 1, R1 < 256 ? R1 : 256))) return st;
  p.in = in;
  p.out = s1;
  if ((st = launch_pass<1>(l3, m1, m1, p, batch * R2 * (R1 / kTileCols), s))) return st;
  p.in = s1;
  p.out = s2;
  if ((st = launch_pass<2>(l2, m2, o2, p, batch * R1 * (R3 / kTileCols), s))) return st;
  p.in = s2;
  p.out = out;
  if ((st = launch_pass<3>(l1, m3, o3, p, batch * R2 * (R3 / kTileCols), s))) return st;
  return SP_OK;
}

int check_n(int64_t n, int* e) {
  const int le = ilog2_exact(n);
  if (le < kMinLogN || le > kMaxLogN) {
    set_error("long FFT length %lld: needs a power of two in [2^%d, 2^%d]", (long long)n, kMinLogN,
              kMaxLogN);
    return SP_ERR_UNSUPPORTED;
  }
  *e = le;
  return SP_OK;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Launch geometry and rotation step of the untangle kernels (kUntT indices per thread).
unsigned untangle_blocks(int64_t m, int batch) {
  const int64_t per_row = cdiv(m / 2 + 1, int64_t(kUntB) * kUntT);
  return unsigned(per_row * batch);
}
double2 untangle_step(int64_t m) {
  // exp(-i pi kUntB / m); kUntB / m is a power of two, so the angle is exact before cos/sin
  const double a = 3.141592653589793238462643383279502884 * double(kUntB) / double(m);
  return make_double2(std::cos(a), -std::sin(a));
}

int64_t ws_need(int64_t n_complex, int batch) { return 2 * int64_t(batch) * n_complex * 8 + 256; }

// Real length n = 2 C 2^e with C odd in [1, kMaxMixC] and e in [kMinLogN, kMaxLogN].
int split_real(int64_t n, int* C, int* e, const char* who) {
  int64_t h = n / 2, odd = h;
  while (odd > 0 && odd % 2 == 0) odd /= 2;
  const int le = (n > 0 && n % 2 == 0 && odd <= kMaxMixC) ? ilog2_exact(h / odd) : -1;
  if (le < kMinLogN || le > kMaxLogN) {
    set_error("%s: length %lld is not 2 C 2^e with C odd <= %d and e in [%d, %d]", who,
              (long long)n, kMaxMixC, kMinLogN, kMaxLogN);
    return SP_ERR_UNSUPPORTED;
  }
  *C = int(odd);
  *e = le;
  return SP_OK;
}

// W_n^m = exp(-i pi / C) for n = 2 C m, in FP64
double2 half_branch_twiddle(int C) {
  const double t = 3.141592653589793238462643383279502884 / double(C);
  return make_double2(std::cos(t), -std::sin(t));
}

template <int C>
cudaError_t launch_combine_t(unsigned grid, cudaStream_t s, const float2* Z, float2* X, int64_t m,
                             int64_t ldx, int64_t nout) {
  return launch_pdl(k_mixed_combine<C>, dim3(grid), kUntB, 0, s, Z, X, m, ldx, nout,
                    half_branch_twiddle(C));
}

template <int C>
cudaError_t launch_fold_t(unsigned grid, cudaStream_t s, const float2* X, int64_t ldx,
                          int64_t nbins, float2* Yp, int64_t m, float scale, int64_t kfix,
                          float ffix) {
  return launch_pdl(k_mixed_fold_pretwist<C>, dim3(grid), kUntB, 0, s, X, ldx, nbins, Yp, m,
                    half_branch_twiddle(C), scale, kfix, ffix);
}

#define B2S_MIXED_SWITCH(C, CALL)                                         \
  switch (C) {                                                            \
    case 3: return CALL(3);                                               \
    case 5: return CALL(5);                                               \
    case 7: return CALL(7);                                               \
    case 9: return CALL(9);                                               \
    case 11: return CALL(11);                                             \
    case 13: return CALL(13);                                             \
    case 15: return CALL(15);                                             \
    default: return cudaErrorInvalidValue;                                \
  }

cudaError_t launch_combine(int C, unsigned grid, cudaStream_t s, const float2* Z, float2* X,
                           int64_t m, int64_t ldx, int64_t nout) {
#define B2S_CALL(c) launch_combine_t<c>(grid, s, Z, X, m, ldx, nout)
  B2S_MIXED_SWITCH(C, B2S_CALL)
#undef B2S_CALL
}

cudaError_t launch_fold(int C, unsigned grid, cudaStream_t s, const float2* X, int64_t ldx,
                        int64_t nbins, float2* Yp, int64_t m, float scale, int64_t kfix,
                        float ffix) {
#define B2S_CALL(c) launch_fold_t<c>(grid, s, X, ldx, nbins, Yp, m, scale, kfix, ffix)
  B2S_MIXED_SWITCH(C, B2S_CALL)
#undef B2S_CALL
}
#undef B2S_MIXED_SWITCH

// One-sided spectrum (bins below nout, row stride ldx) of `batch` real rows of n = 2 C m
// samples; s1, s2 hold batch n/2 complex each and err follows them.
int rfft_real(const float* x, float2* X, int batch, int C, int e, int64_t ldx, int64_t nout,
              float2* s1, float2* s2, int* err, cudaStream_t s) {
  const int64_t m = int64_t(1) << e;
  int st;
  if (C == 1) {
    // the n real samples are m interleaved complex values; Z lands in s1 (free after pass 2)
    if ((st = fft3(reinterpret_cast<const float2*>(x), s1, s2, s1, batch, e, 0, err, s)))
      return st;
    B2S_CHECK_CUDA(launch_pdl(k_rfft_untangle, dim3(untangle_blocks(m, batch)), kUntB, 0, s,
                              static_cast<const float2*>(s1), X, m, ldx, nout, untangle_step(m)),
                   "rfft untangle launch");
    return SP_OK;
  }
  const int64_t M = 2 * m;
  // branches D_s (batch C rows of M reals) in s2; their packed transforms Z_s land in s1
  B2S_CHECK_CUDA(launch_pdl(k_mixed_deinterleave, dim3(unsigned(batch * (M / kMixQ))), kMixB, 0,
                            s, x, reinterpret_cast<float*>(s2), C, M),
                 "mixed deinterleave launch");
  if ((st = fft3(s2, s1, s2, s1, batch * C, e, 0, err, s))) return st;
  const unsigned grid = unsigned(cdiv(m / 2 + 1, kUntB) * batch);
  B2S_CHECK_CUDA(launch_combine(C, grid, s, s1, X, m, ldx, nout), "mixed combine launch");
  return SP_OK;
}

// Real rows (n = 2 C m samples each) from one-sided spectra X (nbins bins, row stride ldx),
// every bin times scale and bin kfix also times ffix.
int irfft_real(const float2* X, int64_t ldx, int64_t nbins, float* y, int batch, int C, int e,
               float scale, int64_t kfix, float ffix, float2* s1, float2* s2, int* err,
               cudaStream_t s) {
  const int64_t m = int64_t(1) << e;
  int st;
  if (C == 1) {
    B2S_CHECK_CUDA(launch_pdl(k_irfft_pretwist, dim3(untangle_blocks(m, batch)), kUntB, 0, s, X,
                              ldx, nbins, s2, m, untangle_step(m), scale, kfix, ffix),
                   "irfft pretwist launch");
    // Y (in s2) -> S1 (s1) -> S2 (s2, Y already consumed by pass 1) -> y
    return fft3(s2, s1, s2, reinterpret_cast<float2*>(y), batch, e, 1, err, s);
  }
  const int64_t M = 2 * m;
  const unsigned grid = unsigned(cdiv(m / 2 + 1, kUntB) * batch);
  B2S_CHECK_CUDA(launch_fold(C, grid, s, X, ldx, nbins, s2, m, scale, kfix, ffix),
                 "mixed fold launch");
  // packed branch spectra (s2) -> branch signals D_s in s1 -> interleaved into y
  if ((st = fft3(s2, s1, s2, s1, batch * C, e, 1, err, s))) return st;
  B2S_CHECK_CUDA(launch_pdl(k_mixed_interleave, dim3(unsigned(batch * (M / kMixQ))), kMixB, 0,
                            s, reinterpret_cast<const float*>(s1), y, C, M),
                 "mixed interleave launch");
  return SP_OK;
}

}  // namespace
}  // namespace b2s

extern "C" {

int64_t sp_fft_workspace_size(int64_t n, int batch) {
  using namespace b2s;
  int e;
  if (batch < 1) {
    set_error("batch must be >= 1");
    return SP_ERR_ARG;
  }
  int C;
  const int st = check_n(n, &e) == SP_OK ? SP_OK : split_real(2 * n, &C, &e,
                                                              "sp_fft_workspace_size");
  if (st != SP_OK) return st;
  return ws_need(n, batch);
}

int sp_fft_c64(const float* in, float* out, int batch, int64_t n, int inverse, void* workspace,
               size_t workspace_bytes, void* stream) {
  using namespace b2s;
  int e;
  int st = check_n(n, &e);
  if (st != SP_OK) return st;
  if (!in || !out || !workspace || batch < 1 || !aligned16(in) || !aligned16(out) ||
      !aligned16(workspace)) {
    set_error("sp_fft_c64: null or misaligned (16 B) pointer, or batch < 1");
    return SP_ERR_ARG;
  }
  if (int64_t(workspace_bytes) < ws_need(n, batch)) {
    set_error("workspace too small: need %lld bytes", (long long)ws_need(n, batch));
    return SP_ERR_WORKSPACE;
  }
  auto s = static_cast<cudaStream_t>(stream);
  float2* s1 = static_cast<float2*>(workspace);
  float2* s2 = s1 + int64_t(batch) * n;
  int* err = reinterpret_cast<int*>(s2 + int64_t(batch) * n);
  B2S_CHECK_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s), "error word reset");
  return fft3(reinterpret_cast<const float2*>(in), s1, s2, reinterpret_cast<float2*>(out), batch,
              e, inverse, err, s);
}

int sp_rfft_c64(const float* x, float* X, int batch, int64_t n, int64_t ldx_out, void* workspace,
                size_t workspace_bytes, void* stream) {
  using namespace b2s;
  int e, C;
  int st = split_real(n, &C, &e, "sp_rfft_c64");
  if (st != SP_OK) return st;
  const int64_t h = n / 2;
  if (!x || !X || !workspace || batch < 1 || ldx_out < h + 1 || !aligned16(x) ||
      !aligned16(workspace) || (reinterpret_cast<uintptr_t>(X) & 7u)) {
    set_error("sp_rfft_c64: null or misaligned pointer, batch < 1 or ldx_out < n/2+1");
    return SP_ERR_ARG;
  }
  if (int64_t(workspace_bytes) < ws_need(h, batch)) {
    set_error("workspace too small: need %lld bytes", (long long)ws_need(h, batch));
    return SP_ERR_WORKSPACE;
  }
  auto s = static_cast<cudaStream_t>(stream);
  float2* s1 = static_cast<float2*>(workspace);
  float2* s2 = s1 + int64_t(batch) * h;
  int* err = reinterpret_cast<int*>(s2 + int64_t(batch) * h);
  B2S_CHECK_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s), "error word reset");
  return rfft_real(x, reinterpret_cast<float2*>(X), batch, C, e, ldx_out, h + 1, s1, s2, err, s);
}

int sp_hilbert_c64(const float* x, float* out, int batch, int64_t n, void* workspace,
                   size_t workspace_bytes, void* stream) {
  using namespace b2s;
  int e;
  if (n % 2) {
    set_error("sp_hilbert_c64: n must be even");
    return SP_ERR_UNSUPPORTED;
  }
  const int64_t m = n / 2;
  int st = check_n(m, &e);
  if (st != SP_OK) return st;
  int en;
  if ((st = check_n(n, &en)) != SP_OK) return st;
  if (!x || !out || !workspace || batch < 1 || !aligned16(x) || !aligned16(out) ||
      !aligned16(workspace)) {
    set_error("sp_hilbert_c64: null or misaligned (16 B) pointer, or batch < 1");
    return SP_ERR_ARG;
  }
  if (int64_t(workspace_bytes) < ws_need(n, batch)) {
    set_error("workspace too small: need %lld bytes", (long long)ws_need(n, batch));
    return SP_ERR_WORKSPACE;
  }
  auto s = static_cast<cudaStream_t>(stream);
  float2* s1 = static_cast<float2*>(workspace);
  float2* s2 = s1 + int64_t(batch) * n;
  int* err = reinterpret_cast<int*>(s2 + int64_t(batch) * n);
  B2S_CHECK_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s), "error word reset");
  float2* y = reinterpret_cast<float2*>(out);
  // packed m-point transform of the n reals (Z in s1), the analytic spectrum into `out`, then
  // the n-point inverse transform of `out` in place (pass 1 reads it before pass 3 writes it)
  if ((st = fft3(reinterpret_cast<const float2*>(x), s1, s2, s1, batch, e, 0, err, s))) return st;
  B2S_CHECK_CUDA(launch_pdl(k_hilbert_spectrum, dim3(untangle_blocks(m, batch)), kUntB, 0, s,
                            static_cast<const float2*>(s1), y, m, untangle_step(m)),
                 "hilbert spectrum launch");
  return fft3(y, s1, s2, y, batch, en, 1, err, s);
}

int sp_irfft_f32(const float* X, int64_t ldx, int nbins, float* x, int batch, int64_t n,
                 void* workspace, size_t workspace_bytes, void* stream) {
  using namespace b2s;
  int e, C;
  int st = split_real(n, &C, &e, "sp_irfft_f32");
  if (st != SP_OK) return st;
  const int64_t h = n / 2;
  if (!X || !x || !workspace || batch < 1 || nbins < 1 || ldx < nbins || !aligned16(x) ||
      !aligned16(workspace) || (reinterpret_cast<uintptr_t>(X) & 7u)) {
    set_error("sp_irfft_f32: null or misaligned pointer or bad sizes");
    return SP_ERR_ARG;
  }
  if (int64_t(workspace_bytes) < ws_need(h, batch)) {
    set_error("workspace too small: need %lld bytes", (long long)ws_need(h, batch));
    return SP_ERR_WORKSPACE;
  }
  auto s = static_cast<cudaStream_t>(stream);
  float2* s1 = static_cast<float2*>(workspace);
  float2* s2 = s1 + int64_t(batch) * h;
  int* err = reinterpret_cast<int*>(s2 + int64_t(batch) * h);
  B2S_CHECK_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s), "error word reset");
  return irfft_real(reinterpret_cast<const float2*>(X), ldx, nbins, x, batch, C, e, 1.0f, -1,
                    1.0f, s1, s2, err, s);
}

int64_t sp_resample_workspace_size(int64_t n, int64_t num, int batch) {
  using namespace b2s;
  int e, C;
  int st;
  if (batch < 1) {
    set_error("batch must be >= 1");
    return SP_ERR_ARG;
  }
  if ((st = split_real(n, &C, &e, "sp_resample_f32")) ||
      (st = split_real(num, &C, &e, "sp_resample_f32")))
    return st;
  const int64_t nc = (n > num ? n : num) / 2, m2 = (n < num ? n : num) / 2 + 1;
  return ws_need(nc, batch) + cdiv(int64_t(batch) * m2 * 8, 256) * 256;
}

int sp_resample_f32(const float* x, int batch, int64_t n, float* y, int64_t num, void* workspace,
                    size_t workspace_bytes, void* stream) {
  using namespace b2s;
  int ef, Cf, ei, Ci;
  int st;
  if ((st = split_real(n, &Cf, &ef, "sp_resample_f32")) ||
      (st = split_real(num, &Ci, &ei, "sp_resample_f32")))
    return st;
  if (!x || !y || !workspace || batch < 1 || !aligned16(x) || !aligned16(y) ||
      !aligned16(workspace)) {
    set_error("sp_resample_f32: null or misaligned (16 B) pointer, or batch < 1");
    return SP_ERR_ARG;
  }
  const int64_t need = sp_resample_workspace_size(n, num, batch);
  if (int64_t(workspace_bytes) < need) {
    set_error("workspace too small: need %lld bytes", (long long)need);
    return SP_ERR_WORKSPACE;
  }
  const int64_t nc = (n > num ? n : num) / 2, m = n < num ? n : num, m2 = m / 2 + 1;
  auto s = static_cast<cudaStream_t>(stream);
  float2* s1 = static_cast<float2*>(workspace);
  float2* s2 = s1 + int64_t(batch) * nc;
  int* err = reinterpret_cast<int*>(s2 + int64_t(batch) * nc);
  float2* Xb = reinterpret_cast<float2*>(reinterpret_cast<char*>(err) + 256);
  B2S_CHECK_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s), "error word reset");
  // the m2 lowest bins of rfft_n(x); the unpaired bin m/2 of an even m is doubled (joining the
  // +-m/2 pair, downsampling) or halved (split into a pair, upsampling); scale num/n
  if ((st = rfft_real(x, Xb, batch, Cf, ef, m2, m2, s1, s2, err, s))) return st;
  const int64_t kfix = (m % 2 == 0 && num != n) ? m / 2 : -1;
  const float ffix = num < n ? 2.0f : 0.5f;
  return irfft_real(Xb, m2, m2, y, batch, Ci, ei, float(double(num) / double(n)), kfix, ffix, s1,
                    s2, err, s);
}

int sp_fft_sticky_error(int clear) {
  int* w = b2s::sticky_word();
  if (!w) return 0;
  volatile int* v = w;
  const int st = *v;
  if (clear && st) *v = 0;
  return st;
}

uint32_t sp_fft_set_wait_limit(uint32_t polls) {
  return b2s::g_wait_polls.exchange(polls == 0xffffffffu ? b2s::kMbarSpinLimit : polls);
}

int sp_fft_error_word(const void* workspace, int64_t n, int batch, int64_t* offset) {
  (void)workspace;
  if (!offset || batch < 1 || n < 1) return SP_ERR_ARG;
  *offset = 2 * int64_t(batch) * n * 8;
  return SP_OK;
}

}
