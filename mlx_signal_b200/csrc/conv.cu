// C-ABI: fused overlap-save FFT convolution (real rows, one shared real filter).
#include <utility>

#include "capi_common.h"
#include "conv_kernels.cuh"

namespace b2s {
namespace {

constexpr int kConvMinLog = 8, kConvMaxLog = 12;
constexpr int kConvMaxTaps = (1 << kConvMaxLog) / 2 + 1;  // keeps STEP >= L/2 at L = 4096

struct ConvInfo {
  const void* fn = nullptr;
  int threads = 0, teams = 0;
  size_t smem = 0;
  void (*launch)(dim3, int, size_t, cudaStream_t, const ConvParams&) = nullptr;
};

template <int LOG_L>
void launch_conv(dim3 g, int th, size_t sm, cudaStream_t s, const ConvParams& p) {
  k_conv_ols<LOG_L><<<g, th, sm, s>>>(p);
}

template <int LOG_L>
ConvInfo conv_info() {
  using CFG = ConvCfg<LOG_L>;
  ConvInfo f;
  f.fn = reinterpret_cast<const void*>(&k_conv_ols<LOG_L>);
  f.threads = CFG::THREADS;
  f.teams = CFG::TEAMS;
  f.smem = CFG::SMEM;
  f.launch = &launch_conv<LOG_L>;
  return f;
}

template <int... LS>
ConvInfo conv_lookup(int log_l, std::integer_sequence<int, LS...>) {
  ConvInfo out;
  (void)((log_l == LS + kConvMinLog ? (out = conv_info<LS + kConvMinLog>(), true) : false) || ...);
  return out;
}

// Block length for n2 taps: the power of two in [2^8, 2^12] with the fewest FFT operations per
// output sample, L log2 L / (L - n2 + 1), among those keeping STEP = L - n2 + 1 >= L/2.
int conv_block_log(int n2) {
  int best = -1;
  double best_cost = 0.0;
  for (int lg = kConvMinLog; lg <= kConvMaxLog; ++lg) {
    const int L = 1 << lg, step = L - n2 + 1;
    if (2 * step < L) continue;
    const double cost = double(L) * lg / step;
    if (best < 0 || cost < best_cost) {
      best = lg;
      best_cost = cost;
    }
  }
  return best;
}

}  // namespace
}  // namespace b2s

extern "C" {

int sp_conv_block_len(int n2) {
  if (n2 < 1 || n2 > b2s::kConvMaxTaps) {
    b2s::set_error("filter length %d outside the fused convolution range [1, %d]", n2,
                   b2s::kConvMaxTaps);
    return SP_ERR_UNSUPPORTED;
  }
  return 1 << b2s::conv_block_log(n2);
}

int sp_conv_ols_f32(const float* x, int64_t rows, int64_t n1, int64_t ld_x, const float* h,
                    int n2, int64_t j0, int64_t nout, float* out, int64_t ld_out, void* stream) {
  using namespace b2s;
  if (rows < 0 || n1 < 1 || n2 < 1 || ld_x < n1 || nout < 0 || ld_out < nout || j0 < 0 ||
      j0 + nout > n1 + n2 - 1) {
    set_error("invalid convolution arguments (rows=%lld n1=%lld n2=%d j0=%lld nout=%lld)",
              (long long)rows, (long long)n1, n2, (long long)j0, (long long)nout);
    return SP_ERR_ARG;
  }
  if (n2 > kConvMaxTaps) {
    set_error("filter length %d outside the fused convolution range [1, %d]", n2, kConvMaxTaps);
    return SP_ERR_UNSUPPORTED;
  }
  if (rows == 0 || nout == 0) return SP_OK;
  if (!x || !h || !out) {
    set_error("null pointer");
    return SP_ERR_ARG;
  }
  const int lg = conv_block_log(n2);
  const ConvInfo f =
      conv_lookup(lg, std::make_integer_sequence<int, kConvMaxLog - kConvMinLog + 1>{});
  ConvParams p;
  p.x = x;
  p.h = h;
  p.out = out;
  p.ld_x = ld_x;
  p.ld_out = ld_out;
  p.rows = rows;
  p.n1 = n1;
  p.n2 = n2;
  p.j0 = j0;
  p.nout = nout;
  p.step = (1 << lg) - n2 + 1;
  p.nblk = cdiv(nout, p.step);
  p.total = rows * p.nblk;
  int sms = 0;
  const int nb = resident_ctas(f.fn, f.threads, f.smem, &sms);
  if (nb <= 0) {
    set_error("no resident CTA for the convolution kernel (L=%d)", 1 << lg);
    return SP_ERR_UNSUPPORTED;
  }
  const int64_t npairs = cdiv(p.total, 2);
  int64_t blocks = cdiv(npairs, f.teams);
  const int64_t cap = int64_t(nb) * sms;
  if (blocks > cap) blocks = cap;
  f.launch(dim3(unsigned(blocks)), f.threads, f.smem, static_cast<cudaStream_t>(stream), p);
  B2S_CHECK_CUDA(cudaGetLastError(), "convolution kernel launch");
  return SP_OK;
}

}
