// Instantiations of k_welch_half (50%-overlap welch) for every fused nfft >= 2, with and without
// the shared-memory block totals; lookup detrend index 0 none, 1 constant (time domain), 2
// constant (spectral correction).
#include "dispatch.cuh"

namespace b2s {
namespace {
// BLOCKED: the instantiation with shared-memory block totals (long team ranges). The plain
// register sums are used from nfft 2048 up, whose kernels are bound by shared-memory traffic
// (measured 3-5 % faster at 4096 and 8192); nfft <= 1024 keeps the block totals in every case
// (at 1024, FP32-bound, plain sums measured ~0.8 % slower).
template <bool BLOCKED>
struct Fam {
  template <int LOG_L, int DET>
  struct F {
    static constexpr int LL = LOG_L < 1 ? 1 : LOG_L;
    static constexpr bool B = BLOCKED || LL <= 10;
    // lookup index 2 selects the spectral constant detrend
    static constexpr int DD = DET == 2 ? kDetrendConstantSpectral : DET;
    static void launch(dim3 g, int t, size_t sm, cudaStream_t st, const MeanParams& p) {
      launch_half(k_welch_half<LL, team_log_e<LL>(), DD, B>, g, t, sm, st, p);
    }
    static MeanInfo get() {
      using CFG = MeanCfg<LL, team_log_e<LL>()>;
      MeanInfo k;
      k.fn = reinterpret_cast<const void*>(&k_welch_half<LL, team_log_e<LL>(), DD, B>);
      k.threads = CFG::THREADS;
      k.smem = welch_half_smem<CFG>();
      k.teams = CFG::TEAMS;
      k.launch = &launch;
      return k;
    }
  };
};
}  // namespace

MeanInfo mean_lookup_welch_half(int log_l, int det, bool blocked) {
  return blocked ? lookup_all<MeanInfo, Fam<true>::F, kMaxLogLReal>(log_l, det)
                 : lookup_all<MeanInfo, Fam<false>::F, kMaxLogLReal>(log_l, det);
}

}  // namespace b2s
