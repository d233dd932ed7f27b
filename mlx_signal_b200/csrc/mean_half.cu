// Instantiations of k_welch_half (50%-overlap welch) for every fused nfft >= 2; lookup detrend
// index 0 none, 1 constant (time domain), 2 constant (spectral correction).
#include "dispatch.cuh"

namespace b2s {
namespace {
template <int LOG_L, int DET>
struct F {
  static constexpr int LL = LOG_L < 1 ? 1 : LOG_L;
  // lookup index 2 selects the spectral constant detrend
  static constexpr int DD = DET == 2 ? kDetrendConstantSpectral : DET;
  static void launch(dim3 g, int t, size_t sm, cudaStream_t st, const MeanParams& p) {
    launch_half(k_welch_half<LL, team_log_e<LL>(), DD>, g, t, sm, st, p);
  }
  static MeanInfo get() {
    using CFG = MeanCfg<LL, team_log_e<LL>()>;
    MeanInfo k;
    k.fn = reinterpret_cast<const void*>(&k_welch_half<LL, team_log_e<LL>(), DD>);
    k.threads = CFG::THREADS;
    k.smem = welch_half_smem<CFG>();
    k.teams = CFG::TEAMS;
    k.launch = &launch;
    return k;
  }
};
}  // namespace

MeanInfo mean_lookup_welch_half(int log_l, int det) { return lookup_all<MeanInfo, F, kMaxLogLReal>(log_l, det); }

}  // namespace b2s
