// Instantiations of k_welch_mean for every fused nfft and detrend kind.
#include "dispatch.cuh"

namespace b2s {
namespace {
template <int LOG_L, int DET>
struct F {
  static void launch(dim3 g, int t, size_t sm, cudaStream_t st, const MeanParams& p) {
    k_welch_mean<LOG_L, team_log_e<LOG_L>(), DET><<<g, t, sm, st>>>(p);
  }
  static MeanInfo get() {
    using CFG = MeanCfg<LOG_L, team_log_e<LOG_L>()>;
    MeanInfo k;
    k.fn = reinterpret_cast<const void*>(&k_welch_mean<LOG_L, team_log_e<LOG_L>(), DET>);
    k.threads = CFG::THREADS;
    k.smem = welch_mean_smem<CFG>();
    k.teams = CFG::TEAMS;
    k.launch = &launch;
    return k;
  }
};
}  // namespace

MeanInfo mean_lookup_welch(int log_l, int det) { return lookup_all<MeanInfo, F, kMaxLogLReal>(log_l, det); }

}  // namespace b2s
