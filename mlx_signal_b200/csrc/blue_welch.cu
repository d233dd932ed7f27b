// Instantiations of k_blue_welch (non-power-of-two nfft) for transform lengths 2^4..2^13 and
// detrend none / constant / linear.
#include "dispatch.cuh"

namespace b2s {
namespace {
template <int LOG_L, int DET>
struct F {
  static constexpr int LM = LOG_L < 4 ? 4 : LOG_L;
  static void launch(dim3 g, int t, size_t sm, cudaStream_t st, const MeanParams& p) {
    k_blue_welch<LM, DET><<<g, t, sm, st>>>(p);
  }
  static MeanInfo get() {
    if constexpr (LOG_L < 4) {
      return MeanInfo{};
    } else {
      using CFG = BlueCfg<LM>;
      MeanInfo k;
      k.fn = reinterpret_cast<const void*>(&k_blue_welch<LM, DET>);
      k.threads = CFG::THREADS;
      k.smem = CFG::SMEM;
      k.teams = CFG::TEAMS;
      k.launch = &launch;
      return k;
    }
  }
};
}  // namespace

MeanInfo blue_lookup_welch(int log_m, int det) { return lookup_all<MeanInfo, F, kMaxLogLReal>(log_m, det); }

}  // namespace b2s
