// Instantiations of k_cross_half (50%-overlap csd and coherence) for every fused nfft >= 2;
// lookup detrend index 0 none, 1 constant (time domain), 2 constant (spectral correction).
#include "dispatch.cuh"

namespace b2s {
namespace {
template <bool CSD>
struct Mode {
  template <int LOG_L, int DET>
  struct F {
    static constexpr int LL = LOG_L < 1 ? 1 : LOG_L;
    static constexpr int DD = DET == 2 ? kDetrendConstantSpectral : DET;
    static void launch(dim3 g, int t, size_t sm, cudaStream_t st, const MeanParams& p) {
      launch_half(k_cross_half<LL, team_log_e<LL>(), DD, CSD>, g, t, sm, st, p);
    }
    static MeanInfo get() {
      using CFG = MeanCfg<LL, team_log_e<LL>()>;
      MeanInfo k;
      k.fn = reinterpret_cast<const void*>(&k_cross_half<LL, team_log_e<LL>(), DD, CSD>);
      k.threads = CFG::THREADS;
      k.smem = HalfSmem<CFG>::BYTES;
      k.teams = CFG::TEAMS;
      k.launch = &launch;
      return k;
    }
  };
};
}  // namespace

MeanInfo mean_lookup_cross_half(int log_l, int det, bool csd) {
  return csd ? lookup_all<MeanInfo, Mode<true>::F, kMaxLogLReal>(log_l, det)
             : lookup_all<MeanInfo, Mode<false>::F, kMaxLogLReal>(log_l, det);
}

}  // namespace b2s
