// Instantiations of k_frames<..., kFrameCross> for every fused nfft and detrend kind.
#include "dispatch.cuh"

namespace b2s {
namespace {
template <int LOG_L, int DET>
struct F {
  static void launch(dim3 g, int t, size_t sm, cudaStream_t st, const FrameParams& p) {
    k_frames<LOG_L, team_log_e<LOG_L>(), DET, kFrameCross><<<g, t, sm, st>>>(p);
  }
  static FrameInfo get() {
    using CFG = MeanCfg<LOG_L, team_log_e<LOG_L>()>;
    FrameInfo k;
    k.fn = reinterpret_cast<const void*>(&k_frames<LOG_L, team_log_e<LOG_L>(), DET, kFrameCross>);
    k.threads = CFG::THREADS;
    k.smem = CFG::SMEM;
    k.teams = CFG::TEAMS;
    k.launch = &launch;
    return k;
  }
};
}  // namespace

FrameInfo frame_lookup_cross(int log_l, int det) { return lookup_all<FrameInfo, F, kMaxLogLReal>(log_l, det); }

}  // namespace b2s
