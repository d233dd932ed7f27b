// Instantiations of k_frames_cplx<..., POWER=1> (complex input, power) for every fused nfft
// and detrend kind.
#include "dispatch.cuh"

namespace b2s {
namespace {
template <int LOG_L, int DET>
struct F {
  static void launch(dim3 g, int t, size_t sm, cudaStream_t st, const FrameParams& p) {
    k_frames_cplx<LOG_L, team_log_e<LOG_L>(), DET, 1><<<g, t, sm, st>>>(p);
  }
  static FrameInfo get() {
    using CFG = MeanCfg<LOG_L, team_log_e<LOG_L>()>;
    FrameInfo k;
    k.fn = reinterpret_cast<const void*>(&k_frames_cplx<LOG_L, team_log_e<LOG_L>(), DET, 1>);
    k.threads = CFG::THREADS;
    k.smem = CFG::SMEM;
    k.teams = CFG::TEAMS;
    k.launch = &launch;
    return k;
  }
};
}  // namespace

FrameInfo cplx_lookup_frames_power(int log_l, int det) {
  return lookup_all<FrameInfo, F>(log_l, det);
}

}  // namespace b2s
