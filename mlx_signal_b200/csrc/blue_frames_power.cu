// Instantiations of k_blue_frames<..., kFramePower> (non-power-of-two nfft) for transform
// lengths 2^4..2^12 and detrend none / constant / linear.
#include "dispatch.cuh"

namespace b2s {
namespace {
template <int LOG_L, int DET>
struct F {
  static constexpr int LM = LOG_L < 4 ? 4 : LOG_L;
  static void launch(dim3 g, int t, size_t sm, cudaStream_t st, const FrameParams& p) {
    k_blue_frames<LM, DET, kFramePower><<<g, t, sm, st>>>(p);
  }
  static FrameInfo get() {
    if constexpr (LOG_L < 4) {
      return FrameInfo{};
    } else {
      using CFG = BlueCfg<LM>;
      FrameInfo k;
      k.fn = reinterpret_cast<const void*>(&k_blue_frames<LM, DET, kFramePower>);
      k.threads = CFG::THREADS;
      k.smem = CFG::SMEM;
      k.teams = CFG::TEAMS;
      k.launch = &launch;
      return k;
    }
  }
};
}  // namespace

FrameInfo blue_lookup_frames_power(int log_m, int det) {
  return lookup_all<FrameInfo, F, kMaxLogLReal>(log_m, det);
}

}  // namespace b2s
