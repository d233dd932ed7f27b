// Instantiations of k_frames_half<..., kFrameStft> (hop == nperseg/2 == nfft/2) for nfft 64..4096;
// lookup detrend index 0 none, 1 constant (time domain), 2 constant (spectral correction).
// Shorter transforms keep the general per-frame kernel (an empty info here).
#include "dispatch.cuh"

namespace b2s {
namespace {
template <int LOG_L, int DET>
struct F {
  static constexpr int LL = LOG_L < 6 ? 6 : LOG_L;
  static constexpr int DD = DET == 2 ? kDetrendConstantSpectral : DET;
  static void launch(dim3 g, int t, size_t sm, cudaStream_t st, const FrameParams& p) {
    k_frames_half<LL, team_log_e<LL>(), kFrameStft, DD><<<g, t, sm, st>>>(p);
  }
  static FrameInfo get() {
    if constexpr (LOG_L < 6) {
      return FrameInfo{};
    } else {
      using CFG = MeanCfg<LL, team_log_e<LL>()>;
      FrameInfo k;
      k.fn = reinterpret_cast<const void*>(&k_frames_half<LL, team_log_e<LL>(), kFrameStft, DD>);
      k.threads = CFG::THREADS;
      k.smem = HalfSmem<CFG>::BYTES;
      k.teams = CFG::TEAMS;
      k.launch = &launch;
      return k;
    }
  }
};
}  // namespace

FrameInfo frame_half_lookup_stft(int log_l, int det) { return lookup_all<FrameInfo, F, kMaxLogLReal>(log_l, det); }

}  // namespace b2s
