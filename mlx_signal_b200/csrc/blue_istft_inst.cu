// Instantiations of the chirp-z fused istft (non-power-of-two nfft <= 2048) for transform lengths
// 2^4..2^12.
#include "blue_istft.cuh"
#include "dispatch.cuh"

namespace b2s {
namespace {
template <int LOG_L, int UNUSED>
struct F {
  static constexpr int LM = LOG_L < 4 ? 4 : LOG_L;
  static void launch(dim3 g, int t, size_t sm, cudaStream_t st, const IstftParams& p) {
    k_blue_istft<LM><<<g, t, sm, st>>>(p);
  }
  static IstftInfo get() {
    if constexpr (LOG_L < 4) {
      return IstftInfo{};
    } else {
      using CFG = BlueIstftCfg<LM>;
      IstftInfo k;
      k.fn = reinterpret_cast<const void*>(&k_blue_istft<LM>);
      k.threads = CFG::THREADS;
      k.smem = CFG::SMEM;
      k.teams = CFG::TEAMS;
      k.launch = &launch;
      return k;
    }
  }
};
}  // namespace

IstftInfo istft_blue_lookup(int log_m) { return lookup_all<IstftInfo, F>(log_m, 0); }

}  // namespace b2s
