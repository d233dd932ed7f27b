// Instantiations of the two-sided (complex) fused istft kernel for every power-of-two nfft in
// [2, 4096].
#include "dispatch.cuh"

namespace b2s {
namespace {
template <int LOG_L, int UNUSED>
struct F {
  static constexpr int LL = LOG_L < 1 ? 1 : LOG_L;
  static void launch(dim3 g, int t, size_t sm, cudaStream_t st, const IstftParams& p) {
    k_istft_cplx<LL, team_log_e<LL>()><<<g, t, sm, st>>>(p);
  }
  static IstftInfo get() {
    using CFG = IstftCplxCfg<LL, team_log_e<LL>()>;
    IstftInfo k;
    k.fn = reinterpret_cast<const void*>(&k_istft_cplx<LL, team_log_e<LL>()>);
    k.threads = CFG::THREADS;
    k.smem = CFG::SMEM;
    k.teams = CFG::TEAMS;
    k.launch = &launch;
    return k;
  }
};
}  // namespace

IstftInfo istft_cplx_lookup(int log_l) { return lookup_all<IstftInfo, F>(log_l, 0); }

}  // namespace b2s
