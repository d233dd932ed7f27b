// C-ABI support: error text, version, occupancy cache.
#include "capi_common.h"

namespace b2s {

namespace {
thread_local std::string g_last_error;
std::mutex g_occ_mu;
struct OccKey {
  const void* k;
  int dev, threads;
  size_t smem;
  bool operator==(const OccKey& o) const {
    return k == o.k && dev == o.dev && threads == o.threads && smem == o.smem;
  }
};
struct OccHash {
  size_t operator()(const OccKey& o) const {
    return std::hash<const void*>()(o.k) ^ (size_t(o.dev) << 48) ^ (size_t(o.threads) << 32) ^ o.smem;
  }
};
std::unordered_map<OccKey, int, OccHash> g_occ;
std::unordered_map<int, int> g_sms;
}  // namespace

void set_error(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

int cuda_status(cudaError_t e, const char* where) {
  set_error("%s: %s", where, cudaGetErrorString(e));
  return SP_ERR_CUDA;
}

int resident_ctas(const void* kernel, int threads, size_t smem, int* num_sms) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  std::lock_guard<std::mutex> lk(g_occ_mu);
  auto its = g_sms.find(dev);
  if (its == g_sms.end()) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
    its = g_sms.emplace(dev, sms).first;
  }
  *num_sms = its->second;
  OccKey key{kernel, dev, threads, smem};
  auto it = g_occ.find(key);
  if (it != g_occ.end()) return it->second;
  if (smem > 48 * 1024) {
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) !=
        cudaSuccess)
      return -1;
  }
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, smem) != cudaSuccess)
    return -1;
  g_occ.emplace(key, nb);
  return nb;
}

}  // namespace b2s

extern "C" {

int sp_version(void) { return SP_VERSION; }

const char* sp_last_error(void) { return b2s::g_last_error.c_str(); }

}
