// C-ABI and kernel entry of the persistent batched launch (welch requests and streaming-STFT
// chunks of uneven size and segment length in one batched launch over device work queues).
#include <algorithm>
#include <mutex>
#include <numeric>
#include <vector>

#include "batch_kernels.cuh"
#include "capi_common.h"
#include "dispatch.cuh"

namespace b2s {

// Inter-pass twiddles of the 2048-point class, which exceed the 128-thread kernel's shared
// twiddle slot; built once per device by k_batch_init (FP64 sincospi, rounded once, as the
// shared tables).
using BatchPlan11 = Plan<11, batch_log_e<11>()>;
__device__ float2 g_batch_tw11[BatchPlan11::TW];

__global__ void k_batch_init() {
  build_twiddles<BatchPlan11>(g_batch_tw11, int(blockIdx.x * blockDim.x + threadIdx.x),
                              int(gridDim.x * blockDim.x));
}

constexpr int kBatchMinBlocks = 3;
constexpr int kBatchBigMinBlocks = 2;

// Queue words (int): [0] next item and [1] CTAs finished of the 128-thread kernel, [2] and [3]
// the same for the 256-thread kernel.
__device__ __forceinline__ void batch_take(const BatchParams& bp, int* qnext, int first, int end,
                                           int nreq, int* s_item, int* s_req) {
  if (threadIdx.x == 0) {
    const int it = first + atomicAdd(qnext, 1);
    const int* item_begin = reinterpret_cast<const int*>(bp.desc + sizeof(BatchHeader));
    int lo = 0;
    if (it < end) {  // largest request index with item_begin <= it
      int hi = nreq - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (ldg_i(item_begin + mid) <= it) lo = mid;
        else hi = mid - 1;
      }
    }
    *s_item = it;
    *s_req = lo;
  }
  __syncthreads();
}

// The last CTA out of a kernel returns its two queue words to zero for the next launch.
__device__ __forceinline__ void batch_finish(int* q) {
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(q + 1, 1) == int(gridDim.x) - 1) {
      q[0] = 0;
      q[1] = 0;
      __threadfence();
    }
  }
}

// Classes 256 ... 2048 (items [first_small, total)). Launched as a programmatic dependent of
// k_batch_big: its CTAs take SMs as the 4096-class CTAs drain. The two kernels share no data
// (disjoint requests, partial slots, row counters and queue words); each CTA waits for the
// 4096-class grid before it exits, so the launch completes after both.
__global__ void __launch_bounds__(kBatchThreads, kBatchMinBlocks) k_batch(BatchParams bp) {
  extern __shared__ float4 smem[];
  __shared__ int s_item, s_req, s_nrows;
  __shared__ int s_rows[16];
  const BatchHeader* hdr = reinterpret_cast<const BatchHeader*>(bp.desc);
  const int* item_begin = reinterpret_cast<const int*>(bp.desc + sizeof(BatchHeader));
  const int nreq = ldg_i(&hdr->nreq);
  const int total = ldg_i(&hdr->total_items);
  const int first = ldg_i(&hdr->first_small);
  const BatchReqDev* reqs = reinterpret_cast<const BatchReqDev*>(bp.desc + batch_req_offset(nreq));
  BatchTables cur;
  cur.log_l = -1;
  cur.win = nullptr;
  cur.wdft = nullptr;
  cur.n_low = -1;
  for (;;) {
    batch_take(bp, bp.queue, first, total, nreq, &s_item, &s_req);
    const int it = s_item;
    if (it >= total) break;
    const int ri = s_req;
    const BatchReqDev* rq = reqs + ri;
    const int local = it - ldg_i(item_begin + ri);
    switch (ldg_i(&rq->log_l)) {
      case 8: batch_item<8, batch_log_e<8>(), kBatchThreads, BatchSmall>(rq, local, smem, cur, g_batch_tw11, s_rows, &s_nrows); break;
      case 9: batch_item<9, batch_log_e<9>(), kBatchThreads, BatchSmall>(rq, local, smem, cur, g_batch_tw11, s_rows, &s_nrows); break;
      case 10: batch_item<10, batch_log_e<10>(), kBatchThreads, BatchSmall>(rq, local, smem, cur, g_batch_tw11, s_rows, &s_nrows); break;
      case 11: batch_item<11, batch_log_e<11>(), kBatchThreads, BatchSmall>(rq, local, smem, cur, g_batch_tw11, s_rows, &s_nrows); break;
      default: break;  // the encoder places the 4096 class before first_small
    }
    __syncthreads();
  }
  pdl_wait();
  batch_finish(bp.queue);
}

// The 4096-point class (items [0, first_small)): one 256-thread team per CTA, 16 points per thread,
// every table in shared memory. Starts its dependent (k_batch) at once.
__global__ void __launch_bounds__(kBatchBigThreads, kBatchBigMinBlocks) k_batch_big(BatchParams bp) {
  extern __shared__ float4 smem[];
  __shared__ int s_item, s_req, s_nrows;
  __shared__ int s_rows[16];
  pdl_trigger();
  const BatchHeader* hdr = reinterpret_cast<const BatchHeader*>(bp.desc);
  const int* item_begin = reinterpret_cast<const int*>(bp.desc + sizeof(BatchHeader));
  const int nreq = ldg_i(&hdr->nreq);
  const int end = ldg_i(&hdr->first_small);
  const BatchReqDev* reqs = reinterpret_cast<const BatchReqDev*>(bp.desc + batch_req_offset(nreq));
  BatchTables cur;
  cur.log_l = -1;
  cur.win = nullptr;
  cur.wdft = nullptr;
  cur.n_low = -1;
  for (;;) {
    batch_take(bp, bp.queue + 2, 0, end, nreq, &s_item, &s_req);
    const int it = s_item;
    if (it >= end) break;
    const int ri = s_req;
    const BatchReqDev* rq = reqs + ri;
    const int local = it - ldg_i(item_begin + ri);
    if (ldg_i(&rq->log_l) == 12)
      batch_item<12, batch_log_e<12>(), kBatchBigThreads, BatchBig>(rq, local, smem, cur, nullptr,
                                                                    s_rows, &s_nrows);
    __syncthreads();
  }
  batch_finish(bp.queue + 2);
}

namespace {

constexpr int64_t kQueueBytes = 256;

bool batch_class(int nperseg, int* log_l) {
  const int l = ilog2_exact(nperseg);
  if (l == 8 || l == 9 || l == 10 || l == 11 || l == 12) {
    *log_l = l;
    return true;
  }
  return false;
}

int teams_of(int log_l) {
  const int P = (1 << log_l) >> batch_log_e_rt(log_l);
  return P >= 64 ? 1 : kBatchThreads / P;
}

int64_t align256(int64_t v) { return (v + 255) & ~int64_t(255); }

int64_t stream_frames(int64_t tail_len, int64_t n, int nperseg, int hop, int64_t* new_tail) {
  const int64_t m = tail_len + n;
  const int64_t f = m >= nperseg ? (m - nperseg) / hop + 1 : 0;
  if (new_tail) *new_tail = m - f * hop;
  return f;
}

struct ReqPlan {
  int log_l = 0, nseg = 0, G = 0, chunks = 0, tasks = 0, items = 0, nbins = 0, new_tail = 0;
  int64_t part_floats = 0;
};

int plan_request(const sp_batch_request& r, int idx, ReqPlan* p) {
  if (!batch_class(r.nperseg, &p->log_l)) {
    set_error("request %d: nperseg=%d is not a batched class (256, 512, 1024, 2048, 4096)", idx,
              r.nperseg);
    return SP_ERR_UNSUPPORTED;
  }
  const int L = r.nperseg;
  if (r.rows < 0 || r.rows >= (int64_t(1) << 24) || (!r.x && r.n > 0 && r.rows > 0) || !r.win ||
      r.ld < r.n || r.n < 0 ||
      r.n >= (int64_t(1) << 31) || r.seg_per_task < 0) {
    set_error("request %d: invalid rows/n/ld or null pointer", idx);
    return SP_ERR_ARG;
  }
  const int teams = teams_of(p->log_l);
  if (r.kind == SP_BATCH_WELCH) {
    if (r.hop != L / 2 || r.n < L || (r.detrend != SP_DETREND_NONE &&
                                      r.detrend != SP_DETREND_CONSTANT)) {
      set_error("request %d: batched welch needs hop == nperseg/2, n >= nperseg and detrend "
                "none/constant", idx);
      return SP_ERR_ARG;
    }
    const int P = L >> batch_log_e_rt(p->log_l);
    if (r.detrend == SP_DETREND_CONSTANT && (!r.win_dft_low || r.n_low < 1 || r.n_low > P)) {
      set_error("request %d: constant detrend needs 1 <= n_low <= %d window-spectrum bins", idx,
                P);
      return SP_ERR_ARG;
    }
    if (!r.out) {
      set_error("request %d: null output", idx);
      return SP_ERR_ARG;
    }
    p->nseg = int((r.n - L) / (L / 2) + 1);
    int G = r.seg_per_task > 0 ? r.seg_per_task : 64;
    G += G & 1;
    if (G > p->nseg + (p->nseg & 1)) G = p->nseg + (p->nseg & 1);
    p->G = G;
    p->chunks = int(cdiv(p->nseg, G));
    p->nbins = r.onesided ? L / 2 + 1 : L;
    p->part_floats = r.rows * int64_t(p->chunks) * welch_slot_floats(L);
  } else if (r.kind == SP_BATCH_STFT_STREAM) {
    if (r.hop < 1 || r.hop > L || r.tail_len < 0 || r.tail_len >= L || r.tail_ld < L ||
        !r.tail_in || !r.tail_out || r.tail_in == r.tail_out || r.onesided != 1) {
      set_error("request %d: stream chunk needs 1 <= hop <= nperseg, 0 <= tail_len < nperseg, "
                "tail_ld >= nperseg, distinct tail buffers and one-sided output", idx);
      return SP_ERR_ARG;
    }
    int64_t nt = 0;
    const int64_t f = stream_frames(r.tail_len, r.n, L, r.hop, &nt);
    if (f >= (int64_t(1) << 30)) {
      set_error("request %d: too many frames", idx);
      return SP_ERR_ARG;
    }
    if (f > 0 && !r.out) {
      set_error("request %d: null output", idx);
      return SP_ERR_ARG;
    }
    p->nseg = int(f);
    p->new_tail = int(nt);
    int G = r.seg_per_task > 0 ? r.seg_per_task : 16;
    G += G & 1;
    p->G = G;
    p->chunks = f > 0 ? int(cdiv(f, G)) : 1;
    p->nbins = L / 2 + 1;
  } else {
    set_error("request %d: unknown kind %d", idx, r.kind);
    return SP_ERR_ARG;
  }
  const int64_t tasks = r.rows * int64_t(p->chunks);
  if (tasks >= (int64_t(1) << 30)) {
    set_error("request %d: too many tasks", idx);
    return SP_ERR_ARG;
  }
  p->tasks = int(tasks);
  p->items = int(cdiv(tasks, teams));
  return SP_OK;
}

// Encoding order: larger FFT classes first (longer items start early), input order within a
// class.
std::vector<int> batch_order(const sp_batch_request* reqs, int nreq) {
  std::vector<int> ord(nreq);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(),
                   [&](int a, int b) { return reqs[a].nperseg > reqs[b].nperseg; });
  return ord;
}

int plan_all(const sp_batch_request* reqs, int nreq, std::vector<ReqPlan>* plans,
             int64_t* ws_bytes, int64_t* total_items) {
  if (nreq < 0 || (nreq > 0 && !reqs)) {
    set_error("invalid request array");
    return SP_ERR_ARG;
  }
  plans->assign(size_t(nreq), ReqPlan());
  int64_t cnt = 0, part = 0, items = 0;
  for (int i = 0; i < nreq; ++i) {
    const int st = plan_request(reqs[i], i, &(*plans)[i]);
    if (st != SP_OK) return st;
    if (reqs[i].kind == SP_BATCH_WELCH) {
      cnt += reqs[i].rows;
      part += (*plans)[i].part_floats;
    }
    items += (*plans)[i].items;
  }
  if (items >= (int64_t(1) << 31)) {
    set_error("batch too large: %lld work items", (long long)items);
    return SP_ERR_ARG;
  }
  // A stream's next chunk reads the tail its previous chunk writes: two chunks of one stream
  // (a shared tail buffer) cannot be in the same launch.
  std::vector<std::pair<const void*, int>> tails;
  for (int i = 0; i < nreq; ++i) {
    if (reqs[i].kind != SP_BATCH_STFT_STREAM) continue;
    tails.emplace_back(reqs[i].tail_in, i);
    tails.emplace_back(reqs[i].tail_out, i);
  }
  std::sort(tails.begin(), tails.end());
  for (size_t k = 1; k < tails.size(); ++k) {
    if (tails[k].first == tails[k - 1].first) {
      set_error("requests %d and %d share a stream tail buffer (one chunk per stream per batch)",
                tails[k - 1].second, tails[k].second);
      return SP_ERR_ARG;
    }
  }
  *ws_bytes = kQueueBytes + align256(cnt * 4) + part * 4;
  *total_items = items;
  return SP_OK;
}

std::mutex g_batch_mu;
constexpr int kMaxDev = 64;
bool g_batch_ready[kMaxDev] = {};

}  // namespace
}  // namespace b2s

extern "C" {

int64_t sp_batch_stream_frames(int64_t tail_len, int64_t n, int nperseg, int hop,
                               int64_t* new_tail_len) {
  if (tail_len < 0 || n < 0 || nperseg < 1 || hop < 1 || hop > nperseg) {
    b2s::set_error("invalid stream chunk geometry");
    return SP_ERR_ARG;
  }
  return b2s::stream_frames(tail_len, n, nperseg, hop, new_tail_len);
}

int sp_batch_supported(int nperseg) {
  int l = 0;
  return b2s::batch_class(nperseg, &l) ? 1 : 0;
}

int sp_batch_plan(const sp_batch_request* reqs, int nreq, int64_t* desc_bytes,
                  int64_t* ws_bytes) {
  std::vector<b2s::ReqPlan> plans;
  int64_t ws = 0, items = 0;
  const int st = b2s::plan_all(reqs, nreq, &plans, &ws, &items);
  if (st != SP_OK) return st;
  if (desc_bytes) *desc_bytes = b2s::batch_desc_bytes(nreq);
  if (ws_bytes) *ws_bytes = ws;
  return SP_OK;
}

int sp_batch_encode(const sp_batch_request* reqs, int nreq, void* ws, size_t ws_bytes,
                    void* desc_host, size_t desc_bytes) {
  using namespace b2s;
  std::vector<ReqPlan> plans;
  int64_t need = 0, items = 0;
  int st = plan_all(reqs, nreq, &plans, &need, &items);
  if (st != SP_OK) return st;
  if (!desc_host || desc_bytes < size_t(batch_desc_bytes(nreq))) {
    set_error("descriptor buffer too small: need %lld bytes", (long long)batch_desc_bytes(nreq));
    return SP_ERR_WORKSPACE;
  }
  if (!ws || ws_bytes < size_t(need)) {
    set_error("batch workspace too small: need %lld bytes, got %zu", (long long)need, ws_bytes);
    return SP_ERR_WORKSPACE;
  }
  unsigned char* blob = static_cast<unsigned char*>(desc_host);
  BatchHeader* hdr = reinterpret_cast<BatchHeader*>(blob);
  hdr->magic = kBatchMagic;
  hdr->nreq = nreq;
  hdr->total_items = int(items);
  hdr->first_small = 0;
  int* ib = reinterpret_cast<int*>(blob + sizeof(BatchHeader));
  BatchReqDev* rd = reinterpret_cast<BatchReqDev*>(blob + batch_req_offset(nreq));
  unsigned char* wsb = static_cast<unsigned char*>(ws);
  int* cnt = reinterpret_cast<int*>(wsb + kQueueBytes);
  int64_t cnt_total = 0;
  for (int i = 0; i < nreq; ++i)
    if (reqs[i].kind == SP_BATCH_WELCH) cnt_total += reqs[i].rows;
  float* part = reinterpret_cast<float*>(wsb + kQueueBytes + align256(cnt_total * 4));
  const std::vector<int> ord = batch_order(reqs, nreq);
  int item = 0;
  for (int j = 0; j < nreq; ++j) {
    const int i = ord[size_t(j)];
    const sp_batch_request& r = reqs[i];
    const ReqPlan& p = plans[size_t(i)];
    ib[j] = item;
    item += p.items;
    if (p.log_l == 12) hdr->first_small = item;  // the class sorts first (batch_order)
    BatchReqDev d = {};
    d.x = r.x;
    d.win = r.win;
    d.out = r.out;
    d.ld = r.ld;
    d.kind = r.kind;
    d.log_l = p.log_l;
    d.rows = int(r.rows);
    d.nseg = p.nseg;
    d.G = p.G;
    d.chunks = p.chunks;
    d.tasks = p.tasks;
    d.nbins = p.nbins;
    d.hop = r.hop;
    d.scale = r.scale;
    d.onesided = r.onesided;
    if (r.kind == SP_BATCH_WELCH) {
      d.wdft = r.detrend == SP_DETREND_CONSTANT
                   ? reinterpret_cast<const float2*>(r.win_dft_low) : nullptr;
      d.n_low = r.detrend == SP_DETREND_CONSTANT ? r.n_low : 0;
      d.cnt = cnt;
      d.part = part;
      cnt += r.rows;
      part += p.part_floats;
    } else {
      d.tail_in = r.tail_in;
      d.tail_out = r.tail_out;
      d.tail_ld = r.tail_ld;
      d.tail_len = r.tail_len;
      d.new_tail_len = p.new_tail;
    }
    rd[j] = d;
  }
  ib[nreq] = item;
  return SP_OK;
}

int sp_batch_max_grid(void) {
  int sms = 0;
  const int nb = b2s::resident_ctas(reinterpret_cast<const void*>(b2s::k_batch),
                                    b2s::kBatchThreads, b2s::kBatchSmemBytes, &sms);
  return nb > 0 ? nb * sms : 0;
}

int sp_batch_run(const void* desc_dev, void* ws, int grid, void* stream) {
  using namespace b2s;
  if (!desc_dev || !ws) {
    set_error("null descriptor or workspace");
    return SP_ERR_ARG;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int dev = 0;
  B2S_CHECK_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDev) {
    set_error("device index %d beyond the supported %d", dev, kMaxDev);
    return SP_ERR_ARG;
  }
  {
    std::lock_guard<std::mutex> lk(g_batch_mu);
    if (!g_batch_ready[dev]) {
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      B2S_CHECK_CUDA(cudaStreamIsCapturing(s, &cs), "cudaStreamIsCapturing");
      if (cs != cudaStreamCaptureStatusNone) {
        set_error("the first sp_batch_run on a device builds its tables and must not be captured");
        return SP_ERR_ARG;
      }
      B2S_CHECK_CUDA(cudaFuncSetAttribute(reinterpret_cast<const void*>(k_batch),
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(kBatchSmemBytes)),
                     "cudaFuncSetAttribute(k_batch)");
      B2S_CHECK_CUDA(cudaFuncSetAttribute(reinterpret_cast<const void*>(k_batch_big),
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(kBatchBigSmemBytes)),
                     "cudaFuncSetAttribute(k_batch_big)");
      k_batch_init<<<17, 128, 0, s>>>();
      B2S_CHECK_CUDA(cudaGetLastError(), "batch table init");
      g_batch_ready[dev] = true;
    }
  }
  const int maxg = sp_batch_max_grid();
  int sms = 0;
  const int nbig = resident_ctas(reinterpret_cast<const void*>(k_batch_big), kBatchBigThreads,
                                 kBatchBigSmemBytes, &sms);
  if (maxg <= 0 || nbig <= 0) {
    set_error("no resident CTA for the batch kernels");
    return SP_ERR_UNSUPPORTED;
  }
  if (grid <= 0 || grid > maxg) grid = maxg;
  BatchParams bp;
  bp.desc = static_cast<const unsigned char*>(desc_dev);
  bp.queue = static_cast<int*>(ws);
  // the 4096 class first (its CTAs start the dependent launch at once), then the other classes
  // as a programmatic dependent that fills SMs as the first kernel's CTAs finish
  k_batch_big<<<nbig * sms, kBatchBigThreads, kBatchBigSmemBytes, s>>>(bp);
  B2S_CHECK_CUDA(cudaGetLastError(), "batch kernel launch (4096 class)");
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(grid));
  cfg.blockDim = dim3(unsigned(kBatchThreads));
  cfg.dynamicSmemBytes = kBatchSmemBytes;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  B2S_CHECK_CUDA(cudaLaunchKernelEx(&cfg, k_batch, bp), "batch kernel launch");
  return SP_OK;
}

}
