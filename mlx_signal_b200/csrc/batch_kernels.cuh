// Persistent batched kernels: many independent spectral requests of uneven size and segment
// length in ONE batched launch (two persistent grids over one descriptor table), pulled from
// device work queues.
//
// Work model. The host encodes a descriptor table: a header, the first work item of every request
// (item_begin, an exclusive prefix over requests) and one BatchReqDev per request. A request's
// work is split into team tasks (a contiguous range of segments of one row, or of frame pairs of
// one stream chunk); TEAMS consecutive tasks of one request form a CTA work item. Each CTA takes
// the next item with an atomic on the queue head, finds its request by binary search over
// item_begin, switches to the request's FFT class (L = 256, 512, 1024, 2048 or 4096) and runs the
// same register/shared-memory team FFT as the single-request kernels. Tables (window, low-bin
// window spectrum, twiddles) are reloaded only when the class or the window changes between items.
// Two persistent kernels share the descriptor table: the 4096 class (sorted first, items
// [0, first_small)) runs one 256-thread team per CTA, 16 points per thread, the shape of the
// single-request 4096 kernel; the other classes run on 128-thread CTAs (teams of 32 or 128).
//
// Welch requests (hop = L/2, the reference's default noverlap) use the half-overlap pair loop of
// the single-request welch kernel, with the spectral form of the constant detrend (a zero
// window-spectrum table for detrend=None). Each task writes mirror-combined partial sums; the CTA
// whose task completes a row (fenced atomic row counter) reduces that row's partials in FP64 in a
// fixed order and writes the PSD, so the result of a request does not depend on what else is in
// the batch. Streaming-STFT chunks read a virtual row tail || chunk (the tail is the unconsumed
// end of the previous chunk of that stream), write complex frames, and the task holding the last
// frames writes the new tail to the other buffer of a ping-pong pair.
//
// The queue head, the completion count of CTAs and every row counter return to zero by the end of
// each launch, so the launch has fixed arguments and replays from a CUDA graph for any batch.
//
// Reference behaviour this batches: per-call welch (src/mlx_signal_processing/spectral.py:492-526
// -> _stft_metal.rfft_power_mean :530-557) and stft (spectral.py:694-738 ->
// _stft_metal.rfft_frames :192-220); the reference has no batched or streaming form.
#pragma once

#include "frame_kernels.cuh"
#include "mean_kernels.cuh"

namespace b2s {

enum : int { kBatchWelch = 0, kBatchStftStream = 1 };

// One request in device memory (144 bytes, 16-byte aligned).
struct alignas(16) BatchReqDev {
  const float* x;
  const float* win;
  const float2* wdft;  // welch constant detrend: DFT_L(win) for bins < n_low, else nullptr
  float* out;
  float* part;         // welch: partial slots [tasks][L/2+1]
  int* cnt;            // welch: per-row completion counters [rows]
  const float* tail_in;
  float* tail_out;
  int64_t ld;
  int64_t tail_ld;
  int kind, log_l, rows, nseg;  // nseg: welch segments / stft frames per row
  int G, chunks, tasks, nbins;  // G: segments (welch) or frames (stft) per task
  int n_low, onesided, tail_len, new_tail_len;
  int hop, pad0;
  float scale, pad1;
};
static_assert(sizeof(BatchReqDev) == 144, "descriptor layout");

struct alignas(16) BatchHeader {
  int magic;
  int nreq;
  int total_items;
  int first_small;  // items [0, first_small) are the 4096-point class (256-thread kernel)
};
constexpr int kBatchMagic = 0x42415443;  // "BATC"

// Descriptor blob: header | item_begin[nreq + 1] (padded to 16 B) | BatchReqDev[nreq].
__host__ __device__ inline int64_t batch_req_offset(int nreq) {
  return int64_t(sizeof(BatchHeader)) + ((int64_t(nreq + 1) * 4 + 15) & ~int64_t(15));
}
__host__ __device__ inline int64_t batch_desc_bytes(int nreq) {
  return batch_req_offset(nreq) + int64_t(nreq) * int64_t(sizeof(BatchReqDev));
}

struct BatchParams {
  const unsigned char* desc;
  int* queue;  // [0] next item, [1] CTAs finished
};

constexpr int kBatchThreads = 128;     // classes 256 ... 2048: teams of 32 or 128 threads
constexpr int kBatchBigThreads = 256;  // class 4096: one 256-thread team, 16 points per thread

// Shared-memory layout of a batched kernel (float4 units for the scratch, element counts for the
// rest): scratch | window | low-bin window spectrum (2 x LOWB complex) | twiddles (TWC complex:
// every class whose table fits; larger ones read a global table) | exchange buffers (BUFC complex,
// TEAMS x BUF of every class the kernel runs).
template <int SCR_F4, int WINF, int LOWB, int TWC, int BUFC>
struct BatchLayout {
  static constexpr int kScratchF4 = SCR_F4, kWinFloats = WINF, kLowBins = LOWB, kTwSmem = TWC,
                       kBufC = BUFC;
  static constexpr size_t kBytes = size_t(SCR_F4) * 16 + size_t(WINF) * 4 + size_t(2 * LOWB) * 8 +
                                   size_t(TWC) * 8 + size_t(BUFC) * 8;
};
// 128-thread kernel: twiddles of the classes <= 1024 in shared memory (2048 reads a global table)
using BatchSmall = BatchLayout<8, 4096, 128, 1024, 4224>;
// 256-thread kernel (Plan<12, 4>: three radix-16 passes): every table in shared memory
using BatchBig = BatchLayout<8, 4096, 256, 4352, 4352>;
constexpr size_t kBatchSmemBytes = BatchSmall::kBytes;
constexpr size_t kBatchBigSmemBytes = BatchBig::kBytes;

__device__ __forceinline__ int ldg_i(const int* p) { return __ldg(p); }

// Sample i of the virtual stream row tail[0:T] || chunk[...].
__device__ __forceinline__ float stream_sample(const float* __restrict__ tail, int T,
                                               const float* __restrict__ chunk, int64_t i) {
  return i < T ? __ldg(tail + i) : __ldg(chunk + (i - T));
}

template <class PL>
__device__ __forceinline__ void stream_load_pair(float2 (&v)[PL::E], const float* tail, int T,
                                                 const float* chunk, int64_t sa, int64_t sb,
                                                 bool two, int t) {
  if (sa >= T) {
    load_pair<PL>(v, chunk + (sa - T), chunk + (sb - T), two, t, PL::L);
  } else {
    static_for<0, PL::E>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      const int n = slot_elem<PL, e>(t);
      v[e].x = stream_sample(tail, T, chunk, sa + n);
      v[e].y = two ? stream_sample(tail, T, chunk, sb + n) : 0.f;
    });
  }
}

// Per-CTA record of the tables currently in shared memory.
struct BatchTables {
  int log_l;
  const float* win;
  const float2* wdft;
  int n_low;
};

// One CTA work item of request rq (item `local` of the request) with class (LOG_L, LOG_E) on an
// NT-thread CTA whose shared memory has layout LAY.
template <int LOG_L, int LOG_E, int NT, class LAY>
__device__ __forceinline__ void batch_item(const BatchReqDev* __restrict__ rq, int local,
                                           float4* smem, BatchTables& cur,
                                           const float2* __restrict__ tw_global, int* s_rows,
                                           int* s_nrows) {
  using CFG = MeanCfg<LOG_L, LOG_E>;
  using PL = typename CFG::PL;
  constexpr int L = PL::L, E = PL::E, P = PL::P;
  static_assert(CFG::THREADS == NT, "class and kernel CTA size differ");
  static_assert(CFG::TEAMS * CFG::SCRATCH <= LAY::kScratchF4, "scratch");
  static_assert(CFG::TEAMS * PL::BUF <= LAY::kBufC, "exchange buffers");
  static_assert(P <= LAY::kLowBins && L <= LAY::kWinFloats, "tables");
  constexpr bool kTwInSmem = PL::TW <= LAY::kTwSmem;
  float* win = reinterpret_cast<float*>(smem + LAY::kScratchF4);
  float2* wlo = reinterpret_cast<float2*>(win + LAY::kWinFloats);
  float2* whi = wlo + LAY::kLowBins;
  float2* tws = whi + LAY::kLowBins;
  float2* bufs = tws + LAY::kTwSmem;
  const int tid = threadIdx.x;

  const int kind = ldg_i(&rq->kind);
  const float* w = rq->win;
  const float2* wd = kind == kBatchWelch ? rq->wdft : nullptr;
  const int nl = kind == kBatchWelch ? ldg_i(&rq->n_low) : 0;
  bool reload = false;
  if (cur.log_l != LOG_L) {
    if constexpr (kTwInSmem) build_twiddles<PL>(tws, tid, NT);
    cur.log_l = LOG_L;
    cur.win = nullptr;
    cur.n_low = -1;
    reload = true;
  }
  if (cur.win != w) {
    for (int i = tid; i < L; i += NT) win[i] = __ldg(w + i);
    cur.win = w;
    reload = true;
  }
  if (cur.wdft != wd || cur.n_low != nl) {
    load_window_lowbins<P>(wlo, whi, wd, nl, tid, NT);
    cur.wdft = wd;
    cur.n_low = nl;
    reload = true;
  }
  if (reload) __syncthreads();  // uniform: every thread tracks the same table state

  const int team = tid / P;
  HalfCtx<PL> c;
  c.win = win;
  c.wlo = wlo;
  c.whi = whi;
  c.tw = kTwInSmem ? tws : tw_global;
  c.buf = bufs + team * PL::BUF;
  c.scratch = smem + team * CFG::SCRATCH;
  c.t = tid - team * P;
  c.mask = team_mask<P>();
  const int t = c.t;

  const int tasks = ldg_i(&rq->tasks), chunks = ldg_i(&rq->chunks), G = ldg_i(&rq->G);
  const int nseg = ldg_i(&rq->nseg);
  const int64_t ld = rq->ld;
  const int task0 = local * CFG::TEAMS;
  const int task = task0 + team;

  if (kind == kBatchWelch) {
    if (task < tasks) {
      const int row = task / chunks, ch = task - row * chunks;
      const int s0 = ch * G;
      const int s1 = min(s0 + G, nseg);
      float acc[E];
#pragma unroll
      for (int e = 0; e < E; ++e) acc[e] = 0.f;
      welch_half_range<PL, kDetrendConstantSpectral, false, false>(c, rq->x + int64_t(row) * ld,
                                                                   s0, s1, acc);
      flush_mirror<PL>(acc, rq->part + int64_t(task) * welch_slot_floats(L), c.buf, t, c.mask);
    }
    // Publish this item's partials, then count them against their rows.
    __threadfence();
    __syncthreads();
    if (tid == 0) {
      int n = 0;
      const int tend = min(task0 + CFG::TEAMS, tasks);
      int k = task0;
      while (k < tend) {
        const int row = k / chunks;
        const int rend = min(tend, (row + 1) * chunks);
        const int add = rend - k;
        int* cp = rq->cnt + row;
        if (atomicAdd(cp, add) + add == chunks) {
          *cp = 0;  // every task of the row has arrived: reset for the next launch
          s_rows[n++] = row;
        }
        k = rend;
      }
      *s_nrows = n;
      __threadfence();
    }
    __syncthreads();
    const int nrows = *s_nrows;
    if (nrows > 0) {
      const int nbins = ldg_i(&rq->nbins);
      const int onesided = ldg_i(&rq->onesided);
      const double scale = double(__ldg(&rq->scale)) / double(nseg);
      constexpr int SLOT = welch_slot_floats(L);
      for (int i = 0; i < nrows; ++i) {
        const int row = s_rows[i];
        const float* q = rq->part + int64_t(row) * chunks * SLOT;
        float* o = rq->out + int64_t(row) * nbins;
        for (int k = tid; k < nbins; k += NT) {
          const int kc = k <= L / 2 ? k : L - k;
          const float* qk = q + kc;
          // eight independent FP64 sums keep eight L2 loads in flight per thread (this reduce
          // of the last row to complete sits in the launch's tail); fixed order throughout
          double a[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
          int cc = 0;
          for (; cc + 7 < chunks; cc += 8) {
            float v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = __ldcg(qk + int64_t(cc + j) * SLOT);
#pragma unroll
            for (int j = 0; j < 8; ++j) a[j] += double(v[j]);
          }
          for (int j = 0; cc < chunks; ++cc, ++j) a[j] += double(__ldcg(qk + int64_t(cc) * SLOT));
          double fac = 0.5 * scale;
          if (onesided && k != 0 && 2 * k != L) fac *= 2.0;
          o[k] = float((((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]))) * fac);
        }
      }
    }
    return;
  }

  // Streaming STFT chunk: frames of tail || chunk, two frames per complex FFT.
  if (task < tasks) {
    const int row = task / chunks, ch = task - row * chunks;
    const int f0 = ch * G;
    const int f1 = min(f0 + G, nseg);
    const int hop = ldg_i(&rq->hop);
    const int T = ldg_i(&rq->tail_len);
    const int64_t tld = rq->tail_ld;
    const float* tail = rq->tail_in + int64_t(row) * tld;
    const float* xr = rq->x + int64_t(row) * ld;
    const float scale = __ldg(&rq->scale);
    constexpr int NB = L / 2 + 1;
    float2* orow = reinterpret_cast<float2*>(rq->out) + int64_t(row) * nseg * NB;
    for (int s = f0; s < f1; s += 2) {
      const bool two = s + 1 < f1;
      const int64_t sa = int64_t(s) * hop;
      float2 v[E];
      stream_load_pair<PL>(v, tail, T, xr, sa, sa + hop, two, t);
      static_for<0, E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        const float wv = win[slot_elem<PL, e>(t)];
        v[e] = make_float2(v[e].x * wv, v[e].y * wv);
      });
      team_pass0<PL>(v);
      team_passes<PL>(v, c.buf, c.tw, t, c.mask);
      // mirrors of the one-sided bins k <= L/2: registers e >= E/2, and bin 0 itself
#pragma unroll
      for (int e = E / 2; e < E; ++e) c.buf[PL::pad(t + e * P)] = v[e];
      if (t == 0) c.buf[0] = v[0];
      team_sync<P>(c.mask);
      float2* oa = orow + int64_t(s) * NB;
#pragma unroll
      for (int e = 0; e <= E / 2; ++e) {
        const int k = t + e * P;
        if (k < NB) {
          const float2 z = v[e];
          const float2 m = c.buf[PL::pad((L - k) & (L - 1))];
          const float hs = 0.5f * scale;
          oa[k] = make_float2(hs * (z.x + m.x), hs * (z.y - m.y));
          if (two) oa[NB + k] = make_float2(hs * (z.y + m.y), hs * (m.x - z.x));
        }
      }
      team_sync<P>(c.mask);
    }
    if (ch == chunks - 1) {
      const int nt = ldg_i(&rq->new_tail_len);
      const int64_t start = int64_t(nseg) * hop;
      float* to = rq->tail_out + int64_t(row) * tld;
      for (int i = t; i < nt; i += P) to[i] = stream_sample(tail, T, xr, start + i);
    }
  }
}

}  // namespace b2s
