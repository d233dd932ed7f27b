"""Continuous-batching request loop for spectral analysis on one GPU.

`SpectralServer` admits welch requests and streaming-STFT chunks as they arrive, under a fixed
HBM budget, and runs each admitted group as ONE persistent batched launch (`sp_batch_run`). The
launcher has several slots (CUDA stream + workspace + descriptor buffers each), so requests that
arrive while a batch is on the GPU are admitted as soon as a slot and memory free up, and their
launch overlaps the tail of the previous one on the device. Streaming state -- the unconsumed
tail of every stream -- stays resident in one device tensor; at most one chunk of a stream is in
flight at a time, since the next chunk reads the tail that chunk writes.

The loop is single-threaded and non-blocking: `step()` retires completed batches (event
queries), moves pending requests into a new batch while a slot is free, and launches it;
`submit_*` only appends to the pending queue. Latency of a request = the host time at which its
batch was seen complete minus its arrival (submit) time.

`run_per_request` drives the plain per-request path (one `welch` call per request; for stream
chunks, concatenate tail and chunk, one `stft` call, keep the new tail) with the same arrival
schedule: the baseline the batched loop is measured against.

The reference has no request loop; each request there is one welch (spectral.py:492-526) or
stft (spectral.py:694-738) call.
"""

from __future__ import annotations

import collections
import gc
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import batch as _b
from ._array import device
from .autotune import default_cache

__all__ = ["ServerStats", "SpectralServer", "poisson_schedule", "run_per_request", "run_schedule"]

KIND_WELCH, KIND_STREAM = _b.KIND_WELCH, _b.KIND_STREAM


@dataclass
class _Pending:
    rid: int
    kind: int
    x: torch.Tensor            # welch: (rows, n); stream: (m,) chunk of a 1-row stream
    arrival: float
    nperseg: int
    stream: int = -1
    detrend: int = 1
    scale: float = 1.0
    onesided: int = 1
    nbytes: int = 0
    ld: int = 0


@dataclass
class ServerStats:
    latencies: list = field(default_factory=list)   # seconds, per completed request
    completed: int = 0
    batches: int = 0
    batch_sizes: list = field(default_factory=list)
    first_arrival: float | None = None
    last_done: float | None = None
    peak_bytes: int = 0

    def summary(self) -> dict:
        lat = np.asarray(self.latencies) * 1e3
        span = (self.last_done - self.first_arrival) if self.completed else 0.0
        return {
            "completed": self.completed,
            "req_per_s": self.completed / span if span > 0 else 0.0,
            "p50_ms": float(np.percentile(lat, 50)) if lat.size else None,
            "p99_ms": float(np.percentile(lat, 99)) if lat.size else None,
            "mean_batch": float(np.mean(self.batch_sizes)) if self.batch_sizes else 0.0,
            "batches": self.batches,
            "peak_inflight_bytes": self.peak_bytes,
        }


class SpectralServer:
    """Continuous batching of welch requests and streaming-STFT chunks (see module doc).

    hbm_budget: device bytes that in-flight requests may hold (input + output + partial sums);
    a request larger than the whole budget is rejected at submit. max_batch: requests per
    launch. slots: launches that may be in flight at once.
    """

    def __init__(self, hbm_budget: int = 2 << 30, max_batch: int = 1024, slots: int = 3,
                 use_graph: bool = True, window="hann", fs: float = 1.0,
                 stream_nperseg: int = 1024, stream_noverlap: int = 768, max_streams: int = 256,
                 keep_results: bool = False):
        self.dev = device()
        self.budget = int(hbm_budget)
        self.max_batch = int(max_batch)
        self.window = window
        self.fs = float(fs)
        ws = max(1 << 20, self.budget)
        self.launcher = _b.BatchLauncher(max_requests=max_batch, ws_bytes=ws, slots=slots,
                                         use_graph=use_graph)
        # streams: one row each; tails[s, parity, :] on the device
        self.sN = int(stream_nperseg)
        self.shop = self.sN - int(stream_noverlap)
        self.s_tables = _b._tables(window, self.sN)
        self.s_scale = 1.0 / self.s_tables.sum_w
        self.max_streams = int(max_streams)
        self.tails = torch.zeros((self.max_streams, 2, self.sN), dtype=torch.float32,
                                 device=self.dev)
        self.tail_len = np.zeros(self.max_streams, np.int64)
        self.parity = np.zeros(self.max_streams, np.int64)
        self.frames_emitted = np.zeros(self.max_streams, np.int64)
        self.busy = np.zeros(self.max_streams, bool)
        self.pending: collections.deque[_Pending] = collections.deque()
        # stream chunks that wait behind an earlier chunk of their stream (in flight, chosen for
        # the batch being built, or itself waiting), per stream in arrival order; streams in the
        # order their first waiting chunk arrived
        self.held: dict[int, collections.deque[_Pending]] = {}
        self.inflight: collections.deque = collections.deque()
        self.used = 0
        self.next_rid = 0
        self.keep_results = keep_results
        self.results: dict[int, object] = {}
        self.stats = ServerStats()
        self._tables: dict[int, _b._Tables] = {}

    # ----------------------------------------------------------------------------- submit
    def _welch_tables(self, N: int):
        t = self._tables.get(N)
        if t is None:
            t = _b._tables(self.window, N)
            self._tables[N] = t
        return t

    def submit_welch(self, x: torch.Tensor, nperseg: int = 256, detrend="constant",
                     scaling="density", return_onesided: bool = True,
                     arrival: float | None = None) -> int:
        """Queue welch(x, fs, window, nperseg, noverlap=nperseg//2, detrend, scaling) for a
        (rows, n) float32 CUDA tensor. Returns the request id."""
        if nperseg not in _b.BATCH_NPERSEG or x.shape[-1] < nperseg:
            raise ValueError(f"batched welch needs nperseg in {_b.BATCH_NPERSEG} and n >= nperseg")
        if x.dtype != torch.float32 or not x.is_cuda or x.dim() != 2 or x.stride(-1) != 1:
            raise ValueError("server welch input: (rows, n) float32 CUDA tensor, unit inner stride")
        tb = self._welch_tables(nperseg)
        code = 1 if detrend in ("constant", "c") else 0 if detrend in (False, None) else -1
        if code < 0:
            raise ValueError("server welch: detrend must be 'constant' or False")
        scale = (1.0 / (self.fs * tb.sum_w2)) if scaling == "density" else 1.0 / tb.sum_w ** 2
        rows, n = x.shape
        G = default_cache().get("welch", nperseg, rows)
        nseg = (n - nperseg) // (nperseg // 2) + 1
        chunks = -(-nseg // max(2, G + (G & 1)))
        nb = nperseg // 2 + 1 if return_onesided else nperseg
        nbytes = rows * n * 4 + rows * nb * 4 + rows * chunks * (nperseg // 2 + 1) * 4
        if nbytes > self.budget:
            raise ValueError(f"request needs {nbytes} device bytes, above the HBM budget")
        rid = self.next_rid
        self.next_rid += 1
        t = time.perf_counter() if arrival is None else arrival
        ld = x.stride(0) if rows > 1 else n
        self.pending.append(_Pending(rid, KIND_WELCH, x, t, nperseg, -1, code, scale,
                                     int(bool(return_onesided)), nbytes, int(ld)))
        return rid

    def submit_chunk(self, stream: int, chunk: torch.Tensor, arrival: float | None = None) -> int:
        """Queue the next chunk ((m,) float32 CUDA) of stream `stream` (0 <= stream <
        max_streams). Chunks of one stream are processed in submission order."""
        if not 0 <= stream < self.max_streams:
            raise ValueError("stream id out of range")
        if (chunk.dtype != torch.float32 or not chunk.is_cuda or chunk.dim() != 1
                or (chunk.shape[0] > 1 and chunk.stride(0) != 1)):
            raise ValueError("server stream chunk: (m,) float32 CUDA tensor")
        m = chunk.shape[0]
        nbytes = m * 4 + ((m + self.sN) // self.shop + 1) * (self.sN // 2 + 1) * 8
        rid = self.next_rid
        self.next_rid += 1
        t = time.perf_counter() if arrival is None else arrival
        self.pending.append(_Pending(rid, KIND_STREAM, chunk, t, self.sN, stream, 0,
                                     self.s_scale, 1, nbytes, m))
        return rid

    # ----------------------------------------------------------------------------- loop
    def _retire(self, now: float) -> None:
        while self.inflight and self.inflight[0][0].query():
            ev, reqs, nbytes, outs = self.inflight.popleft()
            self.used -= nbytes
            for r, o in zip(reqs, outs):
                self.stats.latencies.append(now - r.arrival)
                if r.kind == KIND_STREAM:
                    self.busy[r.stream] = False
                if self.keep_results:
                    self.results[r.rid] = o
            self.stats.completed += len(reqs)
            self.stats.last_done = now

    def queued(self) -> bool:
        """True while some submitted request has not been launched."""
        return bool(self.pending) or bool(self.held)

    def _select(self) -> list[_Pending]:
        """FIFO admission while the batch and the budget have room. Waiting chunks of streams
        that are free again go first (they arrived before anything still pending); a chunk of a
        stream with a chunk in flight, in this batch or already waiting moves once to that
        stream's held queue, so one selection costs O(streams + batch), not a rescan of the
        backlog."""
        chosen = []
        room = self.budget - self.used
        taken = set()
        for s in list(self.held):
            if len(chosen) >= self.max_batch:
                return chosen
            if self.busy[s]:
                continue
            q = self.held[s]
            r = q[0]
            if r.nbytes > room:
                return chosen
            q.popleft()
            if not q:
                del self.held[s]
            chosen.append(r)
            room -= r.nbytes
            taken.add(s)
        while self.pending and len(chosen) < self.max_batch:
            r = self.pending[0]
            if r.kind == KIND_STREAM and (self.busy[r.stream] or r.stream in taken
                                          or r.stream in self.held):
                self.pending.popleft()
                q = self.held.get(r.stream)
                if q is None:
                    q = self.held[r.stream] = collections.deque()
                q.append(r)
                continue
            if r.nbytes > room:
                break
            self.pending.popleft()
            chosen.append(r)
            room -= r.nbytes
            if r.kind == KIND_STREAM:
                taken.add(r.stream)
        return chosen

    def _launch(self, reqs: list[_Pending]) -> None:
        k = len(reqs)
        a = np.zeros(k, dtype=_b.REQ_DTYPE)
        kinds = np.fromiter((r.kind for r in reqs), np.int32, k)
        isw = kinds == KIND_WELCH
        iss = ~isw
        a["kind"] = kinds
        a["nperseg"] = np.fromiter((r.nperseg for r in reqs), np.int32, k)
        a["onesided"] = np.fromiter((r.onesided for r in reqs), np.int32, k)
        a["x"] = np.fromiter((r.x.data_ptr() for r in reqs), np.uint64, k)
        ns = np.fromiter((r.x.shape[-1] for r in reqs), np.int64, k)
        rows = np.fromiter((r.x.shape[0] if r.kind == KIND_WELCH else 1 for r in reqs),
                           np.int64, k)
        a["n"] = ns
        a["ld"] = np.fromiter((r.ld for r in reqs), np.int64, k)
        a["rows"] = rows
        a["scale"] = np.fromiter((r.scale for r in reqs), np.float32, k)
        # welch columns
        N = a["nperseg"].astype(np.int64)
        a["hop"] = np.where(isw, N // 2, self.shop)
        det = np.fromiter((r.detrend for r in reqs), np.int32, k)
        a["detrend"] = np.where(isw, det, 0)
        tabs = [self._welch_tables(int(n)) if w else None for n, w in zip(N, isw)]
        a["win"] = np.fromiter((t.win.data_ptr() if t is not None else
                                self.s_tables.win.data_ptr() for t in tabs), np.uint64, k)
        a["win_dft_low"] = np.fromiter((t.wdft.data_ptr() if (t is not None and d == 1) else 0
                                        for t, d in zip(tabs, det)), np.uint64, k)
        a["n_low"] = np.fromiter((t.n_low if (t is not None and d == 1) else 0
                                  for t, d in zip(tabs, det)), np.int32, k)
        a["seg_per_task"] = np.fromiter(
            (default_cache().get("welch" if w else "stft_stream", int(n), int(rw))
             for w, n, rw in zip(isw, N, rows)), np.int32, k)
        # stream columns: frames and tails from the host state
        sid = np.fromiter((r.stream for r in reqs), np.int64, k)
        s_idx = np.where(iss)[0]
        ssid = sid[s_idx]
        tl = self.tail_len[ssid]
        m = tl + ns[s_idx]
        f = np.where(m >= self.sN, (m - self.sN) // self.shop + 1, 0)
        par = self.parity[ssid]
        base = self.tails.data_ptr()
        stride_s = 2 * self.sN * 4
        a["tail_len"][s_idx] = tl
        a["tail_ld"][s_idx] = self.sN
        a["tail_in"][s_idx] = base + ssid * stride_s + par * self.sN * 4
        a["tail_out"][s_idx] = base + ssid * stride_s + (1 - par) * self.sN * 4
        # outputs: one flat buffer per batch, 8-byte aligned slices
        nb = np.where(isw, np.where(a["onesided"] == 1, N // 2 + 1, N), self.sN // 2 + 1)
        out_f = np.zeros(k, np.int64)
        out_f[isw] = rows[isw] * nb[isw]
        out_f[s_idx] = 2 * f * (self.sN // 2 + 1)
        out_f += out_f & 1
        offs = np.concatenate([[0], np.cumsum(out_f)[:-1]])
        out = torch.empty(int(out_f.sum()) + 2, dtype=torch.float32, device=self.dev)
        a["out"] = out.data_ptr() + offs * 4
        ev = self.launcher.launch(a, keep=(reqs, out))
        # stream state advances at encode time (the next chunk of a stream waits for `busy`)
        self.tail_len[ssid] = m - f * self.shop
        self.parity[ssid] ^= 1
        first = self.frames_emitted[ssid].copy()
        self.frames_emitted[ssid] += f
        self.busy[ssid] = True
        outs = []
        fi = dict(zip(s_idx.tolist(), zip(f.tolist(), first.tolist())))
        for i, r in enumerate(reqs):
            o = int(offs[i])
            if r.kind == KIND_WELCH:
                outs.append(("welch", out, o, int(rows[i]), int(nb[i])))
            else:
                nf, f0 = fi[i]
                outs.append(("stream", out, o, nf, f0))
        nbytes = sum(r.nbytes for r in reqs)
        self.used += nbytes
        self.stats.peak_bytes = max(self.stats.peak_bytes, self.used)
        self.inflight.append((ev, reqs, nbytes, outs))
        self.stats.batches += 1
        self.stats.batch_sizes.append(k)

    def step(self) -> int:
        """Retire finished batches, then launch one batch if a slot is free. Returns the number
        of requests launched."""
        now = time.perf_counter()
        self._retire(now)
        if not self.queued() or len(self.inflight) >= len(self.launcher.slots):
            return 0
        reqs = self._select()
        if not reqs:
            return 0
        if self.stats.first_arrival is None:
            self.stats.first_arrival = min(r.arrival for r in reqs)
        self._launch(reqs)
        return len(reqs)

    def drain(self) -> None:
        """Run the loop until every submitted request has completed."""
        while self.queued() or self.inflight:
            if self.step() == 0 and self.inflight:
                self.inflight[0][0].synchronize()
        self._retire(time.perf_counter())

    # ----------------------------------------------------------------------------- results
    def result(self, rid: int):
        """Welch: (rows, nbins) float32 PSD. Stream chunk: (first_frame, frames) with frames the
        (nfreq, nframes) complex64 scipy.signal.stft layout of this chunk's frames. Needs
        keep_results=True and the request completed."""
        tag, out, o, a, b = self.results[rid]
        if tag == "welch":
            return out[o : o + a * b].view(a, b)
        nb = self.sN // 2 + 1
        z = out[o : o + 2 * a * nb].view(torch.complex64).view(a, nb)
        return b, z.transpose(0, 1)


def poisson_schedule(rate: float, duration: float, pool: torch.Tensor, seed: int = 0,
                     n_streams: int = 256, stream_frac: float = 0.7,
                     chunk=(4096, 65536), welch_rows=(1, 16), welch_log2n=(14, 20),
                     welch_nperseg=(256, 1024)):
    """Seeded synthetic load: Poisson arrivals at `rate` per second for `duration` seconds;
    a `stream_frac` share are streaming-STFT chunks (stream uniform over n_streams, length
    uniform in `chunk`), the rest welch requests (rows uniform in welch_rows, length
    2^U(welch_log2n), nperseg uniform over welch_nperseg, 50% overlap). Payloads are views into
    the device tensor `pool` (float32, 1-D) at seeded offsets, so inputs are resident in HBM.
    Returns a list of (arrival_s, kind, payload, params) in arrival order."""
    rs = np.random.default_rng(seed)
    t = np.cumsum(rs.exponential(1.0 / rate, size=int(rate * duration * 1.2) + 16))
    t = t[t < duration]
    P = pool.shape[0]
    sched = []
    for ti in t:
        if rs.random() < stream_frac:
            m = int(rs.integers(chunk[0], chunk[1] + 1))
            off = int(rs.integers(0, P - m))
            sched.append((float(ti), KIND_STREAM, pool[off : off + m],
                          {"stream": int(rs.integers(0, n_streams))}))
        else:
            rows = int(rs.integers(welch_rows[0], welch_rows[1] + 1))
            n = int(2 ** rs.uniform(welch_log2n[0], welch_log2n[1]))
            N = int(rs.choice(welch_nperseg))
            off = int(rs.integers(0, P - rows * n))
            sched.append((float(ti), KIND_WELCH, pool[off : off + rows * n].view(rows, n),
                          {"nperseg": N}))
    return sched


class _CollectorPaused:
    """Pause Python's cyclic garbage collector for a request loop. A full collection walks every
    tracked object (request tuples, tensor views, per-request records): with tens of thousands
    of requests queued it stalls the loop for tens to hundreds of milliseconds, which shows up
    as p99 latency. Reference counting still frees everything; the collector is re-enabled (and
    run once) when the loop ends."""

    def __enter__(self):
        self.was = gc.isenabled()
        gc.collect()
        gc.disable()
        return self

    def __exit__(self, *exc):
        if self.was:
            gc.enable()
        return False


def run_schedule(server: SpectralServer, schedule) -> ServerStats:
    """Drive `server` with an open-loop arrival schedule (arrival times relative to the start):
    each request is submitted when its time comes, and the loop keeps stepping until all have
    completed. Latencies count from the scheduled arrival. The loop runs with the cyclic
    garbage collector paused (_CollectorPaused)."""
    with _CollectorPaused():
        t0 = time.perf_counter()
        i = 0
        n = len(schedule)
        while i < n or server.queued() or server.inflight:
            now = time.perf_counter()
            while i < n and t0 + schedule[i][0] <= now:
                arr, kind, x, p = schedule[i]
                if kind == KIND_WELCH:
                    server.submit_welch(x, nperseg=p["nperseg"], arrival=t0 + arr)
                else:
                    server.submit_chunk(p["stream"], x, arrival=t0 + arr)
                i += 1
            server.step()
    return server.stats


def run_per_request(schedule, fs: float = 1.0, window="hann", stream_nperseg: int = 1024,
                    stream_noverlap: int = 768, max_streams: int = 256):
    """The plain per-request path on an arrival schedule: (arrival, kind, payload, params) in
    arrival order, processed FIFO on the current stream as soon as each arrives; completion is
    observed through one CUDA event per request. Runs with the garbage collector paused, as
    run_schedule does. Returns ServerStats."""
    with _CollectorPaused():
        return _run_per_request(schedule, fs, window, stream_nperseg, stream_noverlap)


def _run_per_request(schedule, fs, window, stream_nperseg, stream_noverlap):
    from .spectral import stft, welch

    stats = ServerStats()
    tails: dict[int, torch.Tensor] = {}
    inflight: collections.deque = collections.deque()
    hop = stream_nperseg - stream_noverlap
    t0 = time.perf_counter()
    i = 0
    nreq = len(schedule)
    while i < nreq or inflight:
        now = time.perf_counter() - t0
        while inflight and inflight[0][0].query():
            ev, arr = inflight.popleft()
            done = time.perf_counter() - t0
            stats.latencies.append(done - arr)
            stats.completed += 1
            stats.last_done = done
        if i < nreq and schedule[i][0] <= now:
            arr, kind, x, p = schedule[i]
            i += 1
            if stats.first_arrival is None:
                stats.first_arrival = arr
            if kind == KIND_WELCH:
                welch(x, fs=fs, window=window, nperseg=p["nperseg"], detrend=p.get("detrend",
                      "constant"))
            else:
                s = p["stream"]
                u = torch.cat([tails[s], x]) if s in tails else x
                if u.shape[0] >= stream_nperseg:
                    stft(u, fs=fs, window=window, nperseg=stream_nperseg,
                         noverlap=stream_noverlap, boundary=None, padded=False)
                    f = (u.shape[0] - stream_nperseg) // hop + 1
                    tails[s] = u[f * hop:]
                else:
                    tails[s] = u
            ev = torch.cuda.Event()
            ev.record()
            inflight.append((ev, arr))
    return stats
