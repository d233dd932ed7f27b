"""Batched spectral requests: many welch calls and streaming-STFT chunks in ONE batched launch
(`sp_batch_run`: a persistent kernel for the 4096-point class, then one for the other classes as
its programmatic dependent) over a device work queue (C-ABI sp_batch_*, include/b200signal.h).

* `prepare_welch(x, **welch_kwargs)` validates one welch call exactly as `welch` does and, when
  it fits the batched kernel (real input, nperseg == nfft in {256, 512, 1024, 2048, 4096}, 50% overlap,
  detrend False or 'constant', mean averaging), returns a `WelchJob` whose `result()` is what
  `welch` would return; otherwise None.
* `StftStream` keeps a stream's overlap tail resident on the device (two ping-pong buffers per
  stream) and turns each new chunk into a `StreamJob` whose frames continue the stream: the
  concatenation of all chunk outputs equals scipy.signal.stft of the concatenated stream with
  boundary=None, padded=False.
* `BatchLauncher` owns the device workspace and descriptor slots (pinned host + device copy per
  slot, one CUDA stream per slot) and launches a list of jobs as one batched launch, replayed
  from a captured CUDA graph after the first launch of a slot.
* `welch_batch(signals, **kw)` is the one-shot form: one launch for the eligible requests, the
  regular `welch` for the rest.

The reference has no batched form; each request there is one welch (spectral.py:492-526) or
stft (spectral.py:694-738) call.
"""

from __future__ import annotations

import ctypes
import math
import threading
from dataclasses import dataclass

import numpy as np
import torch

from . import _kernels, _lib
from ._array import current_index, device, stream_handle, to_device
from .autotune import default_cache
from .windows import _window_np

__all__ = [
    "BATCH_NPERSEG",
    "BatchLauncher",
    "BatchRequest",
    "REQ_DTYPE",
    "StftStream",
    "StreamJob",
    "WelchJob",
    "plan",
    "prepare_welch",
    "welch_batch",
]

BATCH_NPERSEG = (256, 512, 1024, 2048, 4096)
KIND_WELCH, KIND_STREAM = 0, 1


class BatchRequest(ctypes.Structure):
    """ctypes mirror of sp_batch_request (include/b200signal.h)."""

    _fields_ = [
        ("kind", ctypes.c_int),
        ("nperseg", ctypes.c_int),
        ("hop", ctypes.c_int),
        ("detrend", ctypes.c_int),
        ("onesided", ctypes.c_int),
        ("n_low", ctypes.c_int),
        ("seg_per_task", ctypes.c_int),
        ("tail_len", ctypes.c_int),
        ("rows", ctypes.c_int64),
        ("n", ctypes.c_int64),
        ("ld", ctypes.c_int64),
        ("tail_ld", ctypes.c_int64),
        ("x", ctypes.c_void_p),
        ("win", ctypes.c_void_p),
        ("win_dft_low", ctypes.c_void_p),
        ("tail_in", ctypes.c_void_p),
        ("tail_out", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
        ("scale", ctypes.c_float),
    ]


#: numpy structured mirror of sp_batch_request (same field offsets, 120-byte records), for
#: building a batch's request array column-wise
REQ_DTYPE = np.dtype({
    "names": [f for f, _ in BatchRequest._fields_],
    "formats": ["<i4"] * 8 + ["<i8"] * 4 + ["<u8"] * 6 + ["<f4"],
    "offsets": [getattr(BatchRequest, f).offset for f, _ in BatchRequest._fields_],
    "itemsize": ctypes.sizeof(BatchRequest),
})


# ---------------------------------------------------------------------------------------------
# per-(window, nperseg) device tables
# ---------------------------------------------------------------------------------------------


@dataclass(frozen=True)
class _Tables:
    win: torch.Tensor          # float32 window values (no scale folded in)
    wdft: torch.Tensor | None  # complex64 DFT(win)[0..n_low) for the spectral constant detrend
    n_low: int
    sum_w: float
    sum_w2: float


_TABLES: dict = {}
_TABLES_LOCK = threading.Lock()


def _window_key(window):
    if isinstance(window, str):
        return window
    if isinstance(window, tuple):
        return window
    if isinstance(window, list):
        return tuple(window)
    return None


def _tables(window, nperseg: int) -> _Tables | None:
    """Device window tables for a named window (None for array windows: not batched)."""
    key = _window_key(window)
    if key is None:
        return None
    dev = current_index()
    k = (key, int(nperseg), dev)
    hit = _TABLES.get(k)
    if hit is not None:
        return hit
    with _TABLES_LOCK:
        hit = _TABLES.get(k)
        if hit is None:
            w64 = _window_np(key, int(nperseg))
            w32 = w64.astype(np.float32)
            low = _kernels.window_low_spectrum(w32, int(nperseg))
            wdft = None
            n_low = 0
            if low is not None:
                wdft = torch.from_numpy(np.ascontiguousarray(low[0])).to(device())
                n_low = int(low[1])
            hit = _Tables(torch.from_numpy(w32).to(device()), wdft, n_low,
                          float(w64.sum()), float((w64 * w64).sum()))
            _TABLES[k] = hit
    return hit


def _batch_team(nperseg: int) -> int:
    """Threads per FFT team of the batched kernels' class (32 points per thread at 1024, 16 at
    256, 512, 2048 and 4096): the low window-spectrum bins its constant-detrend correction can
    apply."""
    return nperseg // (32 if nperseg == 1024 else 16)


def _rows_view(X: torch.Tensor) -> tuple[torch.Tensor, int]:
    rows = math.prod(X.shape[:-1]) if X.dim() > 1 else 1
    n = X.shape[-1]
    x2 = X.reshape(rows, n)
    if x2.stride(-1) != 1 or (rows > 1 and x2.stride(0) < n):
        x2 = x2.contiguous()
    ld = x2.stride(0) if rows > 1 else n
    return x2, int(ld)


# ---------------------------------------------------------------------------------------------
# welch requests
# ---------------------------------------------------------------------------------------------


@dataclass
class WelchJob:
    """A validated welch request bound to its output buffer."""

    req: BatchRequest
    out: torch.Tensor         # (rows, nbins) float32
    x: torch.Tensor           # keeps the input alive until the launch completes
    outer: tuple
    axis: int
    nfft: int
    fs: float
    onesided: bool
    nbytes: int               # device bytes this request holds (input view + output + partials)

    def result(self):
        """(freqs, Pxx) exactly as `welch` returns them."""
        f = np.fft.rfftfreq(self.nfft, 1 / self.fs) if self.onesided else np.fft.fftfreq(
            self.nfft, 1 / self.fs)
        freqs = torch.from_numpy(f.astype(np.float32)).to(self.out.device)
        pxx = self.out.reshape(self.outer + (self.out.shape[-1],))
        if pxx.dim() > 1 and self.axis != -1:
            pxx = pxx.movedim(-1, self.axis if self.axis >= 0 else pxx.dim() + self.axis)
        return freqs, pxx


def prepare_welch(x, fs=1.0, window="hann", nperseg=None, noverlap=None, nfft=None,
                  detrend="constant", return_onesided=True, scaling="density", axis=-1,
                  average="mean", *, seg_per_task: int | None = None) -> WelchJob | None:
    """Validate one welch call for the batched kernel; None when the request needs the regular
    path (the caller then uses `welch`). Argument meaning and defaults follow `welch`."""
    if average != "mean":
        return None
    X = to_device(x)
    if X.is_complex() or X.numel() == 0:
        return None
    axis = int(axis)
    if X.dim() > 1 and axis not in (-1, X.dim() - 1):
        X = X.movedim(axis, -1)
    n = X.shape[-1]
    if not isinstance(window, str | tuple | list):
        return None
    nper = 256 if nperseg is None else int(nperseg)
    if nper not in BATCH_NPERSEG or nper > n:
        return None
    if nfft is not None and int(nfft) != nper:
        return None
    if noverlap is not None and int(noverlap) != nper // 2:
        return None
    if detrend in (False, None):
        code = 0
    elif detrend in ("constant", "c"):
        code = 1
    else:
        return None
    tb = _tables(window, nper)
    if tb is None or (code == 1 and (tb.wdft is None or tb.n_low > _batch_team(nper))):
        return None
    if scaling == "density":
        scale = 1.0 / (float(fs) * tb.sum_w2)
    elif scaling == "spectrum":
        scale = 1.0 / tb.sum_w ** 2
    else:
        raise ValueError(f"Unknown scaling: {scaling!r}")
    onesided = bool(return_onesided)
    x2, ld = _rows_view(X)
    rows = x2.shape[0]
    nbins = nper // 2 + 1 if onesided else nper
    out = torch.empty((rows, nbins), dtype=torch.float32, device=x2.device)
    G = seg_per_task if seg_per_task else default_cache().get("welch", nper, rows)
    r = BatchRequest()
    r.kind = KIND_WELCH
    r.nperseg = nper
    r.hop = nper // 2
    r.detrend = code
    r.onesided = int(onesided)
    r.n_low = tb.n_low if code == 1 else 0
    r.seg_per_task = int(G)
    r.rows = rows
    r.n = n
    r.ld = ld
    r.x = x2.data_ptr()
    r.win = tb.win.data_ptr()
    r.win_dft_low = tb.wdft.data_ptr() if code == 1 else None
    r.out = out.data_ptr()
    r.scale = scale
    nseg = (n - nper) // (nper // 2) + 1
    chunks = -(-nseg // max(2, G + (G & 1)))
    nbytes = rows * n * 4 + out.numel() * 4 + rows * chunks * (nper // 2 + 1) * 4 + rows * 4
    return WelchJob(r, out, x2, tuple(X.shape[:-1]), axis, nper, float(fs), onesided, nbytes)


# ---------------------------------------------------------------------------------------------
# streaming STFT
# ---------------------------------------------------------------------------------------------


@dataclass
class StreamJob:
    """One chunk of a stream bound to its output: frames (rows, nframes, nperseg//2+1) c64."""

    req: BatchRequest
    out: torch.Tensor
    x: torch.Tensor
    stream: StftStream
    first_frame: int
    nframes: int
    nbytes: int

    def result(self):
        """(t, Zxx) of this chunk's frames: t in seconds from the stream start (frame centres),
        Zxx (rows, nfreq, nframes) like scipy.signal.stft's output for these frames."""
        s = self.stream
        idx = np.arange(self.first_frame, self.first_frame + self.nframes)
        t = (idx * s.hop + s.nperseg / 2) / s.fs
        tt = torch.from_numpy(t.astype(np.float32)).to(self.out.device)
        return tt, self.out.movedim(-1, -2)


class StftStream:
    """Streaming STFT state resident on the device: the unconsumed tail of the stream (fewer
    than nperseg samples per row) in one of two ping-pong buffers, plus host counters.

    Frames follow scipy.signal.stft(x, fs, window, nperseg, noverlap, boundary=None,
    padded=False, detrend=False, scaling='spectrum') of the concatenated stream. Chunks must be
    submitted in order and at most one chunk of a stream may be in one batch; `busy` marks a
    stream whose latest chunk is encoded but not yet known complete, and `event` is the CUDA
    event after which its tail is valid.
    """

    def __init__(self, rows: int = 1, fs: float = 1.0, window="hann", nperseg: int = 1024,
                 noverlap: int | None = None, *, seg_per_task: int | None = None):
        if nperseg not in BATCH_NPERSEG:
            raise ValueError(f"nperseg must be one of {BATCH_NPERSEG} for a batched stream")
        noverlap = nperseg // 2 if noverlap is None else int(noverlap)
        if not 0 <= noverlap < nperseg:
            raise ValueError("noverlap must be less than nperseg.")
        tb = _tables(window, nperseg)
        if tb is None:
            raise ValueError("streaming STFT needs a named window")
        self.rows = int(rows)
        self.fs = float(fs)
        self.nperseg = int(nperseg)
        self.hop = nperseg - noverlap
        self.tables = tb
        self.scale = 1.0 / tb.sum_w
        self.tails = torch.zeros((2, self.rows, nperseg), dtype=torch.float32, device=device())
        self.parity = 0
        self.tail_len = 0
        self.frames_emitted = 0
        self.samples_seen = 0
        self.seg_per_task = seg_per_task
        self.busy = False
        self.event: torch.cuda.Event | None = None

    def prepare_chunk(self, chunk) -> StreamJob:
        """Bind the next chunk ((rows, m) or (m,) float32) and advance the host state. The chunk
        must stay alive until its batch completes (the job holds a reference)."""
        X = to_device(chunk)
        if X.is_complex():
            raise TypeError("streaming STFT takes real input")
        if X.dim() == 1:
            X = X.reshape(1, -1)
        if X.shape[0] != self.rows:
            raise ValueError(f"chunk has {X.shape[0]} rows, stream has {self.rows}")
        x2, ld = _rows_view(X)
        m = x2.shape[1]
        nt = ctypes.c_int64(0)
        f = _lib.load().sp_batch_stream_frames(self.tail_len, m, self.nperseg, self.hop,
                                               ctypes.byref(nt))
        if f < 0:
            _lib.check(int(f), "sp_batch_stream_frames")
        nb = self.nperseg // 2 + 1
        out = torch.empty((self.rows, int(f), nb), dtype=torch.complex64, device=x2.device)
        G = self.seg_per_task or default_cache().get("stft_stream", self.nperseg, self.rows)
        r = BatchRequest()
        r.kind = KIND_STREAM
        r.nperseg = self.nperseg
        r.hop = self.hop
        r.onesided = 1
        r.seg_per_task = int(G)
        r.tail_len = self.tail_len
        r.rows = self.rows
        r.n = m
        r.ld = ld
        r.tail_ld = self.nperseg
        r.x = x2.data_ptr()
        r.win = self.tables.win.data_ptr()
        r.tail_in = self.tails[self.parity].data_ptr()
        r.tail_out = self.tails[1 - self.parity].data_ptr()
        r.out = out.data_ptr()
        r.scale = self.scale
        job = StreamJob(r, out, x2, self, self.frames_emitted, int(f),
                        self.rows * m * 4 + out.numel() * 8)
        self.parity ^= 1
        self.tail_len = int(nt.value)
        self.frames_emitted += int(f)
        self.samples_seen += m
        return job


# ---------------------------------------------------------------------------------------------
# launching
# ---------------------------------------------------------------------------------------------


class _Slot:
    def __init__(self, ws_bytes: int, desc_bytes: int, dev: torch.device):
        self.stream = torch.cuda.Stream(device=dev)
        self.ws = torch.zeros(ws_bytes, dtype=torch.uint8, device=dev)
        self.desc_host = torch.empty(desc_bytes, dtype=torch.uint8, pin_memory=True)
        self.desc_dev = torch.empty(desc_bytes, dtype=torch.uint8, device=dev)
        self.graph: torch.cuda.CUDAGraph | None = None
        self.event = torch.cuda.Event()
        self.used = False
        self.keep: list = []  # inputs/outputs of the batch in flight


def _as_array(reqs):
    """(address, count, owner) of a request array: a BatchRequest list or a REQ_DTYPE array."""
    if isinstance(reqs, np.ndarray):
        assert reqs.dtype == REQ_DTYPE and reqs.flags.c_contiguous
        return reqs.ctypes.data if len(reqs) else 0, len(reqs), reqs
    arr = (BatchRequest * max(1, len(reqs)))()
    for i, r in enumerate(reqs):
        arr[i] = r
    return ctypes.addressof(arr), len(reqs), arr


class BatchLauncher:
    """Launch batches of jobs as one batched launch (`sp_batch_run`) each.

    Each slot owns a CUDA stream, a zero-initialised workspace (queue, row counters, partial
    sums), and a descriptor buffer pair (pinned host, device). A launch picks the next slot
    (waiting on the host only if that slot's previous batch is still running), encodes the
    descriptors into its pinned buffer and either replays the slot's CUDA graph (descriptor
    copy + kernel, captured at the slot's second launch) or issues the copy and the kernel.
    Several slots let consecutive batches overlap on the device.
    """

    def __init__(self, max_requests: int = 1024, ws_bytes: int = 64 << 20, slots: int = 2,
                 use_graph: bool = True, grid: int = 0):
        self.dev = device()
        self.lib = _lib.load()
        self.max_requests = int(max_requests)
        self.desc_bytes = _desc_bytes(self.max_requests)
        self.ws_bytes = int(ws_bytes)
        self.use_graph = bool(use_graph)
        self.grid = int(grid)
        self.slots = [_Slot(self.ws_bytes, self.desc_bytes, self.dev) for _ in range(slots)]
        self._next = 0
        self.last_stream: torch.cuda.Stream | None = None
        self.launches = 0

    def plan(self, reqs) -> tuple[int, int]:
        """(descriptor bytes, workspace bytes) of a batch."""
        return plan(reqs)

    def _run(self, slot: _Slot) -> None:
        slot.desc_dev.copy_(slot.desc_host, non_blocking=True)
        _lib.check(self.lib.sp_batch_run(slot.desc_dev.data_ptr(), slot.ws.data_ptr(),
                                         self.grid, stream_handle()),
                   "sp_batch_run")

    def launch(self, reqs, wait_events=(), keep=None) -> torch.cuda.Event:
        """Encode and launch `reqs` (BatchRequest list, at most max_requests). The slot's stream
        first waits on `wait_events`. Returns the event recorded after the kernel; `keep`
        (any object) is referenced until that slot is reused."""
        if len(reqs) > self.max_requests:
            raise ValueError(f"{len(reqs)} requests exceed max_requests={self.max_requests}")
        slot = self.slots[self._next]
        self._next = (self._next + 1) % len(self.slots)
        if slot.used:
            slot.event.synchronize()  # its descriptors / workspace are about to be rewritten
        slot.keep = []
        addr, count, _owner = _as_array(reqs)
        _lib.check(self.lib.sp_batch_encode(addr, count, slot.ws.data_ptr(), slot.ws.numel(),
                                            slot.desc_host.data_ptr(), self.desc_bytes),
                   "sp_batch_encode")
        cur = torch.cuda.current_stream(current_index())
        slot.stream.wait_stream(cur)  # inputs produced on the caller's stream
        for ev in wait_events:
            slot.stream.wait_event(ev)
        with torch.cuda.stream(slot.stream):
            if self.use_graph and slot.graph is not None:
                slot.graph.replay()
            elif self.use_graph and slot.used:
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=slot.stream):
                    self._run(slot)
                slot.graph = g
                g.replay()
            else:
                self._run(slot)
            slot.event.record(slot.stream)
        slot.used = True
        slot.keep = [keep]
        self.last_stream = slot.stream
        self.launches += 1
        return slot.event

    def synchronize(self) -> None:
        for s in self.slots:
            if s.used:
                s.event.synchronize()


def plan(reqs) -> tuple[int, int]:
    """Validate a batch (BatchRequest list or REQ_DTYPE array): (descriptor bytes, workspace
    bytes)."""
    addr, count, _owner = _as_array(reqs)
    d = ctypes.c_int64(0)
    w = ctypes.c_int64(0)
    _lib.check(_lib.load().sp_batch_plan(addr, count, ctypes.byref(d), ctypes.byref(w)),
               "sp_batch_plan")
    return int(d.value), int(w.value)


def _desc_bytes(nreq: int) -> int:
    # header (16) + item_begin[nreq+1] padded to 16 + 144 per request
    return 16 + ((4 * (nreq + 1) + 15) & ~15) + 144 * nreq


def welch_batch(signals, **kwargs):
    """welch over many signals: one persistent launch for every request the batched kernel
    serves, the regular `welch` for the others. `signals` is a sequence of arrays (sharing
    `kwargs`) or of (array, per-request kwargs) pairs. Returns the list of (freqs, Pxx)."""
    from .spectral import welch

    items = []
    for s in signals:
        if isinstance(s, tuple) and len(s) == 2 and isinstance(s[1], dict):
            items.append((s[0], {**kwargs, **s[1]}))
        else:
            items.append((s, dict(kwargs)))
    jobs = [prepare_welch(x, **kw) for x, kw in items]
    batch = [j for j in jobs if j is not None]
    if batch:
        lib = _lib.load()
        reqs = [j.req for j in batch]
        d, w = plan(reqs)
        addr, count, _owner = _as_array(reqs)
        dev = device()
        ws = torch.zeros(w, dtype=torch.uint8, device=dev)
        host = torch.empty(d, dtype=torch.uint8, pin_memory=True)
        _lib.check(lib.sp_batch_encode(addr, count, ws.data_ptr(), ws.numel(), host.data_ptr(),
                                       host.numel()), "sp_batch_encode")
        # torch's pinned-memory allocator holds `host` until the copy has run
        desc = host.to(dev, non_blocking=True)
        _lib.check(lib.sp_batch_run(desc.data_ptr(), ws.data_ptr(), 0, stream_handle()),
                   "sp_batch_run")
    out = []
    for (x, kw), j in zip(items, jobs):
        if j is not None:
            out.append(j.result())
        else:
            out.append(welch(x, **kw))
    return out
