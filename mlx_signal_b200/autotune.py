"""Schedules for the batched persistent launch, measured and cached per (kind, nperseg, dtype,
channels).

The schedule knob of the batch kernel is the work of one team task: segments per task for welch
requests (each task then writes one partial row, so larger tasks mean less partial traffic and
fewer counter atomics, smaller tasks a shorter tail), frames per task for streaming-STFT chunks.
The FFT radix sequence is fixed per nperseg by the CTA shape (teams of P = L/E threads, E = 32
points per thread at L = 1024 and 16 at the other classes; 128-thread CTAs up to L = 2048, one
256-thread team per CTA at 4096), and the grids are the resident maxima (the queues balance
them). A schedule changes only how work is cut, never which
arithmetic is done; a request's result is bit-identical under every schedule only up to the
grouping of its partial sums, so the schedule of a request depends on its own
(kind, nperseg, dtype, channels) key, never on the other requests of a batch -- a request gives
the same bits alone and inside any mix.

`ScheduleCache` keeps the chosen values (in memory, and in a JSON file when a path is given or
the MLX_SIGNAL_B200_SCHEDULES environment variable names one); `tune` times the candidates
on the device with CUDA events and records the fastest.
"""

from __future__ import annotations

import json
import os
import threading
from pathlib import Path

import torch

__all__ = ["ScheduleCache", "channels_bucket", "default_cache", "tune"]

WELCH_CANDIDATES = (8, 16, 32, 64, 128)
STREAM_CANDIDATES = (4, 8, 16, 32, 64)
_DEFAULTS = {"welch": 64, "stft_stream": 16}


def channels_bucket(rows: int) -> int:
    """Power-of-two bucket of the channel count (1, 2, 4, ..., 64; larger counts share 64)."""
    b = 1
    while b < rows and b < 64:
        b <<= 1
    return b


def _key(kind: str, nperseg: int, dtype: str, rows: int) -> str:
    return f"{kind}/{int(nperseg)}/{dtype}/c{channels_bucket(int(rows))}"


class ScheduleCache:
    """Chosen segments-per-task by (kind, nperseg, dtype, channels bucket)."""

    def __init__(self, path: str | os.PathLike | None = None):
        self.path = Path(path) if path else None
        self._lock = threading.Lock()
        self._entries: dict[str, dict] = {}
        if self.path is not None and self.path.exists():
            self._entries = json.loads(self.path.read_text())

    def get(self, kind: str, nperseg: int, rows: int, dtype: str = "float32") -> int:
        with self._lock:
            e = self._entries.get(_key(kind, nperseg, dtype, rows))
        return int(e["seg_per_task"]) if e else _DEFAULTS[kind]

    def put(self, kind: str, nperseg: int, rows: int, seg_per_task: int, dtype: str = "float32",
            timings_us: dict | None = None) -> None:
        entry = {"seg_per_task": int(seg_per_task)}
        if timings_us:
            entry["us"] = {str(k): round(float(v), 2) for k, v in timings_us.items()}
        with self._lock:
            self._entries[_key(kind, nperseg, dtype, rows)] = entry
            if self.path is not None:
                self.path.parent.mkdir(parents=True, exist_ok=True)
                tmp = self.path.with_suffix(".tmp")
                tmp.write_text(json.dumps(self._entries, indent=1, sort_keys=True))
                tmp.replace(self.path)

    def entries(self) -> dict[str, dict]:
        with self._lock:
            return dict(self._entries)

    def clear(self) -> None:
        with self._lock:
            self._entries.clear()


_default: ScheduleCache | None = None


def default_cache() -> ScheduleCache:
    global _default
    if _default is None:
        _default = ScheduleCache(os.environ.get("MLX_SIGNAL_B200_SCHEDULES") or None)
    return _default


def tune(kind: str, nperseg: int, channels: int, *, n: int = 1 << 18, copies: int | None = None,
         candidates=None, reps: int = 5, cache: ScheduleCache | None = None,
         seed: int = 0) -> int:
    """Time each candidate segments-per-task on a synthetic batch of `copies` requests of
    (channels, n) float32 N(0,1) samples (enough to fill the device several times over) and
    record the fastest in `cache` (default: the module cache). Returns the chosen value."""
    from . import batch as _batch

    cache = cache or default_cache()
    candidates = tuple(candidates or (WELCH_CANDIDATES if kind == "welch" else STREAM_CANDIDATES))
    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    if copies is None:
        per = channels * max(1, n // max(1, nperseg // 2))
        copies = max(4, min(256, (1 << 22) // max(per, 1)))
    xs = [torch.randn((channels, n), generator=g, device=dev) for _ in range(copies)]
    launcher = _batch.BatchLauncher(max_requests=copies, slots=1, use_graph=False)
    timings = {}
    for G in candidates:
        if kind == "welch":
            jobs = [_batch.prepare_welch(x, nperseg=nperseg, seg_per_task=G) for x in xs]
        else:
            streams = [_batch.StftStream(rows=channels, nperseg=nperseg, noverlap=3 * nperseg // 4,
                                         seg_per_task=G) for _ in xs]
            jobs = [s.prepare_chunk(x) for s, x in zip(streams, xs)]
        reqs = [j.req for j in jobs]
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        best = float("inf")
        for r in range(reps + 1):
            launcher.launch(reqs)  # warm-up on r == 0
            st = launcher.last_stream
            if r == 0:
                continue
            ev0.record(st)
            launcher.launch(reqs)
            ev1.record(st)
            ev1.synchronize()
            best = min(best, ev0.elapsed_time(ev1) * 1e3)
        timings[G] = best
    choice = min(timings, key=timings.get)
    cache.put(kind, nperseg, channels, choice, timings_us=timings)
    return choice
