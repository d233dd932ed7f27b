"""Splitting spectral work over the ranks of a torch.distributed group (one process per GPU).

Channels, requests and streams are independent: `row_range` and `assign_requests` partition
them with no collective (outputs stay on their rank, or the caller gathers them). The one split
that needs an exchange is a single channel too long for one GPU's share: its segments are cut
into contiguous ranges, each rank reads its samples plus the (nperseg - hop)-sample overlap into
the next range (`segment_slice`), computes the SUM of its segments' spectra, and one all-reduce
of the nfreq partial sums (`welch_long`) gives every rank the full average. Segment spectra are
independent of where the cut falls, so the result equals the single-device welch up to the
order of the final sum.

The reference runs on one device; this is the multi-GPU layout of the same computation.
"""

from __future__ import annotations

import heapq

import numpy as np
import torch

__all__ = ["assign_requests", "row_range", "segment_range", "segment_slice", "welch_long"]


def row_range(rows: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous balanced block [r0, r1) of `rows` independent rows for `rank`."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(int(rows), world)
    r0 = rank * base + min(rank, extra)
    return r0, r0 + base + (1 if rank < extra else 0)


def assign_requests(costs, world: int) -> list[int]:
    """Rank of each request: longest-processing-time-first greedy on `costs` (e.g. bytes), ties
    to the lower rank and the earlier request -- deterministic, so every rank computes the same
    assignment without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    out = [0] * len(costs)
    for i in order:
        load, r = heapq.heappop(heap)
        out[i] = r
        heapq.heappush(heap, (load + float(costs[i]), r))
    return out


def segment_range(nseg: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous balanced range [s0, s1) of a channel's `nseg` segments for `rank`."""
    return row_range(nseg, world, rank)


def segment_slice(n: int, nperseg: int, hop: int, s0: int, s1: int) -> tuple[int, int]:
    """Sample range [a, b) holding segments s0..s1-1 (segment s covers [s*hop, s*hop+nperseg)):
    the rank's own hop-spaced starts plus the overlap into the next rank's range."""
    if s1 <= s0:
        return 0, 0
    a = s0 * hop
    b = (s1 - 1) * hop + nperseg
    if b > n:
        raise ValueError("segment range runs past the signal")
    return a, b


def welch_long(x_slice, nseg_total: int, s0: int, s1: int, group=None, *, psd_mean=None,
               **welch_kwargs):
    """Welch PSD of one long channel split over the group's ranks by segment ranges.

    x_slice: this rank's samples `segment_slice(...)` (1-D). Every rank computes the mean PSD of
    its own segments (`psd_mean(x, **welch_kwargs)` -> (freqs, Pxx); default
    mlx_signal_b200.welch), weights it by its segment count, and one SUM all-reduce in float64
    over the group combines the partial sums; returns (freqs, Pxx) of the whole channel on every
    rank. welch_kwargs must give nperseg and may give noverlap (default nperseg // 2),
    window, fs, detrend, scaling, return_onesided; average must be 'mean'."""
    import torch.distributed as dist

    if welch_kwargs.get("average", "mean") != "mean":
        raise ValueError("a segment-split welch needs average='mean'")
    if psd_mean is None:
        from .spectral import welch as psd_mean
    nloc = s1 - s0
    if nloc > 0:
        f, p = psd_mean(x_slice, **welch_kwargs)
        part = torch.as_tensor(p).to(torch.float64) * float(nloc)
        f = torch.as_tensor(f)
    else:  # a rank without segments still joins the all-reduce with zeros
        nper = int(welch_kwargs["nperseg"])
        nfft = int(welch_kwargs.get("nfft") or nper)
        onesided = welch_kwargs.get("return_onesided", True)
        fs = float(welch_kwargs.get("fs", 1.0))
        fr = np.fft.rfftfreq(nfft, 1 / fs) if onesided else np.fft.fftfreq(nfft, 1 / fs)
        f = torch.from_numpy(fr.astype(np.float32))
        part = torch.zeros(fr.shape[0], dtype=torch.float64)
    dev = part.device
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        if dist.get_backend(group) == "nccl" and dev.type != "cuda":
            part = part.cuda()
        dist.all_reduce(part, op=dist.ReduceOp.SUM, group=group)
    pxx = (part / float(nseg_total)).to(torch.float32)
    return f, pxx.to(dev) if pxx.device != dev else pxx
