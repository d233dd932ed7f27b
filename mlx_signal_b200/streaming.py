"""Streaming spectral analysis for one caller: a ShortTimeFFT-style STFT and a running Welch PSD
over unbounded signals delivered in chunks, with their state kept on the device.

The reference has no streaming API (its STFT works on whole arrays, spectral.py:694-738); these
classes give the serving loop's stream state (`batch.StftStream`: the unconsumed tail of each
stream resident in HBM, frames computed by the batched kernel with the tail read in place) a
direct public form:

* `StreamingSTFT.push(chunk) -> (t, Zxx)` returns the frames the chunk completes. Concatenated over
  all pushes they are exactly scipy.signal.stft(concat(chunks), fs, window, nperseg, noverlap,
  boundary=None, padded=False, detrend=False, scaling='spectrum'). Batched nperseg classes with a
  named window run the batched stream kernel (tail || chunk read virtually, no copy); other
  shapes keep the tail and run the fused per-frame kernels on tail || chunk.
* `StreamingWelch.push(chunk)` folds the chunk's complete segments into an FP64 running sum of
  segment powers on the device; `psd()` is scipy.signal.welch(concat(chunks), ...,
  average='mean') of everything pushed so far.

Calls are stream-ordered on torch's current CUDA stream; push chunks of one object in order.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _kernels, _lib, batch
from ._array import device, stream_handle, to_device
from .spectral import _detrend_code, _freqs, stft, welch
from .windows import _window_np, device_vector

__all__ = ["StreamingSTFT", "StreamingWelch"]


def _rows2d(chunk) -> tuple[torch.Tensor, bool]:
    X = to_device(chunk)
    if X.is_complex():
        raise TypeError("streaming analysis takes real input")
    if X.dim() == 1:
        return X.reshape(1, -1), True
    if X.dim() != 2:
        raise ValueError("chunks are (n,) or (rows, n)")
    return X, False


class StreamingSTFT:
    """Streaming STFT of `rows` channels (see the module docstring for the frame semantics)."""

    def __init__(self, rows: int = 1, fs: float = 1.0, window="hann", nperseg: int = 1024,
                 noverlap: int | None = None):
        self.rows = int(rows)
        self.fs = float(fs)
        self.nperseg = int(nperseg)
        noverlap = self.nperseg // 2 if noverlap is None else int(noverlap)
        if self.nperseg < 1 or not 0 <= noverlap < self.nperseg:
            raise ValueError("need nperseg >= 1 and 0 <= noverlap < nperseg")
        self.noverlap = noverlap
        self.hop = self.nperseg - noverlap
        self.window = window
        self.frames_emitted = 0
        self.samples_seen = 0
        self._batched = None
        if self.nperseg in batch.BATCH_NPERSEG and batch._tables(window, self.nperseg) is not None:
            self._batched = batch.StftStream(self.rows, self.fs, window, self.nperseg, noverlap)
            self._ws = torch.zeros(0, dtype=torch.uint8, device=device())
        else:
            self._tail = torch.zeros((self.rows, 0), dtype=torch.float32, device=device())

    def _push_batched(self, X: torch.Tensor):
        job = self._batched.prepare_chunk(X)
        reqs = [job.req]
        d, w = batch.plan(reqs)
        if self._ws.numel() < w:  # zeroed once; the kernel resets its counters on exit
            self._ws = torch.zeros(w, dtype=torch.uint8, device=device())
        lib = _lib.load()
        addr, count, _owner = batch._as_array(reqs)
        host = torch.empty(d, dtype=torch.uint8, pin_memory=True)
        _lib.check(lib.sp_batch_encode(addr, count, self._ws.data_ptr(), self._ws.numel(),
                                       host.data_ptr(), host.numel()), "sp_batch_encode")
        # torch's pinned-memory allocator holds `host` until the copy has run
        desc = host.to(device(), non_blocking=True)
        _lib.check(lib.sp_batch_run(desc.data_ptr(), self._ws.data_ptr(), 0, stream_handle()),
                   "sp_batch_run")
        return job.result()

    def _push_frames(self, X: torch.Tensor):
        buf = torch.cat([self._tail, X], dim=-1) if self._tail.shape[-1] else X
        n = buf.shape[-1]
        nf = (n - self.nperseg) // self.hop + 1 if n >= self.nperseg else 0
        nb = self.nperseg // 2 + 1
        if nf == 0:
            self._tail = buf.contiguous()
            zxx = torch.zeros((self.rows, nb, 0), dtype=torch.complex64, device=buf.device)
        else:
            used = (nf - 1) * self.hop + self.nperseg
            _, _, zxx = stft(buf[:, :used], fs=self.fs, window=self.window,
                             nperseg=self.nperseg, noverlap=self.noverlap, boundary=None,
                             padded=False, detrend=False)
            self._tail = buf[:, nf * self.hop:].contiguous()
        idx = np.arange(self.frames_emitted, self.frames_emitted + nf)
        t = torch.from_numpy(((idx * self.hop + self.nperseg / 2) / self.fs).astype(np.float32))
        return t.to(zxx.device), zxx

    def push(self, chunk):
        """Feed the next chunk ((rows, m) or, with rows == 1, (m,)); returns (t, Zxx) of the frames
        it completes: t in seconds from the stream start (frame centres), Zxx (rows, nfreq,
        nframes) complex64, or (nfreq, nframes) for 1-D chunks."""
        X, flat = _rows2d(chunk)
        if X.shape[0] != self.rows:
            raise ValueError(f"chunk has {X.shape[0]} rows, stream has {self.rows}")
        if X.shape[-1] == 0:
            nb = self.nperseg // 2 + 1
            zxx = torch.zeros((self.rows, nb, 0), dtype=torch.complex64, device=X.device)
            t = torch.zeros(0, dtype=torch.float32, device=X.device)
            return t, (zxx[0] if flat else zxx)
        if self._batched is not None:
            t, zxx = self._push_batched(X)
        else:
            t, zxx = self._push_frames(X)
        self.frames_emitted += zxx.shape[-1]
        self.samples_seen += X.shape[-1]
        return t, (zxx[0] if flat else zxx)


class StreamingWelch:
    """Running Welch PSD (average='mean') of `rows` channels over a stream of chunks."""

    def __init__(self, rows: int = 1, fs: float = 1.0, window="hann", nperseg: int = 256,
                 noverlap: int | None = None, nfft: int | None = None, detrend="constant",
                 return_onesided: bool = True, scaling: str = "density"):
        self.rows = int(rows)
        self.fs = float(fs)
        self.nperseg = int(nperseg)
        noverlap = self.nperseg // 2 if noverlap is None else int(noverlap)
        if self.nperseg < 1 or not 0 <= noverlap < self.nperseg:
            raise ValueError("need nperseg >= 1 and 0 <= noverlap < nperseg")
        self.nfft = self.nperseg if nfft is None else int(nfft)
        if self.nfft < self.nperseg:
            raise ValueError("nfft must be greater than or equal to nperseg.")
        self.noverlap = noverlap
        self.hop = self.nperseg - noverlap
        self.kw = dict(fs=self.fs, window=window, nperseg=self.nperseg, noverlap=noverlap,
                       nfft=self.nfft, detrend=detrend, return_onesided=return_onesided,
                       scaling=scaling)
        self.code = _detrend_code(detrend)
        self.onesided = bool(return_onesided)
        self._fused = None
        if isinstance(window, str | tuple) and _kernels.fused_mean_ok(self.nfft):
            w64 = _window_np(tuple(window) if isinstance(window, tuple) else window,
                             self.nperseg)
            if scaling == "density":
                scale = 1.0 / (self.fs * float((w64 * w64).sum()))
            elif scaling == "spectrum":
                scale = 1.0 / float(w64.sum()) ** 2
            else:
                raise ValueError(f"Unknown scaling: {scaling!r}")
            w32 = (w64 * np.sqrt(scale)).astype(np.float32)
            wdft = None
            if self.code == 1 and self.nperseg == self.nfft and 2 * self.hop == self.nperseg:
                low = _kernels.window_low_spectrum(w32, self.nfft)
                if low is not None:
                    wdft = device_vector(low[0], dtype=torch.complex64)
            self._fused = (device_vector(w32), wdft)
        nout = self.nfft // 2 + 1 if self.onesided else self.nfft
        self._sum = torch.zeros((self.rows, nout), dtype=torch.float64, device=device())
        self._tail = torch.zeros((self.rows, 0), dtype=torch.float32, device=device())
        self.segments = 0
        self.samples_seen = 0

    def push(self, chunk) -> int:
        """Fold the chunk's complete segments into the running sum; returns how many."""
        X, _ = _rows2d(chunk)
        if X.shape[0] != self.rows:
            raise ValueError(f"chunk has {X.shape[0]} rows, stream has {self.rows}")
        buf = torch.cat([self._tail, X], dim=-1) if self._tail.shape[-1] else X
        n = buf.shape[-1]
        nseg = (n - self.nperseg) // self.hop + 1 if n >= self.nperseg else 0
        if nseg:
            used = (nseg - 1) * self.hop + self.nperseg
            seg = buf[:, :used]
            if self._fused is not None:
                win, wdft = self._fused
                mean = _kernels.welch_mean(seg, win, self.nperseg, self.nfft, self.hop,
                                           self.code, self.onesided, wdft=wdft)
            else:
                _, mean = welch(seg, **self.kw)
            self._sum += mean.to(torch.float64) * float(nseg)
            self._tail = buf[:, nseg * self.hop:].contiguous()
        else:
            self._tail = buf.contiguous()
        self.segments += nseg
        self.samples_seen += X.shape[-1]
        return nseg

    def psd(self):
        """(f, Pxx) of everything pushed so far: (nfreq,) and (rows, nfreq) float32."""
        if self.segments == 0:
            raise ValueError("no complete segment yet (fewer than nperseg samples pushed)")
        f = _freqs(self.nfft, self.fs, self.onesided)
        return f, (self._sum / self.segments).to(torch.float32)

    def reset(self) -> None:
        self._sum.zero_()
        self._tail = self._tail[:, :0]
        self.segments = 0
        self.samples_seen = 0
