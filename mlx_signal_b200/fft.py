"""Long FFTs on B200: rfft / irfft / fft / ifft along one axis.

Counterpart of the reference's FFT routing for long transforms (src/mlx_signal_processing/
_fft_core.py:55-104 -> _fourstep.rfft_large / irfft_large / fft_large / ifft_large,
_fourstep.py:177-231, 372-408 -> _fourstep_metal.fft3_last for 2^21..2^26). The C-ABI takes
complex lengths that are powers of two in [2^12, 2^26] (three TMA-staged passes) and real
lengths n = 2 C 2^e with C odd <= 15 (the C decimated branches as one batch of packed
power-of-two transforms around one radix-C kernel on each side). This module routes a transform
to those kernels where they are faster than cuFFT (torch.fft) on B200, by device time measured
with CUDA-graph replay (microseconds, ours / cuFFT):
  complex fft  2^21: 29.9 / 20.1   2^22: 47.2 / 48.8   2^23: 82.1 / 97.9   2^24: 156 / 185
  rfft         n = 2^22: 34.9 / 25.7   2^23: 56.4 / 59.2   2^25: 203 / 231
  irfft        n = 2^22: 42.9 / 40.3   2^23: 72.1 / 88.8   2^25: 244 / 356
  irfft        n = 3 2^22: 117 / 145   5 2^22: 191 / 230   (3 2^20: 42.7 / 41.1)
  rfft         n = 3 2^22: 124 / 99.6  (odd-factor forward: cuFFT is faster at every size)
i.e. from 2^KERNEL_MIN_LOG2 = 2^22 complex points (n/2 for the real transforms); odd-factor
forward transforms stay on cuFFT unless ODD_FORWARD is set (the fused resample uses them
directly). Other lengths run cuFFT (the composed GPU path; the reference uses MLX's own FFT
there). numpy.fft semantics for `n` (zero-pad or truncate) and `axis`.
"""

from __future__ import annotations

import math

import torch

from . import _lib
from ._array import stream_handle, to_device
from ._config import composed_path_notice

__all__ = ["DeviceWaitTimeout", "device_status", "fft", "ifft", "irfft", "rfft"]

MIN_LOG2, MAX_LOG2 = 12, 26   # lengths the C-ABI accepts
KERNEL_MIN_LOG2 = 22          # lengths the Python API routes to the kernels (complex points)
ODD_FORWARD = False           # odd-factor rfft on the kernels (measured slower than cuFFT)
RESAMPLE_MIN_LOG2 = 20        # fused resample from max(n, num)/2 = 2^20 (measured faster)


MAX_ODD = 15                  # largest odd factor C of a real length n = 2 C 2^e


def _pow2_in_range(m: int) -> bool:
    """True when a complex transform of length m runs on the three-pass kernels."""
    lo = max(MIN_LOG2, KERNEL_MIN_LOG2)
    return m >= 1 and (m & (m - 1)) == 0 and lo <= m.bit_length() - 1 <= MAX_LOG2


def _real_split(n: int) -> tuple[int, int] | None:
    """(C, e) with n = 2 C 2^e, C odd <= MAX_ODD and e in the C-ABI's range, else None."""
    if n < 2 or n % 2:
        return None
    h = n // 2
    c = h
    while c % 2 == 0:
        c //= 2
    e = (h // c).bit_length() - 1
    if c > MAX_ODD or not MIN_LOG2 <= e <= MAX_LOG2:
        return None
    return c, e


def _real_in_range(n: int, inverse: bool = False) -> bool:
    """True when a real transform of length n runs on the kernels: n/2 a power of two in the
    routed range, or C 2^e (C odd <= 15; the C branches run as one batch of packed 2^e-point
    transforms) with n/2 >= 2^KERNEL_MIN_LOG2 for the inverse (the forward only with
    ODD_FORWARD)."""
    sp = _real_split(n)
    if sp is None:
        return False
    c, _ = sp
    if c == 1:
        return _pow2_in_range(n // 2)
    return (inverse or ODD_FORWARD) and n // 2 >= (1 << KERNEL_MIN_LOG2)


def _resample_in_range(n: int, num: int) -> bool:
    """True when a real, unwindowed resample n -> num runs as one fused C-ABI call."""
    return (_real_split(n) is not None and _real_split(num) is not None
            and max(n, num) // 2 >= (1 << RESAMPLE_MIN_LOG2))


def _notice_long(func_name: str, m: int) -> None:
    """cuFFT is this module's designed path for complex lengths below 2^KERNEL_MIN_LOG2 (it is
    faster there); a long transform the three-pass kernels cannot take (not a power of two, or
    beyond 2^26) is a fallback and says so."""
    if m >= (1 << KERNEL_MIN_LOG2):
        composed_path_notice(func_name, "length outside the three-pass kernels")


def _last(t: torch.Tensor, axis: int) -> torch.Tensor:
    return t.movedim(axis, -1) if t.dim() > 1 and axis not in (-1, t.dim() - 1) else t


def _back(t: torch.Tensor, axis: int) -> torch.Tensor:
    return t.movedim(-1, axis) if t.dim() > 1 and axis not in (-1, t.dim() - 1) else t


def _fit(t: torch.Tensor, n: int) -> torch.Tensor:
    cur = t.shape[-1]
    if cur == n:
        return t
    if cur > n:
        return t[..., :n]
    pad = torch.zeros(t.shape[:-1] + (n - cur,), dtype=t.dtype, device=t.device)
    return torch.cat([t, pad], dim=-1)


def _rows16(t: torch.Tensor, rows: int, n: int) -> torch.Tensor:
    """t as a contiguous (rows, n) tensor whose data starts on a 16-byte boundary (the TMA
    tensor maps' base rule; a view into the middle of a buffer is copied)."""
    r = t.reshape(rows, n).contiguous()
    return r if r.data_ptr() % 16 == 0 else r.clone()


def _workspace(n_complex: int, batch: int, dev) -> torch.Tensor:
    nbytes = _lib.load().sp_fft_workspace_size(n_complex, batch)
    if nbytes < 0:
        _lib.check(int(nbytes), "sp_fft_workspace_size")
    return torch.empty(int(nbytes), dtype=torch.uint8, device=dev)


class DeviceWaitTimeout(_lib.KernelError):
    """A long transform's bounded device wait ran out (SP_ERR_TIMEOUT in its error word): its
    output is undefined."""


class _StatusWatch:
    """Host watchdog for the long transforms' bounded device waits. A wait that runs out stores
    SP_ERR_TIMEOUT in the transform's workspace word and in a process-wide sticky word in mapped
    pinned host memory (sp_fft_sticky_error); a later call, or `device_status()`, reads the
    sticky word with a plain host load (no copy, no event, allowed while a CUDA graph is being
    captured) and raises DeviceWaitTimeout. `record` only notes which kind of transform ran
    last, for the message."""

    def __init__(self):
        self.last = "long transform"

    def record(self, ws: torch.Tensor, n_complex: int, batch: int, what: str) -> None:
        self.last = what

    def poll(self, wait_all: bool = False) -> int:
        if wait_all and torch.cuda.is_available() and not torch.cuda.is_current_stream_capturing():
            torch.cuda.synchronize()
        status = int(_lib.load().sp_fft_sticky_error(1))
        if status != 0:
            text = ("a bounded device wait ran out; the output of that transform is undefined"
                    if status == _lib.SP_ERR_TIMEOUT else "device error word set")
            raise DeviceWaitTimeout(self.last, status, text)
        return 0


_watch = _StatusWatch()


def device_status() -> int:
    """Wait for every long transform issued so far and return 0, or raise DeviceWaitTimeout if
    one of them recorded a device-side wait timeout."""
    return _watch.poll(wait_all=True)


def rfft(a, n: int | None = None, axis: int = -1) -> torch.Tensor:
    """One-sided FFT of real input (complex64 out, n//2+1 bins)."""
    _watch.poll()
    x = to_device(a)
    if x.is_complex():
        x = x.real
    x = _last(x, axis)
    n = x.shape[-1] if n is None else int(n)
    x = _fit(x, n)
    if _real_in_range(n):
        batch = tuple(x.shape[:-1])
        rows = math.prod(batch)
        xr = _rows16(x, rows, n)
        out = torch.empty((rows, n // 2 + 1), dtype=torch.complex64, device=x.device)
        ws = _workspace(n // 2, rows, x.device)
        _lib.check(_lib.load().sp_rfft_c64(xr.data_ptr(), out.data_ptr(), rows, n, n // 2 + 1,
                                           ws.data_ptr(), ws.numel(), stream_handle()),
                   "sp_rfft_c64")
        _watch.record(ws, n // 2, rows, "rfft")
        return _back(out.reshape(batch + (n // 2 + 1,)), axis)
    if _real_split(n) is None:  # an odd-factor length here is cuFFT by measurement, not a fallback
        _notice_long("rfft", n // 2)
    return _back(torch.fft.rfft(x, n=n, dim=-1), axis)


def irfft(a, n: int | None = None, axis: int = -1) -> torch.Tensor:
    """Inverse of rfft: real float32 output of length n (default 2*(bins-1))."""
    _watch.poll()
    X = to_device(a)
    if not X.is_complex():
        X = X.to(torch.complex64)
    X = _last(X, axis)
    n = 2 * (X.shape[-1] - 1) if n is None else int(n)
    if _real_in_range(n, inverse=True):
        batch = tuple(X.shape[:-1])
        rows = math.prod(batch)
        nb = min(X.shape[-1], n // 2 + 1)
        Xr = X[..., :nb].reshape(rows, nb).contiguous()
        out = torch.empty((rows, n), dtype=torch.float32, device=X.device)
        ws = _workspace(n // 2, rows, X.device)
        _lib.check(_lib.load().sp_irfft_f32(Xr.data_ptr(), nb, nb, out.data_ptr(), rows, n,
                                            ws.data_ptr(), ws.numel(), stream_handle()),
                   "sp_irfft_f32")
        _watch.record(ws, n // 2, rows, "irfft")
        return _back(out.reshape(batch + (n,)), axis)
    if _real_split(n) is None:
        _notice_long("irfft", n // 2)
    return _back(torch.fft.irfft(X, n=n, dim=-1), axis)


def _cfft(a, n, axis, inverse: bool) -> torch.Tensor:
    _watch.poll()
    z = to_device(a)
    if not z.is_complex():
        z = z.to(torch.complex64)
    z = _last(z, axis)
    n = z.shape[-1] if n is None else int(n)
    z = _fit(z, n)
    if _pow2_in_range(n):
        batch = tuple(z.shape[:-1])
        rows = math.prod(batch)
        zr = _rows16(z, rows, n)
        out = torch.empty((rows, n), dtype=torch.complex64, device=z.device)
        ws = _workspace(n, rows, z.device)
        _lib.check(_lib.load().sp_fft_c64(zr.data_ptr(), out.data_ptr(), rows, n, int(inverse),
                                          ws.data_ptr(), ws.numel(), stream_handle()),
                   "sp_fft_c64")
        _watch.record(ws, n, rows, "ifft" if inverse else "fft")
        return _back(out.reshape(batch + (n,)), axis)
    _notice_long("ifft" if inverse else "fft", n)
    f = torch.fft.ifft if inverse else torch.fft.fft
    return _back(f(z, n=n, dim=-1), axis)


def fft(a, n: int | None = None, axis: int = -1) -> torch.Tensor:
    """Complex FFT along `axis` (complex64 out)."""
    return _cfft(a, n, axis, False)


def ifft(a, n: int | None = None, axis: int = -1) -> torch.Tensor:
    """Inverse complex FFT along `axis`, including 1/n."""
    return _cfft(a, n, axis, True)
