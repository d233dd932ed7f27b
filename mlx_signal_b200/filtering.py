"""Analytic signal (Hilbert transform) over the long FFTs (scipy.signal.hilbert semantics).

Counterpart of the reference's `hilbert` (src/mlx_signal_processing/filtering.py:43-84): a real
forward transform of length N, the analytic spectrum (DC and, for even N, Nyquist kept, positive
bins doubled, negative bins zero), and an inverse complex transform of length N. When N and N/2
are powers of two the three-pass kernels take (`mlx_signal_b200.fft` routing), the whole chain
is one C-ABI call (`sp_hilbert_c64`: packed forward transform, one kernel that untangles it into
the masked spectrum, inverse transform in place); other lengths compose `mlx_signal_b200.fft`
transforms (cuFFT where the kernels do not apply) with the mask applied by torch ops. Returns
complex64 on the GPU.
"""

from __future__ import annotations

import torch

import math

from . import _lib
from . import fft as _fft
from ._array import stream_handle, to_device

__all__ = ["hilbert"]


def hilbert(x, N=None, axis=-1):
    """Analytic signal x + i H(x) along `axis`, length N (default: the input length)."""
    X = to_device(x)
    if X.is_complex():
        raise ValueError("x must be real.")
    if N is None:
        N = X.shape[axis]
    N = int(N)
    if N <= 0:
        raise ValueError("N must be positive.")
    moved = X.dim() > 1 and axis not in (-1, X.dim() - 1)
    if moved:
        X = X.movedim(axis, -1)
    if N % 2 == 0 and _fft._pow2_in_range(N // 2) and _fft._pow2_in_range(N):
        out = _fused(_fft._fit(X.to(torch.float32), N), N)
        return out.movedim(-1, axis) if moved else out
    Xr = _fft.rfft(X, n=N, axis=-1)
    h = N // 2
    spec = torch.zeros(Xr.shape[:-1] + (N,), dtype=torch.complex64, device=Xr.device)
    spec[..., 0] = Xr[..., 0]
    if N % 2 == 0:
        spec[..., 1:h] = 2.0 * Xr[..., 1:h]
        spec[..., h] = Xr[..., h]
    else:
        spec[..., 1 : h + 1] = 2.0 * Xr[..., 1 : h + 1]
    out = _fft.ifft(spec, axis=-1)
    return out.movedim(-1, axis) if moved else out


def _fused(x: torch.Tensor, N: int) -> torch.Tensor:
    """Analytic signal of the rows of x (..., N) float32 through sp_hilbert_c64."""
    batch = tuple(x.shape[:-1])
    rows = math.prod(batch)
    xr = _fft._rows16(x, rows, N)
    out = torch.empty((rows, N), dtype=torch.complex64, device=x.device)
    ws = _fft._workspace(N, rows, x.device)
    _lib.check(_lib.load().sp_hilbert_c64(xr.data_ptr(), out.data_ptr(), rows, N, ws.data_ptr(),
                                          ws.numel(), stream_handle()), "sp_hilbert_c64")
    _fft._watch.record(ws, N, rows, "hilbert")
    return out.reshape(batch + (N,))
