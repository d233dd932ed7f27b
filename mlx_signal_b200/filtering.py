"""Analytic signal (Hilbert transform) over the long FFTs (scipy.signal.hilbert semantics).

Counterpart of the reference's `hilbert` (src/mlx_signal_processing/filtering.py:43-84): a real
forward transform of length N, the analytic spectrum (DC and, for even N, Nyquist kept, positive
bins doubled, negative bins zero), and an inverse complex transform of length N. Lengths whose
transforms the three-pass kernels cover (`mlx_signal_b200.fft`) run there; other lengths run
cuFFT through torch (the composed GPU path). Returns complex64 on the GPU.
"""

from __future__ import annotations

import torch

from . import fft as _fft
from ._array import to_device

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
