"""FFT convolution over the long FFTs (scipy.signal.fftconvolve / oaconvolve semantics).

Counterpart of the reference's `fftconvolve` and `oaconvolve` (src/mlx_signal_processing/
convolution.py:135-354): zero-padded transforms, a spectrum product and an inverse transform,
sliced to the 'full' / 'same' / 'valid' output. Along a single axis the padded length is a power
of two when the three-pass kernels (`mlx_signal_b200.fft`) cover it and it costs at most a
quarter more than the 5-smooth length scipy would use; otherwise, and for several axes, cuFFT runs
through torch (the composed GPU path). `oaconvolve` cuts the longer input into blocks, transforms
all blocks as one batch (short transforms: cuFFT), multiplies by the short input's spectrum and
overlap-adds the blocks.
Real data convolved with one filter of at most 2049 taps along one axis (the reference's fused
block-convolution case, convolution.py:288-306) runs the fused overlap-save kernel
(`sp_conv_ols_f32`) in both functions: one launch, blocks of up to 4096 samples, the mode's
output window written directly.
Results are float32 (complex64 if either input is complex) on the GPU.
"""

from __future__ import annotations

import math
import operator

import numpy as np
import torch

from . import _kernels
from . import fft as _fft
from ._array import to_device

__all__ = ["fftconvolve", "oaconvolve"]


def _next_fast_len(n: int) -> int:
    from scipy.fft import next_fast_len

    return int(next_fast_len(int(n), real=True))


def _conv_len(n: int) -> int:
    """Padded transform length for a linear convolution of total length n along one axis."""
    fast = _next_fast_len(n)
    p2 = 1 << max(0, (n - 1).bit_length())
    half_ok = p2 % 2 == 0 and _fft._pow2_in_range(p2 // 2)
    return p2 if half_ok and p2 <= fast + fast // 4 else fast


def _init_axes(a1: torch.Tensor, a2: torch.Tensor, mode: str, axes):
    """scipy's axis handling: default all axes, axes are integers (scalar or iterable), non-
    convolution axes must broadcast, 'valid' needs one input at least as large as the other along
    every axis (swapped if needed), axes where both sizes are 1 are dropped. Returns
    (a1, a2, axes)."""
    if mode not in ("full", "same", "valid"):
        raise ValueError("acceptable mode flags are 'valid', 'same', or 'full'")
    nd = a1.dim()
    if axes is None:
        axes = list(range(nd))
    else:
        try:
            axes = [operator.index(a) for a in np.atleast_1d(axes).tolist()]
        except TypeError:
            raise ValueError("axes must be a scalar or iterable of integers") from None
        axes = [a + nd if a < 0 else a for a in axes]
        if any(a < 0 or a >= nd for a in axes):
            raise ValueError("axes exceeds dimensionality of input")
        if len(set(axes)) != len(axes):
            raise ValueError("all axes must be unique")
    for a in range(nd):
        if a not in axes and a1.shape[a] != a2.shape[a] and a1.shape[a] != 1 \
                and a2.shape[a] != 1:
            raise ValueError(f"incompatible shapes for in1 and in2: {tuple(a1.shape)} and "
                             f"{tuple(a2.shape)}")
    if mode == "valid":
        ge = all(a1.shape[a] >= a2.shape[a] for a in axes)
        le = all(a1.shape[a] <= a2.shape[a] for a in axes)
        if not (ge or le):
            raise ValueError("For 'valid' mode, one must be at least as large as the other in "
                             "every dimension")
        if not ge:
            a1, a2 = a2, a1
    axes = [a for a in axes if a1.shape[a] != 1 and a2.shape[a] != 1]
    return a1, a2, axes


def _centered(t: torch.Tensor, shape) -> torch.Tensor:
    idx = []
    for cur, new in zip(t.shape, shape):
        s = (cur - new) // 2
        idx.append(slice(s, s + new))
    return t[tuple(idx)]


def _apply_mode(ret, s1, s2, mode, axes):
    if mode == "full":
        return ret
    if mode == "same":
        return _centered(ret, s1)
    shape = [ret.shape[a] if a not in axes else s1[a] - s2[a] + 1 for a in range(ret.dim())]
    return _centered(ret, shape)


def _promote(a1, a2):
    cplx = a1.is_complex() or a2.is_complex()
    if cplx:
        a1 = a1.to(torch.complex64)
        a2 = a2.to(torch.complex64)
    return a1, a2, cplx


def _freq_conv(a1, a2, axes, shape, same_input=False):
    a1, a2, cplx = _promote(a1, a2)
    if len(axes) == 1:
        ax = axes[0]
        fl = _conv_len(shape[ax])
        if cplx:
            s1 = _fft.fft(a1, n=fl, axis=ax)
            s2 = s1 if same_input else _fft.fft(a2, n=fl, axis=ax)
            ret = _fft.ifft(s1 * s2, n=fl, axis=ax)
        else:
            s1 = _fft.rfft(a1, n=fl, axis=ax)
            s2 = s1 if same_input else _fft.rfft(a2, n=fl, axis=ax)
            ret = _fft.irfft(s1 * s2, n=fl, axis=ax)
    else:
        fshape = [_next_fast_len(shape[a]) for a in axes]
        if cplx:
            s1 = torch.fft.fftn(a1, s=fshape, dim=axes)
            s2 = s1 if same_input else torch.fft.fftn(a2, s=fshape, dim=axes)
            ret = torch.fft.ifftn(s1 * s2, s=fshape, dim=axes)
        else:
            s1 = torch.fft.rfftn(a1, s=fshape, dim=axes)
            s2 = s1 if same_input else torch.fft.rfftn(a2, s=fshape, dim=axes)
            ret = torch.fft.irfftn(s1 * s2, s=fshape, dim=axes)
    idx = tuple(slice(shape[a]) if a in axes else slice(None) for a in range(ret.dim()))
    return ret[idx]


def _fused_ols(a1, a2, axes, s1, s2, mode):
    """The fused overlap-save kernel's result when it covers the call (one real convolution
    axis, the shorter input a single filter of at most CONV_MAX_TAPS taps: size 1 on every other
    axis), else None. The kernel writes the mode's window of the full convolution directly."""
    if len(axes) != 1 or a1.is_complex() or a2.is_complex():
        return None
    ax = axes[0]
    longer, shorter = (a1, a2) if s1[ax] >= s2[ax] else (a2, a1)
    if shorter.shape[ax] > _kernels.CONV_MAX_TAPS or any(
            d != 1 for i, d in enumerate(shorter.shape) if i != ax):
        return None
    n1, n2 = longer.shape[ax], shorter.shape[ax]
    full = n1 + n2 - 1
    if mode == "full":
        j0, nout = 0, full
    else:
        nout = s1[ax] if mode == "same" else s1[ax] - s2[ax] + 1
        j0 = (full - nout) // 2
    xl = longer.movedim(ax, -1)
    lead = tuple(xl.shape[:-1])
    out = _kernels.conv_ols(xl.reshape(-1, n1), shorter.reshape(-1), j0, nout)
    out = out.reshape(lead + (nout,)).movedim(-1, ax)
    if mode == "same":  # scipy centres every axis on in1's shape
        out = _centered(out, [s1[i] if i != ax else nout for i in range(out.dim())])
    return out


def fftconvolve(in1, in2, mode="full", axes=None):
    """Convolve two N-dimensional arrays with zero-padded FFTs (scipy semantics). A single
    filter of at most 2049 taps along one axis of real data runs the fused overlap-save kernel
    (same result; shorter transforms)."""
    a1, a2 = to_device(in1), to_device(in2)
    if a1.dim() == 0 and a2.dim() == 0:
        return a1 * a2
    if a1.dim() != a2.dim():
        raise ValueError("in1 and in2 should have the same dimensionality")
    if a1.numel() == 0 or a2.numel() == 0:
        return torch.zeros((0,), dtype=a1.dtype, device=a1.device)
    same_input = in1 is in2
    a1, a2, axes = _init_axes(a1, a2, mode, axes)
    s1, s2 = tuple(a1.shape), tuple(a2.shape)
    if not axes:
        return a1 * a2
    fused = _fused_ols(a1, a2, axes, s1, s2, mode)
    if fused is not None:
        return fused
    shape = [max(s1[i], s2[i]) if i not in axes else s1[i] + s2[i] - 1 for i in range(a1.dim())]
    ret = _freq_conv(a1, a2, axes, shape, same_input=same_input)
    return _apply_mode(ret, s1, s2, mode, axes)


def _oa_block(n_long: int, n_short: int) -> int:
    """Block length: the transform length F = block + n_short - 1 is the smallest power of two
    at least 4x the short input (at least 256), capped by the long input."""
    f = max(1 << 8, 1 << max(0, (4 * n_short - 1).bit_length()))
    return max(1, min(f - n_short + 1, n_long))


def oaconvolve(in1, in2, mode="full", axes=None):
    """Convolve with the overlap-add method (scipy semantics; same result as fftconvolve).

    Along a single convolution axis the longer input is cut into blocks of b samples, all blocks
    are transformed as one batch at length F = b + len(short) - 1, multiplied by the short
    input's spectrum, inverse-transformed and overlap-added (block j's F outputs start at j*b).
    With several convolution axes, or inputs of equal length, one padded transform is used."""
    a1, a2 = to_device(in1), to_device(in2)
    if a1.dim() == 0 and a2.dim() == 0:
        return a1 * a2
    if a1.dim() != a2.dim():
        raise ValueError("in1 and in2 should have the same dimensionality")
    if a1.numel() == 0 or a2.numel() == 0:
        return torch.zeros((0,), dtype=a1.dtype, device=a1.device)
    a1, a2, axes = _init_axes(a1, a2, mode, axes)
    s1, s2 = tuple(a1.shape), tuple(a2.shape)
    if not axes:
        return a1 * a2
    fused = _fused_ols(a1, a2, axes, s1, s2, mode)
    if fused is not None:
        return fused
    shape = [max(s1[i], s2[i]) if i not in axes else s1[i] + s2[i] - 1 for i in range(a1.dim())]
    if len(axes) != 1 or s1[axes[0]] == s2[axes[0]]:
        return _apply_mode(_freq_conv(a1, a2, axes, shape), s1, s2, mode, axes)
    ax = axes[0]
    longer, shorter = (a1, a2) if s1[ax] > s2[ax] else (a2, a1)
    longer, shorter, cplx = _promote(longer, shorter)
    L = longer.movedim(ax, -1)
    S = shorter.movedim(ax, -1)
    # broadcast the non-convolution axes (scipy allows size-1 against size-n there)
    lead = torch.broadcast_shapes(L.shape[:-1], S.shape[:-1])
    L = L.expand(lead + (L.shape[-1],))
    S = S.expand(lead + (S.shape[-1],))
    nl, ns = L.shape[-1], S.shape[-1]
    b = _oa_block(nl, ns)
    nblk = math.ceil(nl / b)
    fl = b + ns - 1
    pad = nblk * b - nl
    if pad:
        L = torch.cat([L, torch.zeros(lead + (pad,), dtype=L.dtype, device=L.device)], dim=-1)
    blocks = L.reshape(lead + (nblk, b))
    if cplx:
        prod = _fft.fft(blocks, n=fl, axis=-1) * _fft.fft(S, n=fl, axis=-1).unsqueeze(-2)
        seg = _fft.ifft(prod, n=fl, axis=-1)
    else:
        prod = _fft.rfft(blocks, n=fl, axis=-1) * _fft.rfft(S, n=fl, axis=-1).unsqueeze(-2)
        seg = _fft.irfft(prod, n=fl, axis=-1)
    y = torch.zeros(lead + (nblk * b + ns - 1,), dtype=seg.dtype, device=seg.device)
    y[..., : nblk * b] = seg[..., :b].reshape(lead + (nblk * b,))
    if ns > 1:  # each block's tail overlaps the start of the next blocks
        idx = (torch.arange(nblk, device=y.device)[:, None] * b + b
               + torch.arange(ns - 1, device=y.device)[None, :]).reshape(-1)
        y.index_add_(y.dim() - 1, idx, seg[..., b:].reshape(lead + (nblk * (ns - 1),)))
    y = y[..., : nl + ns - 1].movedim(-1, ax)
    return _apply_mode(y, s1, s2, mode, axes)
