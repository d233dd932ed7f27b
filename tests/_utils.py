"""Shared test helpers: tolerance checks against float64 oracle results."""

import numpy as np
import torch


def as_np(x):
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    return np.asarray(x)


def assert_close(actual, desired, rtol=1e-4, atol_frac=1e-5):
    """|err| <= rtol*|ref| + atol_frac*max|ref| (the reference's tests/_utils.py:13-26 rule)."""
    a = as_np(actual)
    d = np.asarray(desired)
    assert a.shape == d.shape, f"shape mismatch: {a.shape} vs {d.shape}"
    scale = np.max(np.abs(d)) if d.size else 1.0
    if not np.isfinite(scale) or scale == 0.0:
        scale = 1.0
    np.testing.assert_allclose(a, d.astype(a.dtype), rtol=rtol, atol=atol_frac * scale)


def rel_err_bins(actual, desired, floor=1e-6):
    """Max relative error over bins whose magnitude exceeds `floor` x the peak (the
    accuracy bar of this project: <= 1e-5 on bins above 1e-6 of the peak)."""
    a = as_np(actual)
    a = a.astype(np.complex128 if np.iscomplexobj(a) else np.float64)
    d = np.asarray(desired)
    mag = np.abs(d)
    if mag.size == 0:
        return 0.0
    keep = mag > floor * mag.max()
    if not keep.any():
        return 0.0
    return float(np.max(np.abs(a[keep] - d[keep]) / mag[keep]))


def assert_cuda_f32(x, complex_ok=False):
    assert isinstance(x, torch.Tensor), f"expected torch.Tensor, got {type(x)}"
    assert x.is_cuda, "result must live on the GPU"
    allowed = (torch.float32, torch.complex64) if complex_ok else (torch.float32,)
    assert x.dtype in allowed, x.dtype


def make_sig(rng, shape, complex_=False):
    """N(0,1) plus a 0.5-amplitude tone at 0.12 cycles/sample (reference tests make_sig)."""
    x = rng.standard_normal(shape).astype(np.float32)
    n = shape[-1] if isinstance(shape, tuple) else shape
    t = np.arange(n, dtype=np.float32)
    x = x + 0.5 * np.sin(2 * np.pi * 0.12 * t).astype(np.float32)
    if complex_:
        x = (x + 1j * rng.standard_normal(shape)).astype(np.complex64)
    return x
