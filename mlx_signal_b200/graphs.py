"""CUDA-graph capture of a fixed-shape spectral call's launch sequence.

Small requests are launch- and host-bound: a welch call on 1 x 2^16 samples is two kernels of a few
microseconds behind tens of microseconds of argument handling. `GraphedCall` records the kernel
sequence of one call (after a warm-up that fills every host-side cache) into a CUDA graph with
static input buffers; each later call copies new data into those buffers (device to device) and
replays the graph. `graphed_welch` prepares a welch call that way: window, scale, spectral-detrend
table and frequency vector are computed once, outside the capture, and only the launches
(segment kernel + reduction) are captured. The batched launch has its own graph per launcher slot
(`batch.BatchLauncher`).
"""

from __future__ import annotations

import math

import numpy as np
import torch

from . import _kernels
from ._array import device, to_device
from .windows import _window_np, device_vector

__all__ = ["GraphedCall", "graphed_welch"]


class GraphedCall:
    """fn(*inputs) captured once; call(*new_inputs) -> fn's output for the new data.

    `example_inputs` are CUDA tensors whose shapes, dtypes and strides every later call repeats.
    fn may allocate (the graph keeps its private pool) but must only launch device work: no host
    round trips or host-to-device copies from pageable memory inside it."""

    def __init__(self, fn, *example_inputs: torch.Tensor):
        self.inputs = [t.detach().clone() for t in example_inputs]
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            fn(*self.inputs)  # warm-up: builds device tables and caches outside the capture
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.output = fn(*self.inputs)

    def __call__(self, *inputs: torch.Tensor):
        for dst, src in zip(self.inputs, inputs):
            if src.data_ptr() != dst.data_ptr():
                dst.copy_(src, non_blocking=True)
        self.graph.replay()
        return self.output


def graphed_welch(example, fs=1.0, window="hann", nperseg=None, noverlap=None, nfft=None,
                  detrend="constant", return_onesided=True, scaling="density"):
    """A replayable welch for inputs shaped like `example` ((rows, n) or (n,), last axis):
    returns (freqs, call) where call(x) gives the PSD of a new CUDA float32 x of that shape.
    Covers the fused path (real input, power-of-two nfft <= 4096, mean averaging)."""
    X = to_device(example)
    if X.is_complex():
        raise ValueError("graphed_welch covers real input")
    n = X.shape[-1]
    nper = 256 if nperseg is None else int(nperseg)
    nper = min(nper, n)
    w64 = _window_np(tuple(window) if isinstance(window, list) else window, nper)
    nft = nper if nfft is None else int(nfft)
    if not _kernels.fused_mean_ok(nft) or nft < nper:
        raise ValueError("graphed_welch needs a power-of-two nfft <= 4096 and >= nperseg")
    nov = nper // 2 if noverlap is None else int(noverlap)
    hop = nper - nov
    code = _kernels.DETREND_CODES[detrend if detrend in _kernels.DETREND_CODES else False]
    if scaling == "density":
        scale = 1.0 / (float(fs) * float((w64 * w64).sum()))
    elif scaling == "spectrum":
        scale = 1.0 / float(w64.sum()) ** 2
    else:
        raise ValueError(f"Unknown scaling: {scaling!r}")
    w32 = (w64 * math.sqrt(scale)).astype(np.float32)
    win = device_vector(w32)
    wdft = None
    if code == 1 and nper == nft and 2 * hop == nper:
        low = _kernels.window_low_spectrum(w32, nft)
        if low is not None:
            wdft = device_vector(low[0], dtype=torch.complex64)
    onesided = bool(return_onesided)
    rows_shape = tuple(X.shape[:-1])
    rows = int(np.prod(rows_shape)) if rows_shape else 1

    def fn(x):
        out = _kernels.welch_mean(x.reshape(rows, n), win, nper, nft, hop, code, onesided,
                                  wdft=wdft)
        return out.reshape(rows_shape + (out.shape[-1],))

    f = np.fft.rfftfreq(nft, 1 / fs) if onesided else np.fft.fftfreq(nft, 1 / fs)
    freqs = torch.from_numpy(f.astype(np.float32)).to(device())
    return freqs, GraphedCall(fn, X.contiguous())
