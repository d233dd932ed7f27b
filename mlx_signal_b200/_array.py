"""Array conversion and dtype policy: NumPy / torch / lists in, torch CUDA float32/complex64 out.

Mirrors the reference's ``to_mlx`` policy (src/mlx_signal_processing/_array.py:32-70):
float64/complex128 inputs are downcast with a :class:`DowncastWarning` (or rejected under
``float64="strict"``), integers/bools and half types become float32 silently, Python lists use
32-bit defaults silently. Outputs live on the current CUDA device; there is no CPU path.
"""

from __future__ import annotations

import warnings

import numpy as np
import torch

from ._config import DowncastWarning, get_config


_cuda_ready = False
# torch's C-extension accessors for the current device and raw stream (present in the torch
# releases this package is built against); the public helpers below are the fallback
_get_device = getattr(torch._C, "_cuda_getDevice", None)
_get_raw_stream = getattr(torch._C, "_cuda_getCurrentRawStream", None)


def current_index() -> int:
    """Index of torch's current CUDA device. After the first successful check this is one call
    into torch's C extension: the public torch.cuda helpers re-validate availability (environment
    and driver queries) on every call, which cost ~15 us of host time per spectral call."""
    global _cuda_ready
    if not _cuda_ready:
        if not torch.cuda.is_available():
            raise RuntimeError("mlx_signal_b200 needs a CUDA device (there is no CPU path)")
        torch.cuda.init()
        _cuda_ready = True
    return _get_device() if _get_device is not None else torch.cuda.current_device()


def device() -> torch.device:
    return torch.device("cuda", current_index())


def _downcast_notice(src: str) -> None:
    cfg = get_config()
    if cfg.float64 == "strict":
        raise TypeError(
            f"{src} input is not supported with float64='strict' (the kernels compute in "
            "float32). Cast to float32/complex64, or set "
            "mlx_signal_b200.set_config(float64='downcast')."
        )
    if cfg.warn_on_downcast:
        warnings.warn(
            f"{src} input downcast to 32-bit (the CUDA kernels compute in float32); "
            "results are float32-accurate",
            DowncastWarning,
            stacklevel=4,
        )


def check_dtype_policy(x) -> None:
    """Apply the float64 policy (warning or strict error) without converting."""
    if isinstance(x, torch.Tensor):
        if x.dtype == torch.float64:
            _downcast_notice("float64")
        elif x.dtype == torch.complex128:
            _downcast_notice("complex128")
    elif isinstance(x, np.ndarray):
        if x.dtype.kind == "f" and x.dtype.itemsize > 4:
            _downcast_notice(str(x.dtype))
        elif x.dtype.kind == "c" and x.dtype.itemsize > 8:
            _downcast_notice(str(x.dtype))


def _torch_to_32(t: torch.Tensor) -> torch.Tensor:
    if t.dtype in (torch.float32, torch.complex64):
        return t
    if t.dtype == torch.float64:
        _downcast_notice("float64")
        return t.to(torch.float32)
    if t.dtype == torch.complex128:
        _downcast_notice("complex128")
        return t.to(torch.complex64)
    if t.is_complex():
        return t.to(torch.complex64)
    return t.to(torch.float32)


def to_device(x) -> torch.Tensor:
    """Convert to a CUDA tensor of dtype float32 or complex64 (dtype policy applied)."""
    dev = device()
    if isinstance(x, torch.Tensor):
        t = _torch_to_32(x)
        if t.device != dev:
            t = t.to(dev, non_blocking=t.device.type == "cpu" and t.is_pinned())
        return t
    if not isinstance(x, np.ndarray):
        arr = np.asarray(x)
        if arr.dtype.kind == "c":
            arr = arr.astype(np.complex64)
        else:
            arr = arr.astype(np.float32)
        return torch.from_numpy(_c_order(arr)).to(dev)
    if x.dtype == np.float32 or x.dtype == np.complex64:
        arr = x
    elif x.dtype.kind == "f":
        if x.dtype.itemsize > 4:
            _downcast_notice(str(x.dtype))
        arr = x.astype(np.float32)
    elif x.dtype.kind == "c":
        _downcast_notice(str(x.dtype))
        arr = x.astype(np.complex64)
    elif x.dtype.kind in "iub":
        arr = x.astype(np.float32)
    else:
        raise TypeError(f"unsupported input dtype: {x.dtype}")
    return torch.from_numpy(_c_order(arr)).to(dev)


def _c_order(arr: np.ndarray) -> np.ndarray:
    """C-contiguous view or copy that keeps 0-d arrays 0-d (np.ascontiguousarray returns at least
    one dimension, which would turn a scalar input into shape (1,))."""
    return np.asarray(arr, order="C")


def to_numpy(x) -> np.ndarray:
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    return np.asarray(x)


def input_size(x) -> int:
    """Number of elements of an array-like, without converting it."""
    if isinstance(x, torch.Tensor):
        return x.numel()
    return int(np.size(x))


def input_shape(x) -> tuple[int, ...]:
    if isinstance(x, torch.Tensor):
        return tuple(x.shape)
    return tuple(np.shape(x))


def stream_handle() -> int:
    """Raw cudaStream_t of torch's current stream on the current device (read through torch's C
    extension: the same value as torch.cuda.current_stream().cuda_stream without its per-call
    availability checks)."""
    if _get_raw_stream is not None:
        return _get_raw_stream(current_index())
    return torch.cuda.current_stream(current_index()).cuda_stream
