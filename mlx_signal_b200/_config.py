"""Global configuration: dtype policy and warnings.

Mirrors the reference's ``Config`` / ``set_config`` / ``config_context``
(src/mlx_signal_processing/_config.py:42-91) for the options that change results. The
reference's size-based dispatch to scipy.signal (``dispatch``/``gpu_min_size``,
_config.py:94-100) has no counterpart: every call runs on the GPU, there is no CPU path.
``dispatch`` is still accepted for source compatibility; only "auto" and "cuda" (alias "mlx")
are valid, and both mean the CUDA kernels.
"""

from __future__ import annotations

import contextlib
import dataclasses
import warnings

__all__ = [
    "Config",
    "DowncastWarning",
    "FallbackWarning",
    "config_context",
    "get_config",
    "set_config",
]

_DISPATCH_MODES = ("auto", "cuda", "mlx")
_FLOAT64_MODES = ("downcast", "strict")


class FallbackWarning(UserWarning):
    """A call used the composed (library FFT) GPU path instead of a fused kernel."""


class DowncastWarning(UserWarning):
    """float64/complex128 input was downcast to float32/complex64."""


@dataclasses.dataclass
class Config:
    dispatch: str = "auto"
    float64: str = "downcast"  # or "strict" (raise on float64 input)
    warn_on_downcast: bool = True
    warn_on_fallback: bool = False
    #: byte budget of device-resident constant caches (windows, twiddles)
    cache_bytes: int = 64 << 20


_config = Config()


def get_config() -> Config:
    """Return a copy of the current global configuration."""
    return dataclasses.replace(_config)


def set_config(**kwargs) -> None:
    """Update configuration options (validated before anything changes)."""
    for key in kwargs:
        if not hasattr(_config, key):
            raise TypeError(f"unknown config option {key!r}")
    if kwargs.get("dispatch", _config.dispatch) not in _DISPATCH_MODES:
        raise ValueError(
            f"dispatch must be one of {_DISPATCH_MODES} (this build has no CPU/scipy path)"
        )
    if kwargs.get("float64", _config.float64) not in _FLOAT64_MODES:
        raise ValueError(f"float64 must be one of {_FLOAT64_MODES}")
    size = kwargs.get("cache_bytes", _config.cache_bytes)
    if not isinstance(size, int) or isinstance(size, bool) or size < 0:
        raise ValueError("cache_bytes must be a non-negative integer")
    for key, value in kwargs.items():
        setattr(_config, key, value)


@contextlib.contextmanager
def config_context(**kwargs):
    """Temporarily override configuration options within a ``with`` block."""
    old = dataclasses.asdict(_config)
    try:
        set_config(**kwargs)
        yield
    finally:
        _config.__dict__.update(old)


def composed_path_notice(func_name: str, reason: str) -> None:
    """Record that a call runs on the composed GPU path (cuFFT-backed) rather than a fused
    kernel. Silent unless ``warn_on_fallback`` is set."""
    if _config.warn_on_fallback:
        warnings.warn(
            f"mlx_signal_b200.{func_name}: {reason}; using the composed GPU path",
            FallbackWarning,
            stacklevel=3,
        )
