"""Global configuration: dtype policy and warnings.

The option names and exception types follow the reference's ``Config`` / ``set_config`` /
``config_context`` (src/mlx_signal_processing/_config.py:42-91) so that code written against it
keeps working. The reference's size-based dispatch to scipy.signal (``dispatch``/
``gpu_min_size``, _config.py:94-100) has no counterpart: every call runs on the GPU and there is
no CPU path. ``dispatch`` is still accepted for source compatibility; only "auto" and "cuda"
(alias "mlx") are valid, and both mean the CUDA kernels.

Design: the active configuration is one immutable ``Config`` value held in a module slot.
``set_config`` builds the whole replacement value, checks every field of it against the option
table below, and only then swaps it in, so a rejected call leaves nothing half-applied;
``config_context`` restores the exact value object it found on entry.
"""

from __future__ import annotations

import contextlib
import dataclasses
import warnings
from typing import Any, Callable

__all__ = [
    "Config",
    "DowncastWarning",
    "FallbackWarning",
    "config_context",
    "get_config",
    "set_config",
]


class FallbackWarning(UserWarning):
    """A call used the composed (library FFT) GPU path instead of a fused kernel."""


class DowncastWarning(UserWarning):
    """float64/complex128 input was downcast to float32/complex64."""


@dataclasses.dataclass(frozen=True)
class Config:
    dispatch: str = "auto"
    float64: str = "downcast"  # or "strict" (raise on float64 input)
    warn_on_downcast: bool = True
    # loud by default: a shape that leaves the fused kernels says so
    warn_on_fallback: bool = True
    #: byte budget of device-resident constant caches (windows, twiddles)
    cache_bytes: int = 64 << 20


def _one_of(*allowed: str, note: str = "") -> Callable[[str, Any], str | None]:
    def check(name: str, value: Any) -> str | None:
        if value in allowed:
            return None
        return f"{name} must be one of {allowed}{note}"

    return check


def _flag(name: str, value: Any) -> str | None:
    return None if isinstance(value, bool) else f"{name} must be True or False"


def _byte_count(name: str, value: Any) -> str | None:
    ok = isinstance(value, int) and not isinstance(value, bool) and value >= 0
    return None if ok else f"{name} must be a non-negative integer"


# option -> validator returning an error message (or None when the value is acceptable)
_CHECKS: dict[str, Callable[[str, Any], str | None]] = {
    "dispatch": _one_of("auto", "cuda", "mlx", note=" (this build has no CPU/scipy path)"),
    "float64": _one_of("downcast", "strict"),
    "warn_on_downcast": _flag,
    "warn_on_fallback": _flag,
    "cache_bytes": _byte_count,
}

_active: Config = Config()


def get_config() -> Config:
    """The configuration in force (an immutable value; change it with ``set_config``)."""
    return _active


def set_config(**kwargs) -> None:
    """Replace the named options. Unknown names raise TypeError and bad values ValueError,
    before any option changes."""
    global _active
    unknown = sorted(set(kwargs) - set(_CHECKS))
    if unknown:
        raise TypeError(f"unknown config option {unknown[0]!r}")
    candidate = dataclasses.replace(_active, **kwargs)
    for name, check in _CHECKS.items():
        problem = check(name, getattr(candidate, name))
        if problem is not None:
            raise ValueError(problem)
    _active = candidate


@contextlib.contextmanager
def config_context(**kwargs):
    """Apply ``set_config(**kwargs)`` inside a ``with`` block and put the previous
    configuration back on exit (also when the block raises)."""
    global _active
    saved = _active
    try:
        set_config(**kwargs)
        yield _active
    finally:
        _active = saved


def composed_path_notice(func_name: str, reason: str) -> None:
    """Emit a FallbackWarning (unless ``warn_on_fallback`` is off) for a call that runs on the
    composed GPU path (strided frames + torch ops + cuFFT) instead of a fused kernel."""
    if _active.warn_on_fallback:
        warnings.warn(
            f"mlx_signal_b200.{func_name}: {reason}; using the composed GPU path",
            FallbackWarning,
            stacklevel=3,
        )
