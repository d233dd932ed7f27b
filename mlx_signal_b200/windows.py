"""Window functions: cached float64 ``scipy.signal.get_window`` values plus a device cache.

Windows are tiny and computed host-side in float64 so that scale factors (``win.sum()``,
``(win**2).sum()``) keep full precision; the scaled float32 copy the kernels read is uploaded
once per (values, device) and kept in a byte-budget LRU. Follows the reference's
src/mlx_signal_processing/windows.py:20-35 (host cache) and _cache.py:15-54 (byte budget).
"""

from __future__ import annotations

import functools
import threading
from collections import OrderedDict

import numpy as np
import torch
from scipy.signal import get_window as _sp_get_window

from ._config import get_config

__all__ = ["get_window"]


@functools.lru_cache(maxsize=256)
def _window_np(window, Nx: int, fftbins: bool = True) -> np.ndarray:
    """Cached float64 window values (hashable window spec only)."""
    w = _sp_get_window(window, Nx, fftbins=fftbins)
    w = np.ascontiguousarray(w, dtype=np.float64)
    w.setflags(write=False)
    return w


def get_window(window, Nx: int, fftbins: bool = True) -> torch.Tensor:
    """Window of a given length and type as a float32 CUDA tensor (scipy semantics)."""
    from ._array import device

    key = tuple(window) if isinstance(window, list | tuple) else window
    w = _window_np(key, int(Nx), bool(fftbins))
    return torch.from_numpy(w.astype(np.float32)).to(device())


class ByteBudgetCache:
    """LRU keyed by tuples whose total payload stays under a byte budget."""

    def __init__(self, budget_bytes: int):
        self.budget = int(budget_bytes)
        self._entries: OrderedDict[tuple, tuple[object, int]] = OrderedDict()
        self._total = 0
        self._lock = threading.Lock()

    def get(self, key: tuple):
        with self._lock:
            entry = self._entries.get(key)
            if entry is None:
                return None
            self._entries.move_to_end(key)
            return entry[0]

    def put(self, key: tuple, value, nbytes: int) -> None:
        with self._lock:
            if int(nbytes) > self.budget:
                return
            if key in self._entries:
                self._total -= self._entries.pop(key)[1]
            self._entries[key] = (value, int(nbytes))
            self._total += int(nbytes)
            while self._total > self.budget and len(self._entries) > 1:
                _, (_, freed) = self._entries.popitem(last=False)
                self._total -= freed

    def clear(self) -> None:
        with self._lock:
            self._entries.clear()
            self._total = 0

    def __len__(self) -> int:
        return len(self._entries)


DEVICE_CONSTANTS = ByteBudgetCache(get_config().cache_bytes)


def device_vector(values: np.ndarray, dtype=torch.float32) -> torch.Tensor:
    """Upload a small host vector once per (bytes, dtype, device) and cache it."""
    from ._array import device

    dev = device()
    arr = np.ascontiguousarray(values)
    key = (arr.tobytes(), str(dtype), dev.index)
    hit = DEVICE_CONSTANTS.get(key)
    if hit is not None:
        return hit
    t = torch.from_numpy(arr.copy()).to(dev, dtype=dtype)
    DEVICE_CONSTANTS.put(key, t, t.numel() * t.element_size() + len(key[0]))
    return t
