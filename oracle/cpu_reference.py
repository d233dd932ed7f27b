"""The reference's CPU route for the spectral path (test infrastructure / CPU baseline only).

mlx-signal routes work to scipy.signal on its CPU path with its own argument handling
(src/mlx_signal_processing/spectral.py:433-450 for csd/welch, 654-669 spectrogram, 714-731
stft, 842-858 istft). These functions make the same scipy calls on float32 inputs, and
`pool_map_rows` fans independent channels out over host cores with a spawn-started process
pool (safe to use after CUDA has been initialised in the parent).
"""

from __future__ import annotations

import multiprocessing as mp
import os
from functools import partial

import numpy as np
import scipy.signal as sps


def welch(x, **kw):
    """scipy.signal.welch (reference spectral.py:433-450 route via csd(x, x))."""
    return sps.welch(x, **kw)


def csd(x, y, **kw):
    return sps.csd(x, y, **kw)


def coherence(x, y, **kw):
    return sps.coherence(x, y, **kw)


def spectrogram(x, **kw):
    return sps.spectrogram(x, **kw)


def stft(x, **kw):
    return sps.stft(x, **kw)


def istft(z, **kw):
    return sps.istft(z, **kw)


def rfft(x):
    return np.fft.rfft(x)


def welch_f64(x, **kw):
    """The float64 oracle: scipy.signal.welch on the input upcast to float64 (the reference's
    tests compute their goldens this way, tests/test_spectral.py:38-47)."""
    return sps.welch(np.asarray(x, dtype=np.float64), **kw)


def _rows_task(fn_name: str, kw: dict, arrays: tuple[np.ndarray, ...]):
    fn = globals()[fn_name]
    return fn(*arrays, **kw)


_POOL = None


def pool(workers: int | None = None):
    """A persistent spawn-context process pool (one per process)."""
    global _POOL
    if _POOL is None:
        workers = workers or os.cpu_count() or 1
        _POOL = mp.get_context("spawn").Pool(workers)
    return _POOL


def close_pool():
    global _POOL
    if _POOL is not None:
        _POOL.close()
        _POOL.join()
        _POOL = None


def pool_map_rows(fn_name: str, arrays: tuple[np.ndarray, ...], workers: int, **kw):
    """Run fn over row-chunks of `arrays` (leading axis = channels) on `workers` processes and
    concatenate the last element of each result along axis 0."""
    rows = arrays[0].shape[0]
    workers = max(1, min(workers, rows))
    bounds = np.linspace(0, rows, workers + 1).astype(int)
    chunks = [tuple(a[bounds[i] : bounds[i + 1]] for a in arrays) for i in range(workers)]
    res = pool(workers).map(partial(_rows_task, fn_name, kw), chunks)
    return np.concatenate([r[-1] if isinstance(r, tuple) else r for r in res], axis=0)
