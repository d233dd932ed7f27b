"""mlx_signal_b200: B200-native (sm_100a) framed-FFT spectral path with the scipy.signal API.

Drop-in for the spectral hot path of mlx-signal (welch, csd, coherence, periodogram,
spectrogram, stft, istft). Inputs: NumPy arrays, lists or torch tensors; outputs: torch CUDA
tensors (float32 / complex64). The heavy lifting is hand-written CUDA behind a C-ABI
(include/b200signal.h, built into mlx_signal_b200/_lib/libb200signal.so).
"""

from ._config import (
    Config,
    DowncastWarning,
    FallbackWarning,
    config_context,
    get_config,
    set_config,
)
from . import fft
from .convolution import fftconvolve, oaconvolve
from .filtering import hilbert
from .resampling import resample
from .spectral import coherence, csd, istft, periodogram, spectrogram, stft, welch
from .streaming import StreamingSTFT, StreamingWelch
from .windows import get_window

__version__ = "0.1.0"

__all__ = [
    "Config",
    "DowncastWarning",
    "StreamingSTFT",
    "StreamingWelch",
    "FallbackWarning",
    "coherence",
    "config_context",
    "csd",
    "fft",
    "fftconvolve",
    "get_config",
    "get_window",
    "hilbert",
    "istft",
    "oaconvolve",
    "periodogram",
    "resample",
    "set_config",
    "spectrogram",
    "stft",
    "welch",
]
