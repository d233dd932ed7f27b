"""ctypes binding of libb200signal.so (declared in include/b200signal.h).

The library is built in-tree by ``python -m mlx_signal_b200.csrc.build`` (or
``__graft_entry__.build()``). There is no fallback: if the library is missing, every spectral
call raises :class:`ExtensionMissing`.
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libb200signal.so"

c_i = ctypes.c_int
c_i64 = ctypes.c_int64
c_sz = ctypes.c_size_t
c_p = ctypes.c_void_p
c_fp = ctypes.c_void_p  # float* / const float* (device pointers as integers)

#: C-ABI symbol table: name -> (restype, argtypes). Kept in step with include/b200signal.h;
#: tests/test_capi_symbols.py checks both directions.
SIGNATURES: dict[str, tuple[object, list[object]]] = {
    "sp_version": (c_i, []),
    "sp_last_error": (ctypes.c_char_p, []),
    "sp_mean_workspace_size": (c_i64, [c_i, c_i64, c_i64, c_i, c_i, c_i, c_i]),
    "sp_welch_f32": (
        c_i,
        [c_fp, c_i64, c_i64, c_i64, c_fp, c_i, c_i, c_i, c_i, c_i, c_fp, c_p, c_sz, c_p],
    ),
    "sp_welch_f32_ex": (
        c_i,
        [c_fp, c_i64, c_i64, c_i64, c_fp, c_fp, c_i, c_i, c_i, c_i, c_i, c_i, c_fp, c_p, c_sz,
         c_p],
    ),
    "sp_welch_spectral_bins": (c_i, [c_i]),
    "sp_welch_c64": (
        c_i,
        [c_fp, c_i64, c_i64, c_i64, c_fp, c_i, c_i, c_i, c_i, c_fp, c_p, c_sz, c_p],
    ),
    "sp_csd_cplx": (
        c_i,
        [c_fp, c_fp, c_i64, c_i64, c_i64, c_i64, c_fp, c_i, c_i, c_i, c_i, c_fp, c_p, c_sz, c_p],
    ),
    "sp_frames_cplx": (
        c_i,
        [c_fp, c_i64, c_i64, c_i64, c_i, c_i, c_i64, c_fp, c_i, c_i, c_i, c_i, c_i, c_fp, c_p],
    ),
    "sp_welch_f32_noalloc": (
        c_i,
        [c_fp, c_i64, c_i64, c_i64, c_fp, c_i, c_i, c_i, c_i, c_i, c_fp, c_p],
    ),
    "sp_csd_c64": (
        c_i,
        [c_fp, c_fp, c_i64, c_i64, c_i64, c_i64, c_fp, c_i, c_i, c_i, c_i, c_i, c_fp, c_p, c_sz, c_p],
    ),
    "sp_coherence_f32": (
        c_i,
        [c_fp, c_fp, c_i64, c_i64, c_i64, c_i64, c_fp, c_i, c_i, c_i, c_i, c_fp, c_p, c_sz, c_p],
    ),
    "sp_csd_c64_ex": (
        c_i,
        [c_fp, c_fp, c_i64, c_i64, c_i64, c_i64, c_fp, c_fp, c_i, c_i, c_i, c_i, c_i, c_i, c_fp,
         c_p, c_sz, c_p],
    ),
    "sp_coherence_f32_ex": (
        c_i,
        [c_fp, c_fp, c_i64, c_i64, c_i64, c_i64, c_fp, c_fp, c_i, c_i, c_i, c_i, c_i, c_fp, c_p,
         c_sz, c_p],
    ),
    "sp_stft_c64": (
        c_i,
        [c_fp, c_i64, c_i64, c_i64, c_i, c_i, c_i64, c_fp, c_i, c_i, c_i, c_i, c_i, c_fp, c_p],
    ),
    "sp_spectrogram_f32": (
        c_i,
        [c_fp, c_i64, c_i64, c_i64, c_i, c_i, c_i64, c_fp, c_i, c_i, c_i, c_i, c_i, c_fp, c_p],
    ),
    "sp_stft_c64_ex": (
        c_i,
        [c_fp, c_i64, c_i64, c_i64, c_i, c_i, c_i64, c_fp, c_fp, c_i, c_i, c_i, c_i, c_i, c_i,
         c_fp, c_p],
    ),
    "sp_spectrogram_f32_ex": (
        c_i,
        [c_fp, c_i64, c_i64, c_i64, c_i, c_i, c_i64, c_fp, c_fp, c_i, c_i, c_i, c_i, c_i, c_i,
         c_fp, c_p],
    ),
    "sp_csd_frames_c64": (
        c_i,
        [c_fp, c_fp, c_i64, c_i64, c_i64, c_i64, c_fp, c_i, c_i, c_i, c_i, c_i, c_fp, c_p],
    ),
    "sp_istft_f32": (
        c_i,
        [c_fp, c_i64, c_i, c_i64, c_i, c_i, c_fp, ctypes.c_float, c_i, c_i, c_fp, c_p],
    ),
    "sp_istft_f32_ex": (
        c_i,
        [c_fp, c_i64, c_i, c_i64, c_i, c_i, c_fp, ctypes.c_float, c_i, c_i, c_i, c_fp, c_p],
    ),
    "sp_istft_c64": (
        c_i,
        [c_fp, c_i64, c_i, c_i64, c_i, c_i, c_fp, ctypes.c_float, c_i, c_i, c_i, c_fp, c_p],
    ),
    "sp_fft_workspace_size": (c_i64, [c_i64, c_i]),
    "sp_fft_c64": (c_i, [c_fp, c_fp, c_i, c_i64, c_i, c_p, c_sz, c_p]),
    "sp_rfft_c64": (c_i, [c_fp, c_fp, c_i, c_i64, c_i64, c_p, c_sz, c_p]),
    "sp_irfft_f32": (c_i, [c_fp, c_i64, c_i, c_fp, c_i, c_i64, c_p, c_sz, c_p]),
    "sp_resample_workspace_size": (c_i64, [c_i64, c_i64, c_i]),
    "sp_fft_sticky_error": (c_i, [c_i]),
    "sp_resample_f32": (c_i, [c_fp, c_i, c_i64, c_fp, c_i64, c_p, c_sz, c_p]),
    "sp_fft_error_word": (c_i, [c_p, c_i64, c_i, ctypes.POINTER(c_i64)]),
    "sp_fft_set_wait_limit": (ctypes.c_uint32, [ctypes.c_uint32]),
    "sp_hilbert_c64": (c_i, [c_fp, c_fp, c_i, c_i64, c_p, c_sz, c_p]),
    "sp_dft32_tc_c64": (c_i, [c_fp, c_fp, c_i64, c_i, c_p, c_p]),
    "sp_conv_ols_f32": (c_i, [c_fp, c_i64, c_i64, c_i64, c_fp, c_i, c_i64, c_i64, c_fp, c_i64,
                              c_p]),
    "sp_conv_block_len": (c_i, [c_i]),
    "sp_median_frames_f32": (c_i, [c_fp, c_i64, c_i, c_i, c_i64, ctypes.c_float, c_fp, c_p]),
    "sp_batch_stream_frames": (c_i64, [c_i64, c_i64, c_i, c_i, ctypes.POINTER(c_i64)]),
    "sp_batch_supported": (c_i, [c_i]),
    "sp_batch_plan": (c_i, [c_p, c_i, ctypes.POINTER(c_i64), ctypes.POINTER(c_i64)]),
    "sp_batch_encode": (c_i, [c_p, c_i, c_p, c_sz, c_p, c_sz]),
    "sp_batch_max_grid": (c_i, []),
    "sp_batch_run": (c_i, [c_p, c_p, c_i, c_p]),
}

SP_OK = 0
SP_ERR_ARG = -1
SP_ERR_UNSUPPORTED = -2
SP_ERR_WORKSPACE = -3
SP_ERR_CUDA = -4
SP_ERR_TIMEOUT = -5


class ExtensionMissing(ImportError):
    """libb200signal.so is not built (no CPU fallback exists)."""


class KernelError(RuntimeError):
    """A C-ABI call returned an error status."""

    def __init__(self, what: str, status: int, text: str):
        super().__init__(f"{what} failed with status {status}: {text}")
        self.status = status


class Unsupported(KernelError):
    """The fused kernels do not cover this shape (SP_ERR_UNSUPPORTED)."""


_lock = threading.Lock()
_lib: ctypes.CDLL | None = None


def load() -> ctypes.CDLL:
    """Load (once) and return the bound library."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise ExtensionMissing(
                    f"{LIB_PATH} is not built; run `python -m mlx_signal_b200.csrc.build`"
                )
            lib = ctypes.CDLL(str(LIB_PATH))
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def last_error() -> str:
    return load().sp_last_error().decode(errors="replace")


def check(status: int, what: str) -> None:
    if status == SP_OK:
        return
    text = last_error()
    if status == SP_ERR_UNSUPPORTED:
        raise Unsupported(what, status, text)
    raise KernelError(what, status, text)


def call(name: str, *args):
    """Call a C-ABI entry point and raise on a non-zero status."""
    fn = getattr(load(), name)
    check(fn(*args), name)
