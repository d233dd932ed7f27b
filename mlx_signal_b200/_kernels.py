"""Typed launchers over the C-ABI: torch CUDA tensors in, torch CUDA tensors out.

Each launcher validates layout, allocates the output and the workspace through torch's caching
allocator, and launches on torch's current stream. This is the counterpart of the reference's
kernel-module functions (src/mlx_signal_processing/_stft_metal.py: rfft_power_mean :530,
csd_mean :739, coherence_mean :744).
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._array import stream_handle

#: largest nfft served by the fused segment kernels
MAX_FUSED_NFFT = 4096

DETREND_CODES = {False: 0, None: 0, "constant": 1, "c": 1, "linear": 2, "l": 2}


def is_pow2(v: int) -> bool:
    return v >= 1 and (v & (v - 1)) == 0


#: longest power-of-two nfft of the real-input segment-mean and per-frame kernels
MAX_FUSED_NFFT_REAL = 8192


def fused_mean_ok(nfft: int) -> bool:
    """A power-of-two nfft the real-input kernels (welch, csd, coherence, stft, spectrogram)
    compute fused."""
    return is_pow2(nfft) and nfft <= MAX_FUSED_NFFT_REAL


def fused_complex_ok(nfft: int) -> bool:
    """A power-of-two nfft the complex-input kernels compute fused."""
    return is_pow2(nfft) and nfft <= MAX_FUSED_NFFT


#: longest non-power-of-two nfft the Bluestein kernels take (welch, stft, spectrogram)
MAX_BLUE_NFFT = 4096


def blue_ok(nfft: int) -> bool:
    """A non-power-of-two nfft the Bluestein (chirp-z) kernels compute fused."""
    return not is_pow2(nfft) and 3 <= nfft <= MAX_BLUE_NFFT


def _rows(x: torch.Tensor) -> tuple[torch.Tensor, int]:
    """2-D float32 CUDA view with unit inner stride; returns (tensor, row stride)."""
    assert x.dim() == 2 and x.is_cuda and x.dtype == torch.float32
    if x.stride(1) != 1 or (x.shape[0] > 1 and x.stride(0) < x.shape[1]):
        x = x.contiguous()
    ld = x.stride(0) if x.shape[0] > 1 else x.shape[1]
    return x, max(int(ld), x.shape[1])


def _workspace(nbytes: int, dev: torch.device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=dev)


def welch_mean(x: torch.Tensor, win: torch.Tensor, nperseg: int, nfft: int, hop: int,
               detrend: int, onesided: bool, wdft: torch.Tensor | None = None,
               ws: torch.Tensor | None = None) -> torch.Tensor:
    """Mean |FFT(win * detrend(segment))|^2 over segments of each row of x -> (rows, nout).

    `wdft` (optional, complex64 CUDA): the non-zero low bins DFT_nfft(win)[0..n_low) of a window
    whose spectrum vanishes elsewhere; lets the constant detrend run as a spectral correction.
    `ws` (optional): a workspace of at least sp_mean_workspace_size bytes that no other stream
    uses meanwhile (the caller's plan keeps one per stream); allocated here when absent.
    """
    x, ld = _rows(x)
    rows, n = x.shape
    lib = _lib.load()
    if ws is None:
        ws_bytes = lib.sp_mean_workspace_size(0, rows, n, nperseg, nfft, hop, detrend)
        if ws_bytes < 0:
            _lib.check(int(ws_bytes), "sp_mean_workspace_size")
        ws = _workspace(ws_bytes, x.device)
    nout = nfft // 2 + 1 if onesided else nfft
    out = torch.empty((rows, nout), dtype=torch.float32, device=x.device)
    if wdft is not None:
        _lib.check(
            lib.sp_welch_f32_ex(x.data_ptr(), rows, n, ld, win.data_ptr(), wdft.data_ptr(),
                                wdft.numel(), nperseg, nfft, hop, detrend, int(onesided),
                                out.data_ptr(), ws.data_ptr(), ws.numel(), stream_handle()),
            "sp_welch_f32_ex",
        )
        return out
    _lib.check(
        lib.sp_welch_f32(x.data_ptr(), rows, n, ld, win.data_ptr(), nperseg, nfft, hop, detrend,
                         int(onesided), out.data_ptr(), ws.data_ptr(), ws.numel(),
                         stream_handle()),
        "sp_welch_f32",
    )
    return out


def window_low_spectrum(win32, nfft: int):
    """(DFT_nfft(win)[0..n_low) as complex64 numpy, n_low) when the window's spectrum is
    non-zero only on |k| < n_low (mod nfft) and n_low fits the kernel's spectral-detrend
    bins; else None. `win32` are the float32 window values the kernel multiplies by."""
    if not is_pow2(nfft) or nfft < 2:
        return None
    wf = np.fft.fft(np.asarray(win32, dtype=np.float64), n=nfft)
    mag = np.abs(wf)
    peak = mag.max()
    if peak == 0.0:
        return None
    k = np.nonzero(mag > 1e-7 * peak)[0]
    n_low = int(np.max(np.minimum(k, nfft - k))) + 1
    if n_low > _lib.load().sp_welch_spectral_bins(nfft):
        return None
    return wf[:n_low].astype(np.complex64), n_low


def cross_mean(mode: str, x: torch.Tensor, y: torch.Tensor, win: torch.Tensor, nperseg: int,
               nfft: int, hop: int, detrend: int, onesided: bool = True,
               wdft: torch.Tensor | None = None) -> torch.Tensor:
    """mode 'csd': mean conj(X)Y (complex64, one-sided doubling if requested);
    mode 'coherence': |Pxy|^2/(Pxx Pyy) (float32). `wdft`: as for welch_mean (constant detrend
    as a spectral correction in the 50%-overlap kernels)."""
    x, ldx = _rows(x)
    y, ldy = _rows(y)
    assert x.shape == y.shape
    rows, n = x.shape
    lib = _lib.load()
    ws_bytes = lib.sp_mean_workspace_size(1, rows, n, nperseg, nfft, hop, detrend)
    if ws_bytes < 0:
        _lib.check(int(ws_bytes), "sp_mean_workspace_size")
    ws = _workspace(ws_bytes, x.device)
    if mode == "csd":
        nout = nfft // 2 + 1 if onesided else nfft
        out = torch.empty((rows, nout), dtype=torch.complex64, device=x.device)
        if wdft is not None:
            _lib.check(
                lib.sp_csd_c64_ex(x.data_ptr(), y.data_ptr(), rows, n, ldx, ldy, win.data_ptr(),
                                  wdft.data_ptr(), wdft.numel(), nperseg, nfft, hop, detrend,
                                  int(onesided), out.data_ptr(), ws.data_ptr(), ws.numel(),
                                  stream_handle()),
                "sp_csd_c64_ex",
            )
            return out
        _lib.check(
            lib.sp_csd_c64(x.data_ptr(), y.data_ptr(), rows, n, ldx, ldy, win.data_ptr(),
                           nperseg, nfft, hop, detrend, int(onesided), out.data_ptr(),
                           ws.data_ptr(), ws.numel(), stream_handle()),
            "sp_csd_c64",
        )
        return out
    if mode == "coherence":
        out = torch.empty((rows, nfft // 2 + 1), dtype=torch.float32, device=x.device)
        if wdft is not None:
            _lib.check(
                lib.sp_coherence_f32_ex(x.data_ptr(), y.data_ptr(), rows, n, ldx, ldy,
                                        win.data_ptr(), wdft.data_ptr(), wdft.numel(), nperseg,
                                        nfft, hop, detrend, out.data_ptr(), ws.data_ptr(),
                                        ws.numel(), stream_handle()),
                "sp_coherence_f32_ex",
            )
            return out
        _lib.check(
            lib.sp_coherence_f32(x.data_ptr(), y.data_ptr(), rows, n, ldx, ldy, win.data_ptr(),
                                 nperseg, nfft, hop, detrend, out.data_ptr(), ws.data_ptr(),
                                 ws.numel(), stream_handle()),
            "sp_coherence_f32",
        )
        return out
    raise ValueError(mode)


EXT_CODES = {None: 0, "zeros": 1, "even": 2, "odd": 3, "constant": 4}


def frames(kind: str, x: torch.Tensor, win: torch.Tensor, nperseg: int, nfft: int, hop: int,
           detrend: int, onesided: bool, ext: int = 0, ext_mode=None, n_total: int | None = None,
           y: torch.Tensor | None = None, wdft: torch.Tensor | None = None) -> torch.Tensor:
    """Per-frame spectra of each row: (rows, nseg, nbins).

    kind 'stft' -> complex64 X_s; 'power' -> float32 |X_s|^2 with one-sided doubling;
    'cross' -> complex64 conj(X_s) Y_s (no doubling). Boundary extension (`ext` samples per
    side, scipy `boundary` mode `ext_mode`) and zero padding up to `n_total` are virtual.
    `wdft` (optional, complex64 CUDA, DFT_nfft(win) low bins): with detrend 1 (constant) the mean
    is removed as a spectral correction after the transform (stft / power only).
    """
    x, ldx = _rows(x)
    rows, n = x.shape
    n_total = n + 2 * ext if n_total is None else int(n_total)
    nseg = (n_total - nperseg) // hop + 1
    nbins = nfft // 2 + 1 if onesided else nfft
    lib = _lib.load()
    spec = wdft is not None and detrend == 1 and kind in ("power", "stft")
    if kind == "power":
        out = torch.empty((rows, nseg, nbins), dtype=torch.float32, device=x.device)
        if spec:
            _lib.check(lib.sp_spectrogram_f32_ex(x.data_ptr(), rows, n, ldx, ext,
                                                 EXT_CODES[ext_mode], n_total, win.data_ptr(),
                                                 wdft.data_ptr(), wdft.numel(), nperseg, nfft, hop,
                                                 detrend, int(onesided), out.data_ptr(),
                                                 stream_handle()),
                       "sp_spectrogram_f32_ex")
            return out
        _lib.check(lib.sp_spectrogram_f32(x.data_ptr(), rows, n, ldx, ext, EXT_CODES[ext_mode],
                                          n_total, win.data_ptr(), nperseg, nfft, hop, detrend,
                                          int(onesided), out.data_ptr(), stream_handle()),
                   "sp_spectrogram_f32")
        return out
    out = torch.empty((rows, nseg, nbins), dtype=torch.complex64, device=x.device)
    if kind == "stft" and spec:
        _lib.check(lib.sp_stft_c64_ex(x.data_ptr(), rows, n, ldx, ext, EXT_CODES[ext_mode],
                                      n_total, win.data_ptr(), wdft.data_ptr(), wdft.numel(),
                                      nperseg, nfft, hop, detrend, int(onesided), out.data_ptr(),
                                      stream_handle()),
                   "sp_stft_c64_ex")
        return out
    if kind == "stft":
        _lib.check(lib.sp_stft_c64(x.data_ptr(), rows, n, ldx, ext, EXT_CODES[ext_mode], n_total,
                                   win.data_ptr(), nperseg, nfft, hop, detrend, int(onesided),
                                   out.data_ptr(), stream_handle()),
                   "sp_stft_c64")
        return out
    if kind == "cross":
        assert y is not None and ext == 0 and n_total == n
        y, ldy = _rows(y)
        _lib.check(lib.sp_csd_frames_c64(x.data_ptr(), y.data_ptr(), rows, n, ldx, ldy,
                                         win.data_ptr(), nperseg, nfft, hop, detrend,
                                         int(onesided), out.data_ptr(), stream_handle()),
                   "sp_csd_frames_c64")
        return out
    raise ValueError(kind)


def istft_fused(z: torch.Tensor, win: torch.Tensor, scale: float, nperseg: int, hop: int,
                nfft: int | None = None, onesided: bool = True) -> torch.Tensor:
    """Fused inverse STFT of (rows, nseg, nf) complex64 spectra (bins contiguous): inverse FFT of
    length nfft (default nperseg) per frame -- irfft of one-sided spectra, ifft of two-sided
    ones -- its first nperseg samples times win * scale, overlap-add and division by the window
    energy (where it exceeds 1e-10) in one kernel -> (rows, nperseg + (nseg-1)*hop) float32, or
    complex64 for two-sided input."""
    assert z.is_cuda and z.dtype == torch.complex64 and z.dim() == 3
    if z.stride(2) != 1 or z.stride(1) < z.shape[2] or z.stride(0) < z.shape[1] * z.stride(1):
        z = z.contiguous()
    nfft = nperseg if nfft is None else int(nfft)
    rows, nseg, nf = z.shape
    outlen = nperseg + (nseg - 1) * hop
    ld_row = z.stride(0) if rows > 1 else nseg * z.stride(1)
    lib = _lib.load()
    if onesided:
        out = torch.empty((rows, outlen), dtype=torch.float32, device=z.device)
        _lib.check(
            lib.sp_istft_f32_ex(z.data_ptr(), rows, nseg, ld_row, z.stride(1), nf,
                                win.data_ptr(), float(scale), nperseg, nfft, hop, out.data_ptr(),
                                stream_handle()),
            "sp_istft_f32_ex",
        )
        return out
    out = torch.empty((rows, outlen), dtype=torch.complex64, device=z.device)
    _lib.check(
        lib.sp_istft_c64(z.data_ptr(), rows, nseg, ld_row, z.stride(1), min(nf, nfft),
                         win.data_ptr(), float(scale), nperseg, nfft, hop, out.data_ptr(),
                         stream_handle()),
        "sp_istft_c64",
    )
    return out


#: longest filter the fused overlap-save convolution takes
CONV_MAX_TAPS = 2049


def conv_ols(x: torch.Tensor, h: torch.Tensor, j0: int, nout: int) -> torch.Tensor:
    """Full linear convolution window [j0, j0 + nout) of every row of x (rows, n1) float32 CUDA
    with one real filter h (n2 <= CONV_MAX_TAPS taps) -> (rows, nout) float32, in one fused
    overlap-save kernel."""
    x, ld = _rows(x)
    rows, n1 = x.shape
    h = h.reshape(-1)
    assert h.is_cuda and h.dtype == torch.float32
    h = h.contiguous()
    out = torch.empty((rows, nout), dtype=torch.float32, device=x.device)
    _lib.check(
        _lib.load().sp_conv_ols_f32(x.data_ptr(), rows, n1, ld, h.data_ptr(), h.numel(), int(j0),
                                    int(nout), out.data_ptr(), max(int(nout), 1),
                                    stream_handle()),
        "sp_conv_ols_f32",
    )
    return out


def _rows_c(x: torch.Tensor) -> tuple[torch.Tensor, int]:
    """2-D complex64 CUDA view with unit inner stride; returns (tensor, row stride in complex
    elements)."""
    assert x.dim() == 2 and x.is_cuda and x.dtype == torch.complex64
    if x.stride(1) != 1 or (x.shape[0] > 1 and x.stride(0) < x.shape[1]):
        x = x.contiguous()
    ld = x.stride(0) if x.shape[0] > 1 else x.shape[1]
    return x, max(int(ld), x.shape[1])


def welch_mean_complex(x: torch.Tensor, win: torch.Tensor, nperseg: int, nfft: int, hop: int,
                       detrend: int) -> torch.Tensor:
    """Two-sided mean |FFT(win * detrend(segment))|^2 over the segments of each complex row of x
    -> (rows, nfft) float32 (power-of-two nfft)."""
    x, ld = _rows_c(x)
    rows, n = x.shape
    lib = _lib.load()
    ws_bytes = lib.sp_mean_workspace_size(3, rows, n, nperseg, nfft, hop, detrend)
    if ws_bytes < 0:
        _lib.check(int(ws_bytes), "sp_mean_workspace_size")
    out = torch.empty((rows, nfft), dtype=torch.float32, device=x.device)
    ws = _workspace(ws_bytes, x.device)
    _lib.check(lib.sp_welch_c64(x.data_ptr(), rows, n, ld, win.data_ptr(), nperseg, nfft, hop,
                                detrend, out.data_ptr(), ws.data_ptr(), ws.numel(),
                                stream_handle()), "sp_welch_c64")
    return out


def frames_complex(kind: str, x: torch.Tensor, win: torch.Tensor, nperseg: int, nfft: int,
                   hop: int, detrend: int, ext: int = 0, ext_mode=None,
                   n_total: int | None = None) -> torch.Tensor:
    """Per-frame two-sided spectra of complex rows: (rows, nseg, nfft) complex64 ('stft') or
    float32 |X|^2 ('power'); boundary extension and padding virtual, as in `frames`."""
    x, ld = _rows_c(x)
    rows, n = x.shape
    n_total = n + 2 * ext if n_total is None else int(n_total)
    nseg = (n_total - nperseg) // hop + 1
    power = kind == "power"
    out = torch.empty((rows, nseg, nfft), dtype=torch.float32 if power else torch.complex64,
                      device=x.device)
    _lib.check(_lib.load().sp_frames_cplx(x.data_ptr(), rows, n, ld, ext, EXT_CODES[ext_mode],
                                          n_total, win.data_ptr(), nperseg, nfft, hop, detrend,
                                          int(power), out.data_ptr(), stream_handle()),
               "sp_frames_cplx")
    return out


def median_segments(per: torch.Tensor, scale: float) -> torch.Tensor | None:
    """Median over the segment axis of per-frame spectra per (..., nseg, nfreq) (float32, or
    complex64: real and imaginary parts separately), times `scale` -> (..., nfreq); None when
    nseg exceeds the kernel's staged maximum (the caller sorts instead)."""
    cplx = per.is_complex()
    lead = tuple(per.shape[:-2])
    nseg, nf = per.shape[-2], per.shape[-1]
    p = torch.view_as_real(per).flatten(-2) if cplx else per
    rows = int(np.prod(lead)) if lead else 1
    ncols = p.shape[-1]
    p = p.reshape(rows, nseg, ncols)
    # the kernel reads frame s of row r at (r * nseg + s) * stride(1)
    if p.stride(2) != 1 or p.stride(1) < ncols or (rows > 1 and p.stride(0) != nseg * p.stride(1)):
        p = p.contiguous()
    out = torch.empty((rows, ncols), dtype=torch.float32, device=per.device)
    st = _lib.load().sp_median_frames_f32(p.data_ptr(), rows, nseg, ncols, p.stride(1),
                                          float(scale), out.data_ptr(), stream_handle())
    if st == _lib.SP_ERR_UNSUPPORTED:
        return None
    _lib.check(st, "sp_median_frames_f32")
    if cplx:
        out = torch.view_as_complex(out.reshape(rows, nf, 2))
    return out.reshape(lead + (nf,))


def csd_complex(x: torch.Tensor, y: torch.Tensor, win: torch.Tensor, nperseg: int, nfft: int,
                hop: int, detrend: int) -> torch.Tensor:
    """Two-sided mean conj(X) Y over the segments of complex rows x, y -> (rows, nfft) complex64
    (power-of-two nfft)."""
    x, ldx = _rows_c(x)
    y, ldy = _rows_c(y)
    rows, n = x.shape
    lib = _lib.load()
    ws_bytes = lib.sp_mean_workspace_size(4, rows, n, nperseg, nfft, hop, detrend)
    if ws_bytes < 0:
        _lib.check(int(ws_bytes), "sp_mean_workspace_size")
    out = torch.empty((rows, nfft), dtype=torch.complex64, device=x.device)
    ws = _workspace(ws_bytes, x.device)
    _lib.check(lib.sp_csd_cplx(x.data_ptr(), y.data_ptr(), rows, n, ldx, ldy, win.data_ptr(),
                               nperseg, nfft, hop, detrend, out.data_ptr(), ws.data_ptr(),
                               ws.numel(), stream_handle()), "sp_csd_cplx")
    return out


def dft32_tc(z: torch.Tensor, reps: int = 1, err: torch.Tensor | None = None) -> torch.Tensor:
    """32-point complex DFTs of the last axis of z (complex64 CUDA, last dimension 32) on the
    tensor cores (sp_dft32_tc_c64: FP16 head/tail splits, three products, FP32 accumulation).
    `reps` repeats the MMA chain on the staged operands (rate measurement; same result). `err`:
    optional int32 CUDA tensor of one element that receives SP_ERR_TIMEOUT if the bounded wait
    for the MMAs runs out."""
    if z.dtype != torch.complex64 or not z.is_cuda or z.shape[-1] != 32:
        raise ValueError("dft32_tc: complex64 CUDA tensor with a last dimension of 32")
    zc = z.reshape(-1, 32).contiguous()
    out = torch.empty_like(zc)
    lib = _lib.load()
    _lib.check(lib.sp_dft32_tc_c64(zc.data_ptr(), out.data_ptr(), zc.shape[0], int(reps),
                                   None if err is None else err.data_ptr(), stream_handle()),
               "sp_dft32_tc_c64")
    return out.reshape(z.shape)
