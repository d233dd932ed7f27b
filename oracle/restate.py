"""NumPy restatement of the reference's spectral kernels (test infrastructure only).

Each function follows one piece of mlx-signal's GPU algorithm step by step, in float64 unless a
dtype is given, so tests can check (a) that the reference's algorithm equals float64 scipy
(pinning scipy as the parity oracle for it) and (b) intermediate-stage identities the CUDA
kernels rely on. Citations are into the reference tree.
"""

from __future__ import annotations

import numpy as np


# ---------------------------------------------------------------------------------------------
# framed packed-real FFT (src/mlx_signal_processing/_stft_metal.py:33-147, 182-189)
# ---------------------------------------------------------------------------------------------


def tables(N: int, dtype=np.complex128):
    """(tw, ut): Stockham twiddles exp(-2 pi i j / M), j < M/2, and untangle twiddles
    exp(-i pi k / M), k <= M, with M = N/2 (_stft_metal.py:182-189)."""
    M = N // 2
    tw = np.exp(-2j * np.pi * np.arange(max(M // 2, 1)) / M).astype(dtype)
    ut = np.exp(-1j * np.pi * np.arange(M + 1) / M).astype(dtype)
    return tw, ut


def load_segments(x: np.ndarray, nperseg: int, hop: int, win: np.ndarray, detrend) -> np.ndarray:
    """Strided segment load, optional mean detrend, window (_stft_metal.py:33-61):
    (rows, n) -> (rows, nseg, nperseg)."""
    n = x.shape[-1]
    nseg = (n - nperseg) // hop + 1
    idx = np.arange(nperseg)[None, :] + hop * np.arange(nseg)[:, None]
    seg = x[..., idx]
    if detrend in ("constant", "c"):
        seg = seg - seg.mean(axis=-1, keepdims=True)
    return seg * win


def stockham(buf: np.ndarray, tw: np.ndarray) -> np.ndarray:
    """Radix-2 Stockham over the last axis exactly as _stft_metal.py:124-144: per stage,
    B[k + 2jm] = c0 + c1, B[k + 2jm + m] = tw[j*stride] * (c0 - c1)."""
    M = buf.shape[-1]
    if M == 1:
        return buf.copy()
    S = int(np.log2(M))
    A = buf.copy()
    l, stride, m = M // 2, 1, 1
    p = np.arange(M // 2)
    for _ in range(S):
        j = p // m
        k = p - j * m
        c0 = A[..., k + j * m]
        c1 = A[..., k + j * m + l * m]
        B = np.empty_like(A)
        B[..., k + 2 * j * m] = c0 + c1
        B[..., k + 2 * j * m + m] = tw[j * stride] * (c0 - c1)
        A = B
        l >>= 1
        stride <<= 1
        m <<= 1
    return A


def untangle(Z: np.ndarray, ut: np.ndarray) -> np.ndarray:
    """rfft bins 0..M of the packed even/odd FFT Z (_stft_metal.py:85-101)."""
    M = Z.shape[-1]
    k = np.arange(1, M)
    zk = Z[..., k]
    zmk = Z[..., M - k]
    ze = 0.5 * (zk.real + zmk.real) + 0.5j * (zk.imag - zmk.imag)
    zo = 0.5 * (zk.real - zmk.real) + 0.5j * (zk.imag + zmk.imag)
    wzo = ut[k] * zo
    mid = (ze.real + wzo.imag) + 1j * (ze.imag - wzo.real)
    z0 = Z[..., :1]
    first = (z0.real + z0.imag) + 0j
    last = (z0.real - z0.imag) + 0j
    return np.concatenate([first, mid, last], axis=-1)


def rfft_frames(x: np.ndarray, win: np.ndarray, nperseg: int, hop: int, detrend,
                power: bool = False) -> np.ndarray:
    """_stft_metal.rfft_frames (_stft_metal.py:192-220): (rows, nseg, nperseg/2+1)."""
    seg = load_segments(np.asarray(x, dtype=np.float64), nperseg, hop,
                        np.asarray(win, dtype=np.float64), detrend)
    packed = seg[..., 0::2] + 1j * seg[..., 1::2]
    tw, ut = tables(nperseg)
    X = untangle(stockham(packed, tw), ut)
    return np.abs(X) ** 2 if power else X


# ---------------------------------------------------------------------------------------------
# grouped segment means (_stft_metal.py:426-557, 620-746)
# ---------------------------------------------------------------------------------------------

MEAN_TARGET_GROUPS = 2048
MEAN_MAX_GROUP = 64


def group_params(B: int, nseg: int) -> tuple[int, int]:
    """(group_size, ngroups) of _stft_metal._group_params (:433-440)."""
    if nseg <= 1:
        return 1, nseg
    target_per_row = max(1, -(-MEAN_TARGET_GROUPS // max(1, B)))
    group_size = min(nseg, MEAN_MAX_GROUP, max(1, -(-nseg // target_per_row)))
    return group_size, -(-nseg // group_size)


def _grouped_mean(per: np.ndarray) -> np.ndarray:
    """Group partial sums then their sum, times 1/nseg (_reduce_groups :443-455)."""
    B = int(np.prod(per.shape[:-2])) if per.ndim > 2 else 1
    nseg = per.shape[-2]
    gs, ng = group_params(B, nseg)
    parts = [per[..., g * gs : min(nseg, (g + 1) * gs), :].sum(axis=-2) for g in range(ng)]
    total = np.sum(parts, axis=0)
    return total / nseg if nseg > 1 else total


def rfft_power_mean(x, win, nperseg, hop, detrend):
    """_stft_metal.rfft_power_mean (:530-557): mean |X|^2 over segments (no one-sided factor)."""
    return _grouped_mean(rfft_frames(x, win, nperseg, hop, detrend, power=True))


def pair_means(x, y, win, nperseg, hop, detrend):
    """_stft_metal.coherence_mean / csd_mean (:703-746): (Pxx, Pyy, Pxy) segment means."""
    X = rfft_frames(x, win, nperseg, hop, detrend)
    Y = rfft_frames(y, win, nperseg, hop, detrend)
    return (_grouped_mean(np.abs(X) ** 2), _grouped_mean(np.abs(Y) ** 2),
            _grouped_mean(np.conj(X) * Y))


def onesided_factor(nfft: int) -> np.ndarray:
    """spectral._onesided_factor (spectral.py:150-157)."""
    f = np.full(nfft // 2 + 1, 2.0)
    f[0] = 1.0
    if nfft % 2 == 0:
        f[-1] = 1.0
    return f


def welch(x, fs, win_np, nperseg, noverlap, detrend="constant", scaling="density"):
    """The reference's fused welch route (spectral.py:305-353 + 468-488): sqrt(scale) folded
    into the window, grouped power mean, deferred one-sided factor."""
    scale = (1.0 / (fs * (win_np * win_np).sum()) if scaling == "density"
             else 1.0 / win_np.sum() ** 2)
    w = win_np * np.sqrt(scale)
    p = rfft_power_mean(x, w, nperseg, nperseg - noverlap, detrend)
    return p * onesided_factor(nperseg)


def csd(x, y, fs, win_np, nperseg, noverlap, detrend="constant"):
    scale = 1.0 / (fs * (win_np * win_np).sum())
    w = win_np * np.sqrt(scale)
    _, _, pxy = pair_means(x, y, w, nperseg, nperseg - noverlap, detrend)
    return pxy * onesided_factor(nperseg)


def coherence(x, y, win_np, nperseg, noverlap, detrend="constant"):
    """Fast-path coherence (spectral.py:591-617): raw window, |Pxy|^2 / Pxx / Pyy."""
    pxx, pyy, pxy = pair_means(x, y, win_np, nperseg, nperseg - noverlap, detrend)
    return np.abs(pxy) ** 2 / pxx / pyy


# ---------------------------------------------------------------------------------------------
# istft: inverse repack + FFT-as-inverse + gather overlap-add (_stft_metal.py:753-887)
# ---------------------------------------------------------------------------------------------


def istft_frames(z3: np.ndarray, win_np: np.ndarray, scale: float, nperseg: int, hop: int):
    """(..., nseg, M+1) one-sided spectra -> ((..., outlen) signal divided by the window-power
    norm, norm). Follows _ISTFT_SRC (:753-795) and _OLA_SRC (:797-820)."""
    M = nperseg // 2
    z3 = np.asarray(z3, dtype=np.complex128)
    nseg = z3.shape[-2]
    Xk = z3[..., :M].copy()
    Xmk = z3[..., M:0:-1].copy()  # X[M-k] for k = 0..M-1
    Xk[..., 0] = Xk[..., 0].real
    Xmk[..., 0] = Xmk[..., 0].real
    E = 0.5 * (Xk.real + Xmk.real) + 0.5j * (Xk.imag - Xmk.imag)
    wO = 0.5 * (Xk.real - Xmk.real) + 0.5j * (Xk.imag + Xmk.imag)
    _, ut = tables(nperseg)
    O = np.conj(ut[:M]) * wO
    buf = (E.real - O.imag) - 1j * (E.imag + O.real)  # conj(E + i O)
    tw, _ = tables(nperseg)
    Z = stockham(buf, tw)
    wineff = np.asarray(win_np, dtype=np.float64) * (scale / M)
    frames = np.empty(z3.shape[:-1] + (nperseg,))
    frames[..., 0::2] = Z.real * wineff[0::2]
    frames[..., 1::2] = -Z.imag * wineff[1::2]
    outlen = nperseg + (nseg - 1) * hop
    out = np.zeros(z3.shape[:-2] + (outlen,))
    norm = np.zeros(outlen)
    w2 = np.asarray(win_np, dtype=np.float64) ** 2
    for s in range(nseg):
        out[..., s * hop : s * hop + nperseg] += frames[..., s, :]
        norm[s * hop : s * hop + nperseg] += w2
    out = out / np.where(norm > 1e-10, norm, 1.0)
    return out, norm


# ---------------------------------------------------------------------------------------------
# three-pass large FFT (_fourstep_metal.py:15-26, 90-185, 206-215) and real transforms
# (_fourstep.py:195-231, 360-408)
# ---------------------------------------------------------------------------------------------


def digits(n: int) -> tuple[int, int, int]:
    """(R3, R2, R1) of _fourstep_metal._digits (:206-215)."""
    e = n.bit_length() - 1
    if e == 21:
        return (128, 128, 128)
    return (1 << (e - 16), 256, 256)


def fft3(a: np.ndarray, inverse: bool = False, split=None) -> np.ndarray:
    """Three-pass Bailey FFT along the last axis with the reference's index maps:
    x[m3][m2][r] -> S1[m2][r][km3] -> S2[km2][r][km3] -> out[kr][km2][km3]."""
    a = np.asarray(a, dtype=np.complex128)
    n = a.shape[-1]
    R3, R2, R1 = split or digits(n)
    N, M = n, R2 * R3
    sign = 1.0 if inverse else -1.0
    if inverse:
        def dft(v, ax):
            return np.fft.ifft(v, axis=ax) * v.shape[ax]
    else:
        def dft(v, ax):
            return np.fft.fft(v, axis=ax)
    x = a.reshape(a.shape[:-1] + (R3, R2, R1))
    # pass 1: DFT over m3 -> km3, twiddle W_M^(m2 km3), layout S1[m2][r][km3]
    y = dft(x, -3)  # (..., km3, m2, r)
    km3 = np.arange(R3)[:, None, None]
    m2 = np.arange(R2)[None, :, None]
    ph = (m2 * km3) % M
    y = y * np.exp(sign * 2j * np.pi * ph / M)
    if inverse:
        y = y / N
    s1 = np.moveaxis(y, -3, -1)  # (..., m2, r, km3)
    # pass 2: DFT over m2 -> km2, twiddle W_N^(r (km2 R3 + km3)), layout S2[km2][r][km3]
    y = dft(s1, -3)  # (..., km2, r, km3)
    km2 = np.arange(R2)[:, None, None]
    r = np.arange(R1)[None, :, None]
    k3 = np.arange(R3)[None, None, :]
    ph = (r * (km2 * R3 + k3)) % N
    s2 = y * np.exp(sign * 2j * np.pi * ph / N)
    # pass 3: DFT over r -> kr, out[kr][km2][km3]
    y = dft(s2, -2)  # (..., km2, kr, km3)
    return np.moveaxis(y, -2, -3).reshape(a.shape[:-1] + (n,))


def rfft_large(x: np.ndarray, fft=None) -> np.ndarray:
    """Packed real FFT for even n (_fourstep.py:213-231): z = x[0::2] + i x[1::2], Z = FFT_m(z),
    X_k = ze - i w zo (k < m), X_m = Re Z_0 - Im Z_0."""
    x = np.asarray(x, dtype=np.float64)
    n = x.shape[-1]
    m = n // 2
    z = x[..., 0::2] + 1j * x[..., 1::2]
    Z = (fft or np.fft.fft)(z)
    zmk = np.concatenate([Z[..., :1], Z[..., 1:][..., ::-1]], axis=-1)
    w = np.exp(-1j * np.pi * np.arange(m) / m)
    ze = 0.5 * (Z + np.conj(zmk))
    zo = 0.5 * (Z - np.conj(zmk))
    Xk = ze - 1j * (w * zo)
    nyq = (Z[..., :1].real - Z[..., :1].imag) + 0j
    return np.concatenate([Xk, nyq], axis=-1)


def irfft_large(X: np.ndarray, n: int, ifft=None) -> np.ndarray:
    """Inverse of rfft_large for even n (_fourstep.py:372-408): DC/Nyquist taken as real,
    pre-twist E + i wO conj(w), half-length inverse FFT, interleave re/im."""
    X = np.asarray(X, dtype=np.complex128)
    m = n // 2
    cur = X.shape[-1]
    if cur < m + 1:
        X = np.concatenate([X, np.zeros(X.shape[:-1] + (m + 1 - cur,))], axis=-1)
    X = X[..., : m + 1].copy()
    X[..., 0] = X[..., 0].real
    X[..., m] = X[..., m].real
    Xk = X[..., :m]
    xflip = X[..., 1:][..., ::-1]
    E = 0.5 * (Xk + np.conj(xflip))
    wO = 0.5 * (Xk - np.conj(xflip))
    w = np.exp(-1j * np.pi * np.arange(m) / m)
    z = (ifft or np.fft.ifft)(E + 1j * (wO * np.conj(w)))
    out = np.empty(X.shape[:-1] + (n,))
    out[..., 0::2] = z.real
    out[..., 1::2] = z.imag
    return out


# ---------------------------------------------------------------------------------------------
# identities the B200 kernels use (checked against the restatement above in tests)
# ---------------------------------------------------------------------------------------------


def pair_trick_power(xa: np.ndarray, xb: np.ndarray) -> np.ndarray:
    """|FFT xa|^2 + |FFT xb|^2 from one complex FFT of z = xa + i xb:
    (|Z_k|^2 + |Z_{L-k}|^2) / 2 (both inputs real)."""
    Z = np.fft.fft(np.asarray(xa) + 1j * np.asarray(xb), axis=-1)
    Q = np.abs(Z) ** 2
    L = Z.shape[-1]
    return 0.5 * (Q + Q[..., (-np.arange(L)) % L])


def pair_trick_cross(x: np.ndarray, y: np.ndarray):
    """(Pxx, Pyy, Pxy=conj(X)Y) of real x, y from one complex FFT of z = x + i y:
    Q_k = |Z_k|^2, C_k = Z_k Z_{L-k}; Pxy = Im C/2 + i (Q_{L-k} - Q_k)/4,
    Pxx/Pyy = (Q_k + Q_{L-k} +/- 2 Re C)/4."""
    Z = np.fft.fft(np.asarray(x) + 1j * np.asarray(y), axis=-1)
    L = Z.shape[-1]
    mir = (-np.arange(L)) % L
    Q = np.abs(Z) ** 2
    Cc = Z * Z[..., mir]
    pxy = 0.5 * Cc.imag + 0.25j * (Q[..., mir] - Q)
    pxx = 0.25 * (Q + Q[..., mir] + 2 * Cc.real)
    pyy = 0.25 * (Q + Q[..., mir] - 2 * Cc.real)
    return pxx, pyy, pxy
