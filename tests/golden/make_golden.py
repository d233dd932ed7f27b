"""Generate the golden fixtures: seeded float32 inputs and float64 scipy.signal outputs.

The reference (mlx-signal) tests against float64 scipy computed in-test and ships no vectors;
these fixtures freeze that oracle for the workloads of this project (the 1 x 2^16 welch case
exactly, scaled-down versions of the 64 x 2^20 welch and cross-spectral workloads,
stft/istft/spectrogram and packed rfft cases). Run from the repo root:

    python tests/golden/make_golden.py
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import scipy.signal as sps

OUT = Path(__file__).resolve().parent / "spectral_golden.npz"


def multitone(rng, C, n, fs):
    t = np.arange(n) / fs
    x = rng.standard_normal((C, n))
    for c in range(C):
        for _ in range(int(rng.integers(1, 5))):
            x[c] += rng.uniform(0.1, 2.0) * np.sin(2 * np.pi * rng.uniform(0, fs / 2) * t)
    return x.astype(np.float32)


def main():
    rng = np.random.default_rng(20261203)
    g = {}
    # small welch: 1 x 2^16, N(0,1) + unit sinusoid at 0.1 fs; hann 256/128, constant, density
    n1 = 1 << 16
    x1 = (rng.standard_normal(n1) + np.sin(2 * np.pi * 0.1 * np.arange(n1))).astype(np.float32)
    g["welch1_x"] = x1
    g["welch1_f"], g["welch1_p"] = sps.welch(x1.astype(np.float64), fs=1.0, window="hann",
                                             nperseg=256, noverlap=128, detrend="constant",
                                             scaling="density", average="mean")
    # the 64 x 2^20 welch workload scaled down: 4 x 2^13 multi-tone, fs 48 kHz, hann 1024/512
    x2 = multitone(rng, 4, 1 << 13, 48000.0)
    g["welch2_x"] = x2
    g["welch2_f"], g["welch2_p"] = sps.welch(x2.astype(np.float64), fs=48000.0, nperseg=1024,
                                             noverlap=512)
    # the cross-spectral (csd / coherence) workload scaled down: y = 0.7 * circular shift(x) + 0.3 N(0,1)
    x3 = rng.standard_normal((4, 1 << 14)).astype(np.float32)
    shifts = rng.integers(0, 65, size=4)
    y3 = np.stack([0.7 * np.roll(x3[c], int(shifts[c])) for c in range(4)])
    y3 = (y3 + 0.3 * rng.standard_normal(y3.shape)).astype(np.float32)
    g["cross_x"], g["cross_y"] = x3, y3
    _, g["csd_p"] = sps.csd(x3.astype(np.float64), y3.astype(np.float64), fs=48000.0,
                            nperseg=1024, noverlap=512)
    _, g["coh_c"] = sps.coherence(x3.astype(np.float64), y3.astype(np.float64), fs=48000.0,
                                  nperseg=1024, noverlap=512)
    # stft (defaults: boundary zeros, padded) and its istft
    xs = multitone(rng, 2, 4000, 8000.0)
    g["stft_x"] = xs
    g["stft_f"], g["stft_t"], g["stft_z"] = sps.stft(xs.astype(np.float64), fs=8000.0,
                                                     nperseg=256)
    g["istft_t"], g["istft_x"] = sps.istft(g["stft_z"], fs=8000.0, nperseg=256)
    # spectrogram psd with an explicit hann window (the bench form)
    g["spec_x"] = xs
    g["spec_f"], g["spec_t"], g["spec_s"] = sps.spectrogram(xs.astype(np.float64), fs=8000.0,
                                                            window="hann", nperseg=256,
                                                            noverlap=128)
    # packed real FFT (pins the large-n untangle on a small size)
    xr = rng.standard_normal(1 << 16).astype(np.float32)
    g["rfft_x"], g["rfft_X"] = xr, np.fft.rfft(xr.astype(np.float64))
    np.savez_compressed(OUT, **g)
    print(f"wrote {OUT} ({OUT.stat().st_size / 1e6:.2f} MB)")


if __name__ == "__main__":
    main()
