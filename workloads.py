"""Named, seeded workloads for profiling the kernels from the command line (the commands of the
ncu summaries under profiles/ run these):

    python workloads.py NAME [NAME ...] [--repeat K]

Each workload builds its inputs on the current CUDA device (seeded N(0,1) float32) and runs its
public call K times (default 1), so a profiler's kernel filter and launch count select exactly
the launches wanted. `--list` prints the names.
"""

from __future__ import annotations

import argparse
import sys

from pathlib import Path

import numpy as np
import torch

sys.path.insert(0, str(Path(__file__).resolve().parent))

__all__ = ["WORKLOADS", "run"]


def _randn(shape, seed: int) -> torch.Tensor:
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return torch.randn(shape, generator=g, device="cuda")


def _big(seed: int = 3) -> torch.Tensor:
    return _randn((64, 1 << 20), seed)


def _welch(msig, k):
    x = _big()
    return [lambda: msig.welch(x, fs=48000.0, nperseg=1024)] * k


def _welch_n(nperseg):
    def build(msig, k):
        x = _big()
        return [lambda: msig.welch(x, fs=48000.0, nperseg=nperseg)] * k
    return build


def _stft(msig, k):
    x = _big()
    return [lambda: msig.stft(x, nperseg=1024)] * k


def _spectrogram(msig, k):
    x = _big()
    return [lambda: msig.spectrogram(x, nperseg=1024, noverlap=512, window="hann")] * k


def _coherence(msig, k):
    x = _big()
    y = (0.7 * torch.roll(x, 17, dims=-1) + 0.3 * _randn(x.shape, 4)).contiguous()
    return [lambda: msig.coherence(x, y, nperseg=1024)] * k


def _istft(msig, k):
    x = _big()
    _, _, z = msig.stft(x, nperseg=1024)
    return [lambda: msig.istft(z, nperseg=1024)] * k


def _batch48(msig, k):
    from mlx_signal_b200 import batch

    rng = np.random.default_rng(3)
    sigs = []
    for i in range(48):
        c = int(rng.integers(1, 33))
        n = int(2 ** rng.uniform(14, 21))
        nps = int(rng.choice([256, 1024, 4096]))
        sigs.append((_randn((c, max(n, nps)), 100 + i), {"nperseg": nps}))
    return [lambda: batch.welch_batch(sigs)] * k


def _rfft(msig, k):
    x = _randn(1 << 23, 5)
    return [lambda: msig.fft.rfft(x)] * k


def _conv(msig, k):
    x = _randn((8, 1 << 22), 6)
    h = _randn((1, 1025), 7)
    return [lambda: msig.oaconvolve(x, h, axes=-1)] * k


def _blue_welch(msig, k):
    x = _big()
    return [lambda: msig.welch(x, nperseg=1000)] * k


def _blue_stft(msig, k):
    x = _big()[:16].contiguous()
    return [lambda: msig.stft(x, nperseg=1000)] * k


def _rfft_odd(msig, k):
    # both directions on the kernels (the public routing sends this forward length to cuFFT)
    msig.fft.ODD_FORWARD = True
    msig.fft.KERNEL_MIN_LOG2 = 12
    x = _randn(3 << 20, 12)
    X = msig.fft.rfft(x)
    return [lambda: msig.fft.rfft(x), lambda: msig.fft.irfft(X, n=3 << 20)] * k


def _resample_odd(msig, k):
    x = _randn(1 << 22, 13)
    return [lambda: msig.resample(x, 3 << 20)] * k


def _hilbert(msig, k):
    x = _randn(1 << 23, 9)
    return [lambda: msig.hilbert(x)] * k


def _tc_dft32(msig, k):
    from mlx_signal_b200 import _kernels

    z = torch.complex(_randn((1 << 18, 32), 10), _randn((1 << 18, 32), 11))
    return [lambda: _kernels.dft32_tc(z)] * k


WORKLOADS = {
    "welch_64x2p20_n1024": _welch,
    "welch_64x2p20_n256": _welch_n(256),
    "welch_64x2p20_n4096": _welch_n(4096),
    "stft_64x2p20": _stft,
    "spectrogram_64x2p20": _spectrogram,
    "coherence_64x2p20": _coherence,
    "istft_64x2p20": _istft,
    "batch_48": _batch48,
    "rfft_2p23": _rfft,
    "conv_8x2p22_t1025": _conv,
    "bluestein_welch_64x2p20_n1000": _blue_welch,
    "bluestein_stft_16x2p20_n1000": _blue_stft,
    "hilbert_2p23": _hilbert,
    "tc_dft32_2p18": _tc_dft32,
    "rfft_irfft_3x2p20": _rfft_odd,
    "resample_2p22_to_3x2p20": _resample_odd,
}


def run(names, repeat: int = 1) -> None:
    import mlx_signal_b200 as msig

    for name in names:
        if name not in WORKLOADS:
            raise SystemExit(f"unknown workload {name!r}; choose from {sorted(WORKLOADS)}")
        for call in WORKLOADS[name](msig, repeat):
            call()
        torch.cuda.synchronize()


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("names", nargs="*")
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--list", action="store_true")
    a = ap.parse_args(argv)
    if a.list or not a.names:
        print("\n".join(sorted(WORKLOADS)))
        return 0
    run(a.names, a.repeat)
    print("ok")
    return 0


if __name__ == "__main__":
    sys.exit(main())
