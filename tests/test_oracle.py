"""CPU: the oracle's restatement of the reference's kernels against float64 scipy/numpy.

This pins the oracle: the reference's own algorithm (restated step by step in
oracle/restate.py) reproduces float64 scipy.signal / numpy.fft on the reference's test cases,
so scipy is a valid stand-in for the reference's output in the GPU parity tests. It also checks
the two packing identities the B200 kernels rely on.
"""

import numpy as np
import pytest
import scipy.signal as sps

from _utils import make_sig
from oracle import restate


def _rel(got, ref):
    return float(np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-300))


@pytest.mark.parametrize("N", [64, 128, 256, 512, 1024, 2048])
@pytest.mark.parametrize("detrend", [False, "constant"])
def test_packed_stockham_rfft_frames(rng, N, detrend):
    x = rng.standard_normal((2, 6 * N + 13))
    win = rng.standard_normal(N)
    hop = N // 2 + 3
    got = restate.rfft_frames(x, win, N, hop, detrend)
    nseg = (x.shape[-1] - N) // hop + 1
    idx = np.arange(N)[None, :] + hop * np.arange(nseg)[:, None]
    fr = x[:, idx]
    if detrend:
        fr = fr - fr.mean(-1, keepdims=True)
    ref = np.fft.rfft(fr * win, axis=-1)
    assert _rel(got, ref) < 1e-12


WELCH_FUSED_CASES = [
    dict(nperseg=256),
    dict(nperseg=128),
    dict(nperseg=128, noverlap=96),
    dict(nperseg=128, window="hamming"),
    dict(nperseg=128, detrend=False),
    dict(nperseg=128, scaling="spectrum"),
    dict(nperseg=1024, noverlap=512, fs=48000.0),
]


@pytest.mark.parametrize("case", WELCH_FUSED_CASES)
@pytest.mark.parametrize("n", [1024, 4093])
def test_grouped_welch_restatement_matches_scipy(rng, case, n):
    x = make_sig(rng, (3, max(n, 2048))).astype(np.float64)
    kw = dict(fs=1.0, window="hann", noverlap=None, detrend="constant", scaling="density")
    kw.update(case)
    N = kw["nperseg"]
    nov = N // 2 if kw["noverlap"] is None else kw["noverlap"]
    win = sps.get_window(kw["window"], N)
    got = restate.welch(x, kw["fs"], win, N, nov, kw["detrend"], kw["scaling"])
    _, ref = sps.welch(x, **kw)
    assert _rel(got, ref) < 1e-12


def test_pair_means_restatement_matches_scipy(rng):
    x = make_sig(rng, (4, 8192)).astype(np.float64)
    y = 0.5 * x + 0.5 * make_sig(rng, (4, 8192))
    win = sps.get_window("hann", 256)
    got = restate.csd(x, y, 1.0, win, 256, 128)
    _, ref = sps.csd(x, y, nperseg=256)
    assert _rel(got, ref) < 1e-12
    coh = restate.coherence(x, y, win, 256, 128)
    _, cref = sps.coherence(x, y, nperseg=256)
    assert _rel(coh, cref) < 1e-10


@pytest.mark.parametrize("nperseg,noverlap,window", [(256, 128, "hann"), (256, 192, "hann"),
                                                     (512, 256, "hamming")])
def test_istft_restatement_matches_scipy(rng, nperseg, noverlap, window):
    x = make_sig(rng, (2, 4000)).astype(np.float64)
    _, _, z = sps.stft(x, nperseg=nperseg, noverlap=noverlap, window=window)
    win = sps.get_window(window, nperseg)
    out, norm = restate.istft_frames(np.swapaxes(z, -1, -2), win, float(win.sum()), nperseg,
                                     nperseg - noverlap)
    out = out[..., nperseg // 2 : -(nperseg // 2)]
    _, ref = sps.istft(z, nperseg=nperseg, noverlap=noverlap, window=window)
    assert _rel(out, ref) < 1e-10


@pytest.mark.parametrize("e", [21, 22])
@pytest.mark.parametrize("inverse", [False, True])
def test_three_pass_index_maps(rng, e, inverse):
    n = 1 << e
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    got = restate.fft3(x, inverse=inverse)
    ref = np.fft.ifft(x) if inverse else np.fft.fft(x)
    assert _rel(got, ref) < 1e-12


def test_large_real_transforms(rng):
    n = 1 << 21
    x = rng.standard_normal(n)
    X = restate.rfft_large(x, fft=lambda z: restate.fft3(z))
    assert _rel(X, np.fft.rfft(x)) < 1e-12
    back = restate.irfft_large(X, n, ifft=lambda z: restate.fft3(z, inverse=True))
    assert _rel(back, x) < 1e-12


def test_pair_trick_identities(rng):
    a = rng.standard_normal((5, 1024))
    b = rng.standard_normal((5, 1024))
    got = restate.pair_trick_power(a, b)
    ref = np.abs(np.fft.fft(a)) ** 2 + np.abs(np.fft.fft(b)) ** 2
    assert _rel(got, ref) < 1e-12
    pxx, pyy, pxy = restate.pair_trick_cross(a, b)
    X, Y = np.fft.fft(a), np.fft.fft(b)
    assert _rel(pxx, np.abs(X) ** 2) < 1e-11
    assert _rel(pyy, np.abs(Y) ** 2) < 1e-11
    assert _rel(pxy, np.conj(X) * Y) < 1e-11


def test_group_params_match_reference_rule():
    # 64 channels x 2047 segments (the 64 x 2^20, nperseg 1024 welch) -> groups of 64, 32 per row
    assert restate.group_params(64, 2047) == (64, 32)
    assert restate.group_params(2048, 9) == (9, 1)
    assert restate.group_params(1, 1) == (1, 1)
