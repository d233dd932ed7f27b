"""GPU: the CUDA path reproduces the committed golden fixtures (float64 scipy outputs)."""

from pathlib import Path

import numpy as np
import pytest

import mlx_signal_b200 as msig
from _utils import assert_close, rel_err_bins

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden" / "spectral_golden.npz"


@pytest.fixture(scope="module")
def g():
    return np.load(GOLD)


def test_welch_config1_small(g):
    f, p = msig.welch(g["welch1_x"], fs=1.0, window="hann", nperseg=256, noverlap=128,
                      detrend="constant", scaling="density", average="mean")
    assert tuple(p.shape) == (129,)
    assert_close(f, g["welch1_f"])
    assert rel_err_bins(p, g["welch1_p"]) <= 1e-5


def test_welch_config2_scaled(g):
    f, p = msig.welch(g["welch2_x"], fs=48000.0, nperseg=1024, noverlap=512)
    assert rel_err_bins(p, g["welch2_p"]) <= 1e-5


def test_csd_coherence_config3_scaled(g):
    _, pxy = msig.csd(g["cross_x"], g["cross_y"], fs=48000.0, nperseg=1024, noverlap=512)
    assert_close(pxy, g["csd_p"], rtol=2e-4)
    _, c = msig.coherence(g["cross_x"], g["cross_y"], fs=48000.0, nperseg=1024, noverlap=512)
    assert_close(c, g["coh_c"], rtol=1e-3)
    cn = c.cpu().numpy()
    assert cn.min() >= 0.0 and cn.max() <= 1.0


def test_stft_istft_spectrogram(g):
    f, t, z = msig.stft(g["stft_x"], fs=8000.0, nperseg=256)
    assert_close(z, g["stft_z"])
    assert_close(t, g["stft_t"])
    t2, x2 = msig.istft(g["stft_z"].astype(np.complex64), fs=8000.0, nperseg=256)
    assert_close(x2, g["istft_x"])
    f, t, s = msig.spectrogram(g["spec_x"], fs=8000.0, window="hann", nperseg=256,
                               noverlap=128)
    assert_close(s, g["spec_s"], rtol=2e-4)
