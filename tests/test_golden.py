"""CPU: golden fixtures are reproducible and the oracle restatement reproduces them."""

from pathlib import Path

import numpy as np
import scipy.signal as sps

from oracle import restate

GOLD = Path(__file__).resolve().parent / "golden" / "spectral_golden.npz"


def _rel(got, ref):
    return float(np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-300))


def test_fixtures_regenerate_from_scipy():
    g = np.load(GOLD)
    _, p = sps.welch(g["welch1_x"].astype(np.float64), fs=1.0, nperseg=256, noverlap=128)
    assert _rel(p, g["welch1_p"]) < 1e-12
    _, c = sps.coherence(g["cross_x"].astype(np.float64), g["cross_y"].astype(np.float64),
                         fs=48000.0, nperseg=1024, noverlap=512)
    assert _rel(c, g["coh_c"]) < 1e-12


def test_restatement_reproduces_fixtures():
    g = np.load(GOLD)
    hann256 = sps.get_window("hann", 256)
    hann1024 = sps.get_window("hann", 1024)
    p1 = restate.welch(g["welch1_x"][None], 1.0, hann256, 256, 128)[0]
    assert _rel(p1, g["welch1_p"]) < 1e-12
    p2 = restate.welch(g["welch2_x"], 48000.0, hann1024, 1024, 512)
    assert _rel(p2, g["welch2_p"]) < 1e-12
    pc = restate.csd(g["cross_x"], g["cross_y"], 48000.0, hann1024, 1024, 512)
    assert _rel(pc, g["csd_p"]) < 1e-12
    cc = restate.coherence(g["cross_x"], g["cross_y"], hann1024, 1024, 512)
    assert _rel(cc, g["coh_c"]) < 1e-10
    out, _ = restate.istft_frames(np.swapaxes(g["stft_z"], -1, -2), hann256,
                                  float(hann256.sum()), 256, 128)
    assert _rel(out[..., 128:-128], g["istft_x"]) < 1e-10
    X = restate.rfft_large(g["rfft_x"])
    assert _rel(X, g["rfft_X"]) < 1e-12
