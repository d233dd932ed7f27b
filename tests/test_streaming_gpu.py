"""GPU parity of the streaming API: chunked StreamingSTFT frames against scipy.signal.stft of the
concatenated stream (boundary=None, padded=False), StreamingWelch against scipy.signal.welch of
everything pushed so far. Chunk sizes are ragged (empty, shorter than a hop, longer than
nperseg), over the batched stream kernel (nperseg 256/512/1024/4096, named window) and the
per-frame fallback (other nperseg, array windows)."""

import numpy as np
import pytest
import scipy.signal as sps
import torch

import mlx_signal_b200 as msig
from _utils import assert_close

pytestmark = pytest.mark.gpu


def chunks(rng, total, sizes):
    cuts, pos = [], 0
    for s in sizes:
        cuts.append((pos, min(total, pos + s)))
        pos = min(total, pos + s)
    cuts.append((pos, total))
    return cuts


@pytest.mark.parametrize("rows,nperseg,noverlap,window",
                         [(1, 1024, None, "hann"), (3, 256, 192, "hamming"),
                          (2, 4096, None, "hann"), (2, 300, 100, "hann"),
                          (1, 128, 32, ("tukey", 0.25))])
def test_streaming_stft_matches_scipy(rng, rows, nperseg, noverlap, window):
    total = 40000
    x = rng.standard_normal((rows, total)).astype(np.float32)
    st = msig.StreamingSTFT(rows=rows, fs=8.0, window=window, nperseg=nperseg,
                            noverlap=noverlap)
    sizes = [0, 7, nperseg - 1, 3 * nperseg + 5, 1, 5000, 0, 12345]
    ts, zs = [], []
    for a, b in chunks(rng, total, sizes):
        t, z = st.push(torch.from_numpy(x[:, a:b]).cuda())
        assert z.shape[0] == rows and z.shape[-1] == t.shape[0]
        ts.append(t.cpu().numpy())
        zs.append(z.cpu().numpy())
    f_ref, t_ref, z_ref = sps.stft(x.astype(np.float64), fs=8.0, window=window,
                                   nperseg=nperseg, noverlap=noverlap, boundary=None,
                                   padded=False, detrend=False)
    z = np.concatenate(zs, axis=-1)
    assert z.shape == z_ref.shape
    assert_close(np.concatenate(ts), t_ref)
    assert_close(z, z_ref)
    assert st.frames_emitted == z_ref.shape[-1] and st.samples_seen == total


def test_streaming_stft_one_dimensional(rng):
    x = rng.standard_normal(9000).astype(np.float32)
    st = msig.StreamingSTFT(nperseg=512)
    parts = [st.push(x[i:i + 1000])[1] for i in range(0, 9000, 1000)]
    z = torch.cat(parts, dim=-1).cpu().numpy()
    _, _, z_ref = sps.stft(x.astype(np.float64), nperseg=512, boundary=None, padded=False)
    assert z.shape == z_ref.shape
    assert_close(z, z_ref)
    with pytest.raises(ValueError):
        st.push(np.zeros((2, 10), np.float32))


@pytest.mark.parametrize("kw", [{"nperseg": 1024}, {"nperseg": 256, "noverlap": 64},
                                {"nperseg": 512, "detrend": "linear", "scaling": "spectrum"},
                                {"nperseg": 300}, {"nperseg": 128, "nfft": 256,
                                                   "return_onesided": False}])
def test_streaming_welch_matches_scipy(rng, kw):
    rows, total = 2, 60000
    x = rng.standard_normal((rows, total)).astype(np.float32)
    sw = msig.StreamingWelch(rows=rows, fs=100.0, **kw)
    with pytest.raises(ValueError):
        sw.psd()
    pos = 0
    for s in [3, 500, 4097, 1, 20000, 999]:
        sw.push(torch.from_numpy(x[:, pos:pos + s]).cuda())
        pos += s
        if pos >= kw["nperseg"]:
            f, p = sw.psd()
            f_ref, p_ref = sps.welch(x[:, :pos].astype(np.float64), fs=100.0, **kw)
            assert_close(f, f_ref)
            assert_close(p, p_ref)
    sw.reset()
    assert sw.segments == 0
