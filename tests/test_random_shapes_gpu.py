"""GPU parity over seeded random argument combinations against float64 scipy.signal: welch,
csd, coherence, spectrogram and stft with random rows, lengths, nperseg (powers of two and
not), noverlap, nfft, detrend, window, scaling, real / complex input, mean / median averaging
and boundary / padding. Each case uses the reference's tolerance rule (rtol 1e-4, atol 1e-5 of
the peak; csd 2e-4, coherence 1e-3)."""

import warnings

import numpy as np
import pytest
import scipy.signal as sps

import mlx_signal_b200 as msig
from _utils import assert_close

pytestmark = pytest.mark.gpu

WINDOWS = ["hann", "hamming", "blackman", ("tukey", 0.3), "boxcar", ("kaiser", 6.0)]
NPERSEGS = [1, 2, 7, 16, 33, 64, 100, 128, 250, 256, 300, 512, 777, 1000, 1024, 2048]


def _case(rng):
    nperseg = int(rng.choice(NPERSEGS))
    n = int(rng.integers(nperseg, 6 * nperseg + 50))
    rows = int(rng.integers(1, 4))
    kw = {"nperseg": nperseg, "window": WINDOWS[int(rng.integers(len(WINDOWS)))]}
    if nperseg > 1 and rng.random() < 0.6:
        kw["noverlap"] = int(rng.integers(0, nperseg))
    if rng.random() < 0.3:
        kw["nfft"] = nperseg + int(rng.integers(0, nperseg + 1))
    kw["detrend"] = [False, "constant", "linear"][int(rng.integers(3))]
    cplx = rng.random() < 0.25
    return rows, n, kw, cplx


def _degenerate(kw) -> bool:
    """Linear detrend of one- or two-sample segments leaves exact zeros: every output is
    rounding residue (float64 in scipy, float32 here), checked against the input's scale."""
    return kw["detrend"] == "linear" and kw["nperseg"] <= 2


def _assert_residue(got, x, power: bool):
    a = np.abs(got.cpu().numpy())
    scale = float(np.max(np.abs(x))) ** (2 if power else 1)
    assert a.max() <= 1e-5 * scale, f"degenerate case: output {a.max():.3e} vs scale {scale:.3e}"


def _signal(rng, rows, n, cplx):
    x = rng.standard_normal((rows, n)).astype(np.float32)
    x += (rng.standard_normal((rows, 1)) * 2).astype(np.float32)  # DC offsets
    if cplx:
        x = (x + 1j * rng.standard_normal((rows, n))).astype(np.complex64)
    return x


@pytest.mark.parametrize("seed", range(60))
def test_random_welch_csd_coherence(seed):
    rng = np.random.default_rng(1000 + seed)
    rows, n, kw, cplx = _case(rng)
    x = _signal(rng, rows, n, cplx)
    y = (0.6 * np.roll(x, 3, axis=-1) + 0.4 * _signal(rng, rows, n, cplx)).astype(x.dtype)
    x64 = x.astype(np.complex128 if cplx else np.float64)
    y64 = y.astype(np.complex128 if cplx else np.float64)
    average = "median" if rng.random() < 0.3 else "mean"
    scaling = "spectrum" if rng.random() < 0.3 else "density"
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        _, p_ref = sps.welch(x64, fs=100.0, average=average, scaling=scaling, **kw)
        _, p = msig.welch(x, fs=100.0, average=average, scaling=scaling, **kw)
        assert tuple(p.shape) == p_ref.shape
        _, c_ref = sps.csd(x64, y64, fs=100.0, average=average, scaling=scaling, **kw)
        _, c = msig.csd(x, y, fs=100.0, average=average, scaling=scaling, **kw)
        assert tuple(c.shape) == c_ref.shape
        if _degenerate(kw):
            _assert_residue(p, x, True)
            _assert_residue(c, x, True)
            return
        assert_close(p, p_ref)
        assert_close(c, c_ref, rtol=2e-4)
        if kw["nperseg"] > 1:
            _, h_ref = sps.coherence(x64, y64, fs=100.0, **kw)
            _, h = msig.coherence(x, y, fs=100.0, **kw)
            # bins whose auto-spectra are rounding residue (the DC bin of a boxcar window after
            # detrending is exactly zero) have an undefined ratio: compare the others
            _, pxx = sps.welch(x64, fs=100.0, **kw)
            _, pyy = sps.welch(y64, fs=100.0, **kw)
            keep = ((pxx > 1e-9 * pxx.max(axis=-1, keepdims=True))
                    & (pyy > 1e-9 * pyy.max(axis=-1, keepdims=True)))
            assert tuple(h.shape) == h_ref.shape
            hh = h.cpu().numpy()
            np.testing.assert_allclose(hh[keep], h_ref[keep], rtol=1e-3, atol=1e-5)


@pytest.mark.parametrize("seed", range(60))
def test_random_stft_spectrogram(seed):
    rng = np.random.default_rng(2000 + seed)
    rows, n, kw, cplx = _case(rng)
    x = _signal(rng, rows, n, cplx)
    x64 = x.astype(np.complex128 if cplx else np.float64)
    boundary = [None, "zeros", "even", "odd", "constant"][int(rng.integers(5))]
    if boundary in ("even", "odd") and kw["nperseg"] // 2 > n - 1:
        boundary = "zeros"
    padded = bool(rng.random() < 0.5)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        _, t_ref, z_ref = sps.stft(x64, fs=50.0, boundary=boundary, padded=padded, **kw)
        _, t, z = msig.stft(x, fs=50.0, boundary=boundary, padded=padded, **kw)
        assert tuple(z.shape) == z_ref.shape
        assert_close(t, t_ref)
        mode = ["psd", "complex", "magnitude"][int(rng.integers(3))]
        _, _, s_ref = sps.spectrogram(x64, fs=50.0, mode=mode, **kw)
        _, _, s = msig.spectrogram(x, fs=50.0, mode=mode, **kw)
        assert tuple(s.shape) == s_ref.shape
        if _degenerate(kw):
            _assert_residue(z, x, False)
            _assert_residue(s, x, mode == "psd")
            return
        assert_close(z, z_ref)
        assert_close(s, s_ref)


@pytest.mark.parametrize("seed", range(40))
def test_random_istft(seed):
    rng = np.random.default_rng(3000 + seed)
    nperseg = int(rng.choice([8, 16, 64, 100, 128, 256, 512, 1024]))
    noverlap = int(rng.integers(nperseg // 2, nperseg)) if rng.random() < 0.7 else nperseg // 2
    window = WINDOWS[int(rng.integers(len(WINDOWS)))]
    if window == "boxcar" and noverlap == 0:
        noverlap = nperseg // 2
    rows = int(rng.integers(1, 4))
    n = int(rng.integers(nperseg, 6 * nperseg))
    onesided = bool(rng.random() < 0.8)
    x = rng.standard_normal((rows, n))
    if not onesided:
        x = x + 1j * rng.standard_normal((rows, n))
    boundary = bool(rng.random() < 0.7)
    kw = dict(window=window, nperseg=nperseg, noverlap=noverlap)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        _, _, z = sps.stft(x, return_onesided=onesided, boundary="zeros" if boundary else None,
                           **kw)
        t_ref, x_ref = sps.istft(z, input_onesided=onesided, boundary=boundary, **kw)
        zc = z.astype(np.complex64)
        t, xr = msig.istft(zc, input_onesided=onesided, boundary=boundary, **kw)
    assert tuple(xr.shape) == x_ref.shape
    # the overlap-added window energy the reconstruction divides by (scipy's NOLA norm): where
    # it is small, float32 rounding of the frames is amplified by 1/norm, so those samples get a
    # proportionally wider bound
    w2 = sps.get_window(window, nperseg) ** 2
    hop = nperseg - noverlap
    nseg = z.shape[-1]
    norm = np.zeros(nperseg + (nseg - 1) * hop)
    for k in range(nseg):
        norm[k * hop : k * hop + nperseg] += w2
    if boundary:
        norm = norm[nperseg // 2 : -(nperseg // 2)]
    norm = norm[: x_ref.shape[-1]]
    got = xr.cpu().numpy()
    peak = float(np.max(np.abs(x_ref)))
    well = norm >= 1e-2 * norm.max()
    np.testing.assert_allclose(got[..., well], x_ref[..., well], rtol=1e-4, atol=1e-5 * peak)
    bound = 1e-5 * peak * norm.max() / np.maximum(norm, 1e-10)
    assert np.all(np.abs(got - x_ref) <= bound + 1e-4 * np.abs(x_ref))


@pytest.mark.parametrize("seed", range(40))
def test_random_convolutions(seed):
    rng = np.random.default_rng(4000 + seed)
    n1 = int(rng.integers(1, 30000))
    n2 = int(rng.choice([1, 2, 5, 64, 129, 500, 1025, 2049, 3000, int(rng.integers(1, 5000))]))
    rows = int(rng.integers(1, 3))
    a = rng.standard_normal((rows, n1)).astype(np.float32)
    b = rng.standard_normal((1, n2)).astype(np.float32)
    if rng.random() < 0.3:
        a, b = b, a  # filter first
    mode = ["full", "same", "valid"][int(rng.integers(3))]
    if mode == "valid" and not (all(p >= q for p, q in zip(a.shape, b.shape))
                                or all(p <= q for p, q in zip(a.shape, b.shape))):
        mode = "full"
    fn = "oaconvolve" if rng.random() < 0.5 else "fftconvolve"
    ref = getattr(sps, fn)(a.astype(np.float64), b.astype(np.float64), mode=mode, axes=-1)
    got = getattr(msig, fn)(a, b, mode=mode, axes=-1)
    assert tuple(got.shape) == ref.shape
    if ref.size:
        err = float(np.max(np.abs(got.cpu().numpy() - ref)) / max(np.max(np.abs(ref)), 1e-30))
        assert err < 5e-6, f"{fn} {a.shape} {b.shape} {mode}: {err:.3e}"


@pytest.mark.parametrize("seed", range(12))
def test_random_batches(seed):
    """welch_batch over a random mix (batched classes, other nperseg, short rows, windows,
    detrend) against scipy per request."""
    from mlx_signal_b200 import batch

    rng = np.random.default_rng(5000 + seed)
    items = []
    for _ in range(int(rng.integers(1, 24))):
        nps = int(rng.choice([256, 512, 1024, 2048, 4096, 300, 128]))
        n = int(rng.integers(max(1, nps // 2), 5 * nps + 100))
        x = rng.standard_normal((int(rng.integers(1, 5)), n)).astype(np.float32)
        kw = {"nperseg": nps, "detrend": [False, "constant"][int(rng.integers(2))],
              "window": ["hann", "hamming", ("tukey", 0.25)][int(rng.integers(3))]}
        if rng.random() < 0.3:
            kw["noverlap"] = int(rng.integers(0, min(nps, n)))
        items.append((x, kw))
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        res = batch.welch_batch(items)
        for (x, kw), (f, p) in zip(items, res):
            f_ref, p_ref = sps.welch(x.astype(np.float64), **kw)
            assert tuple(p.shape) == p_ref.shape
            assert_close(f, f_ref)
            assert_close(p, p_ref)


@pytest.mark.parametrize("seed", range(12))
def test_random_streams(seed):
    rng = np.random.default_rng(6000 + seed)
    nps = int(rng.choice([256, 512, 1024, 2048, 4096, 200, 333]))
    nov = int(rng.integers(0, nps))
    rows = int(rng.integers(1, 4))
    total = int(rng.integers(nps, 12 * nps))
    x = rng.standard_normal((rows, total)).astype(np.float32)
    st = msig.StreamingSTFT(rows=rows, fs=10.0, nperseg=nps, noverlap=nov)
    sw = msig.StreamingWelch(rows=rows, fs=10.0, nperseg=nps, noverlap=nov)
    pos, zs = 0, []
    while pos < total:
        m = int(rng.integers(0, 3 * nps))
        chunk = x[:, pos : pos + m]
        zs.append(st.push(chunk)[1].cpu().numpy())
        sw.push(chunk)
        pos += m
    _, _, z_ref = sps.stft(x.astype(np.float64), fs=10.0, nperseg=nps, noverlap=nov,
                           boundary=None, padded=False)
    z = np.concatenate(zs, axis=-1)
    assert z.shape == z_ref.shape
    assert_close(z, z_ref)
    _, p_ref = sps.welch(x.astype(np.float64), fs=10.0, nperseg=nps, noverlap=nov)
    assert_close(sw.psd()[1], p_ref)
