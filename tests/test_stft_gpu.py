"""GPU parity: spectrogram / stft / istft against float64 scipy.signal.

Cases follow the reference's tests/test_spectral.py (spectrogram modes, STFT_CASES boundary /
padded / scaling, ISTFT_CASES, batched, layouts, arbitrary axes, validation, round trip) and
test_metal_fft_workaround.py:97-131 (fused frames kernel vs a frame-by-frame oracle for odd hops).
"""

import numpy as np
import pytest
import scipy.signal as sps
import torch

import mlx_signal_b200 as msig
from _utils import assert_close, make_sig

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["psd", "complex", "magnitude", "angle", "phase"])
def test_spectrogram_matches_scipy(rng, mode):
    x = make_sig(rng, (4096,))
    f_ref, t_ref, s_ref = sps.spectrogram(x.astype(np.float64), fs=100.0, mode=mode)
    f, t, s = msig.spectrogram(x, fs=100.0, mode=mode)
    assert s_ref.shape == tuple(s.shape)
    assert_close(f, f_ref)
    assert_close(t, t_ref)
    if mode in ("angle", "phase"):
        mag = np.abs(sps.spectrogram(x.astype(np.float64), fs=100.0, mode="complex")[2])
        keep = mag > 1e-4 * mag.max()
        a = s.cpu().numpy()[keep]
        d = s_ref[keep]
        diff = np.angle(np.exp(1j * (a - d)))
        np.testing.assert_allclose(diff, np.zeros_like(diff), atol=2e-3)
    else:
        assert_close(s, s_ref, rtol=2e-4)


def test_spectrogram_custom_params(rng):
    x = make_sig(rng, (4096,))
    kw = dict(nperseg=200, noverlap=50, nfft=256, scaling="spectrum", detrend="linear")
    f_ref, t_ref, s_ref = sps.spectrogram(x.astype(np.float64), **kw)
    f, t, s = msig.spectrogram(x, **kw)
    assert_close(s, s_ref)


STFT_CASES = [
    {},
    {"nperseg": 128},
    {"nperseg": 128, "noverlap": 100},
    {"nperseg": 128, "nfft": 256},
    {"boundary": "even"},
    {"boundary": "odd"},
    {"boundary": "constant"},
    {"boundary": None},
    {"padded": False},
    {"scaling": "psd"},
    {"detrend": "constant"},
    {"return_onesided": False},
]


@pytest.mark.parametrize("case", STFT_CASES)
def test_stft_matches_scipy(rng, case):
    x = make_sig(rng, (4000,))
    f_ref, t_ref, z_ref = sps.stft(x.astype(np.float64), fs=8000.0, **case)
    f, t, z = msig.stft(x, fs=8000.0, **case)
    assert z_ref.shape == tuple(z.shape)
    assert_close(f, f_ref)
    assert_close(t, t_ref)
    assert_close(z, z_ref)


def test_stft_multidim_axis0(rng):
    x = make_sig(rng, (3000, 4))
    f_ref, t_ref, z_ref = sps.stft(x.astype(np.float64), axis=0)
    f, t, z = msig.stft(x, axis=0)
    assert z_ref.shape == tuple(z.shape)
    assert_close(z, z_ref)


def test_stft_complex_input(rng):
    x = make_sig(rng, (2048,), complex_=True)
    with pytest.warns(UserWarning):
        f_ref, t_ref, z_ref = sps.stft(x.astype(np.complex128))
    f, t, z = msig.stft(x)
    assert_close(z, z_ref)


@pytest.mark.parametrize(
    "n,N,hop,detrend",
    [(5000, 256, 100, False), (5000, 256, 100, "constant"), (40000, 1024, 512, "constant"),
     (40000, 2048, 320, False), (3000, 64, 7, "constant"), (9000, 4096, 1000, "linear")],
)
def test_fused_frames_match_frame_oracle(rng, n, N, hop, detrend):
    """Fused per-frame kernel vs float64 frame-by-frame FFT with a random window (the
    reference's fused-vs-composed check, test_metal_fft_workaround.py:97-131)."""
    x = rng.standard_normal((3, n)).astype(np.float32)
    win = rng.standard_normal(N).astype(np.float32)
    nseg = (n - N) // hop + 1
    idx = np.arange(N)[None, :] + hop * np.arange(nseg)[:, None]
    fr = x.astype(np.float64)[:, idx]
    if detrend:
        fr = sps.detrend(fr, type=detrend, axis=-1)
    ref = np.fft.rfft(fr * win.astype(np.float64), axis=-1)
    from mlx_signal_b200 import _kernels
    code = _kernels.DETREND_CODES[detrend]
    xt = torch.from_numpy(x).cuda()
    wt = torch.from_numpy(win).cuda()
    got = _kernels.frames("stft", xt, wt, N, N, hop, code, True).cpu().numpy()
    np.testing.assert_allclose(got, ref, rtol=1e-4, atol=1e-5 * np.abs(ref).max())
    gotp = _kernels.frames("power", xt, wt, N, N, hop, code, False).cpu().numpy()
    refp = np.abs(np.fft.fft(fr * win.astype(np.float64), axis=-1)) ** 2
    np.testing.assert_allclose(gotp, refp, rtol=1e-4, atol=1e-5 * refp.max())


ISTFT_CASES = [
    {},
    {"boundary": False},
    {"scaling": "psd"},
    {"nperseg": 256, "noverlap": 192},
    {"window": "hamming"},
]


@pytest.mark.parametrize("case", ISTFT_CASES)
def test_istft_matches_scipy(rng, case):
    x = make_sig(rng, (4000,))
    stft_kw = {k: case[k] for k in ("nperseg", "noverlap", "window") if k in case}
    if case.get("scaling") == "psd":
        stft_kw["scaling"] = "psd"
    if case.get("boundary") is False:
        stft_kw["boundary"] = None
    f, t, z = sps.stft(x.astype(np.float64), **stft_kw)
    if case.get("boundary") is False:
        import warnings as _w

        with _w.catch_warnings():
            _w.simplefilter("ignore")
            t_ref, x_ref = sps.istft(z, **case)
            t2, x2 = msig.istft(z, **case)
        assert x_ref.shape == tuple(x2.shape)
        assert_close(x2.cpu().numpy()[128:-128], x_ref[128:-128])
    else:
        t_ref, x_ref = sps.istft(z, **case)
        t2, x2 = msig.istft(z, **case)
        assert x_ref.shape == tuple(x2.shape)
        assert_close(x2, x_ref)
    assert_close(t2, t_ref)


def test_istft_twosided(rng):
    x = make_sig(rng, (2048,))
    _, _, z = sps.stft(x.astype(np.float64), return_onesided=False)
    t_ref, x_ref = sps.istft(z, input_onesided=False)
    t2, x2 = msig.istft(z, input_onesided=False)
    assert_close(x2.real if x2.is_complex() else x2, x_ref.real)


def test_istft_batched(rng):
    x = make_sig(rng, (3, 4000))
    _, _, z = sps.stft(x.astype(np.float64))
    t_ref, x_ref = sps.istft(z)
    t2, x2 = msig.istft(z)
    assert x_ref.shape == tuple(x2.shape)
    assert_close(x2, x_ref)


@pytest.mark.parametrize(
    "perm,freq_axis,time_axis",
    [((0, 1, 2, 3), -2, -1), ((0, 1, 3, 2), -1, -2), ((2, 0, 1, 3), 0, -1), ((2, 3, 0, 1), 0, 1),
     ((3, 2, 0, 1), 1, 0), ((0, 3, 1, 2), 3, 1), ((0, 2, 3, 1), 1, 2), ((0, 3, 2, 1), 2, 1)],
)
@pytest.mark.parametrize("nperseg", [256, 200])
def test_istft_arbitrary_axes(rng, perm, freq_axis, time_axis, nperseg):
    x = make_sig(rng, (2, 3, 1024))
    _, _, z = sps.stft(x.astype(np.float64), nperseg=nperseg)
    z = np.transpose(z.astype(np.complex64), perm)
    _, x_ref = sps.istft(z, nperseg=nperseg, freq_axis=freq_axis, time_axis=time_axis)
    t_got, x_got = msig.istft(z, nperseg=nperseg, freq_axis=freq_axis, time_axis=time_axis)
    assert tuple(x_got.shape) == x_ref.shape
    out_time_ax = (time_axis % z.ndim) - (1 if (freq_axis % z.ndim) < (time_axis % z.ndim) else 0)
    assert len(t_got) == x_got.shape[out_time_ax]
    assert_close(x_got, x_ref)


def test_istft_axis_and_dtype_validation(rng):
    x = make_sig(rng, (2, 1024))
    _, _, z = sps.stft(x, nperseg=128)
    z = z.astype(np.complex64)
    with pytest.raises(ValueError, match="at least 2d"):
        msig.istft(np.ones(16, dtype=np.complex64))
    with pytest.raises(ValueError, match="differing"):
        msig.istft(z, freq_axis=-1, time_axis=-1)
    with pytest.raises(ValueError, match="differing"):
        msig.istft(z, freq_axis=1, time_axis=-2)
    with pytest.raises(IndexError):
        msig.istft(z, freq_axis=5, time_axis=-1)
    z128 = z.astype(np.complex128)
    with msig.config_context(float64="strict"):
        with pytest.raises(TypeError, match="strict"):
            msig.istft(z128, nperseg=128)
    with msig.config_context(float64="downcast", warn_on_downcast=True):
        with pytest.warns(msig.DowncastWarning):
            msig.istft(z128, nperseg=128)


def test_istft_memory_layouts_bit_identical(rng):
    """Equivalent NumPy / torch layouts of one spectrogram give bit-identical istft outputs
    (the reference's tests/test_spectral.py:395-423)."""
    import warnings

    x = make_sig(rng, (2, 3, 2048))
    _, _, z_sp = sps.stft(x.astype(np.float64), nperseg=256)
    z_sp = z_sp.astype(np.complex64)
    _, x_ref = sps.istft(z_sp, nperseg=256)
    t_base, y_base = msig.istft(z_sp, nperseg=256)
    t_base, y_base = t_base.cpu().numpy(), y_base.cpu().numpy()
    assert_close(y_base, x_ref)
    z_ro = z_sp.copy()
    z_ro.setflags(write=False)
    variants = [
        (np.ascontiguousarray(z_sp), {}),
        (np.ascontiguousarray(np.swapaxes(z_sp, -2, -1)), {"time_axis": -2, "freq_axis": -1}),
        (np.asfortranarray(z_sp), {}),
        (np.transpose(z_sp, (2, 0, 1, 3)), {"freq_axis": 0, "time_axis": -1}),
        (z_sp.astype(np.complex128), {}),
        (z_ro, {}),
        (torch.from_numpy(np.ascontiguousarray(z_sp)), {}),
        (torch.from_numpy(np.ascontiguousarray(z_sp)).cuda(), {}),
        (torch.from_numpy(np.ascontiguousarray(np.swapaxes(z_sp, -2, -1))).cuda().transpose(-2, -1),
         {}),
    ]
    for arr, kw in variants:
        for _ in range(2):  # the second CUDA call runs the cached plan
            with warnings.catch_warnings():
                warnings.simplefilter("ignore", msig.DowncastWarning)
                t_got, y_got = msig.istft(arr, nperseg=256, **kw)
            np.testing.assert_array_equal(t_got.cpu().numpy(), t_base)
            np.testing.assert_array_equal(y_got.cpu().numpy(), y_base)


def test_istft_strided_reversed_and_broadcast_views(rng):
    """Sliced, reversed and broadcast views match scipy (the reference's
    tests/test_spectral.py:426-441), as NumPy views and as torch CUDA views."""
    x = make_sig(rng, (3, 2048))
    _, _, z = sps.stft(x.astype(np.float64), nperseg=256)
    z = z.astype(np.complex64)
    zt = torch.from_numpy(np.ascontiguousarray(z)).cuda()
    views = [
        (z[:, :, ::2], zt[:, :, ::2]),
        (z[:, :, ::-1], zt.flip(-1)),
        (np.ascontiguousarray(z)[:, :, ::-1], None),
        (np.broadcast_to(z[:1], (4,) + z.shape[1:]), zt[:1].expand((4,) + z.shape[1:])),
        (z[::2, 3:, 1:-1], zt[::2, 3:, 1:-1]),
    ]
    for view, tview in views:
        _, x_ref = sps.istft(view, nperseg=256, nfft=256)
        for arr in (view, tview) if tview is not None else (view,):
            _, x_got = msig.istft(arr, nperseg=256, nfft=256)
            assert tuple(x_got.shape) == x_ref.shape
            assert_close(x_got, x_ref)


def test_stft_istft_roundtrip_ours(rng):
    x = make_sig(rng, (4096,))
    f, t, z = msig.stft(x, nperseg=256)
    t2, x2 = msig.istft(z, nperseg=256)
    x2 = x2.cpu().numpy()[: len(x)]
    np.testing.assert_allclose(x2, x, rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize(
    "nperseg,noverlap,rows,n",
    [(256, 128, 3, 8000), (1024, 512, 2, 60000), (512, 400, 2, 30000), (128, 27, 4, 7000),
     (64, 60, 2, 5000), (2048, 1024, 1, 50000), (4096, 3000, 1, 60000), (2, 1, 2, 300),
     (512, 256, 5, 600), (16, 8, 3, 100), (4096, 2048, 2, 70000)],
)
def test_fused_istft_matches_scipy(rng, nperseg, noverlap, rows, n):
    """Fused inverse FFT + overlap-add + normalisation vs float64 scipy.istft, including hops
    that do not divide nperseg, team ranges crossing rows and many frames per row."""
    x = rng.standard_normal((rows, n))
    _, _, z = sps.stft(x, nperseg=nperseg, noverlap=noverlap)
    _, x_ref = sps.istft(z, nperseg=nperseg, noverlap=noverlap)
    _, x_got = msig.istft(z.astype(np.complex64), nperseg=nperseg, noverlap=noverlap)
    assert tuple(x_got.shape) == x_ref.shape
    assert_close(x_got, x_ref, rtol=1e-4, atol_frac=1e-5)


def test_fused_istft_bin_count_mismatch(rng):
    """Fewer or more bins than nperseg/2+1 (zero-padded / truncated, as the reference)."""
    x = rng.standard_normal(6000)
    _, _, z = sps.stft(x, nperseg=256)
    for zz in (z[:100], np.concatenate([z, np.ones((7, z.shape[1]))], axis=0)):
        _, x_ref = sps.istft(zz, nperseg=256, nfft=256, input_onesided=True)
        _, x_got = msig.istft(zz.astype(np.complex64), nperseg=256, nfft=256)
        assert_close(x_got, x_ref, rtol=1e-4, atol_frac=1e-5)


def test_fused_istft_roundtrip_large(rng):
    """stft -> istft round trip through the fused kernels on a 16 x 2^18 batch."""
    x = rng.standard_normal((16, 1 << 18)).astype(np.float32)
    _, _, z = msig.stft(x, nperseg=1024, noverlap=512)
    _, x2 = msig.istft(z, nperseg=1024, noverlap=512)
    err = float((x2[:, : x.shape[1]].cpu() - torch.from_numpy(x)).abs().max())
    assert err < 1e-5 * float(np.abs(x).max()) * 10, err


@pytest.mark.parametrize("nperseg,noverlap", [(64, 16), (256, 128), (1024, 768), (4096, 2048),
                                              (512, 0)])
@pytest.mark.parametrize("mode", ["psd", "stft"])
def test_spectral_detrend_frames_match_scipy(rng, nperseg, noverlap, mode):
    """Constant detrend applied as a low-bin spectral correction in the frame kernels (hann
    window: three non-zero DFT bins), on data with a large DC offset, against float64 scipy and
    against the time-domain detrend kernels."""
    from mlx_signal_b200 import _kernels

    x = (rng.standard_normal((3, 20000)) + 5.0).astype(np.float32)
    if mode == "psd":
        f_ref, t_ref, s_ref = sps.spectrogram(x.astype(np.float64), window="hann",
                                              nperseg=nperseg, noverlap=noverlap)
        f, t, s = msig.spectrogram(x, window="hann", nperseg=nperseg, noverlap=noverlap)
    else:
        f_ref, t_ref, s_ref = sps.stft(x.astype(np.float64), window="hann", nperseg=nperseg,
                                       noverlap=noverlap, detrend="constant")
        f, t, s = msig.stft(x, window="hann", nperseg=nperseg, noverlap=noverlap,
                            detrend="constant")
    assert tuple(s.shape) == s_ref.shape
    assert_close(s, s_ref, rtol=1e-4, atol_frac=1e-5)
    # same frames through the time-domain detrend kernel
    win = msig.spectral.device_vector(
        (msig.windows._window_np("hann", nperseg)
         * (np.sqrt(1.0 / (msig.windows._window_np("hann", nperseg) ** 2).sum()) if mode == "psd"
            else 1.0 / msig.windows._window_np("hann", nperseg).sum())).astype(np.float32))
    hop = nperseg - noverlap
    ext = nperseg // 2 if mode == "stft" else 0
    n_ext = x.shape[1] + 2 * ext
    n_total = n_ext + ((-(n_ext - nperseg) % hop) % nperseg if mode == "stft" else 0)
    kind = "power" if mode == "psd" else "stft"
    low = _kernels.window_low_spectrum(win.cpu().numpy(), nperseg)
    assert low is not None
    wd = torch.from_numpy(low[0]).cuda()
    xt = torch.from_numpy(x).cuda()
    a = _kernels.frames(kind, xt, win, nperseg, nperseg, hop, 1, True, ext=ext,
                        ext_mode="zeros" if ext else None, n_total=n_total, wdft=wd)
    b = _kernels.frames(kind, xt, win, nperseg, nperseg, hop, 1, True, ext=ext,
                        ext_mode="zeros" if ext else None, n_total=n_total)
    # both detrend forms carry an error ~ eps * |mean| * |DFT(w)_0| on the lowest bins (the
    # spectral one from cancellation in the DC bin, the time-domain one from the rounded mean)
    assert float((a - b).abs().max()) <= 1e-5 * float(b.abs().max())


@pytest.mark.parametrize("fn", ["stft", "spectrogram"])
def test_memoised_setup_repeats(rng, fn):
    """Repeat calls with one argument set reuse the memoised setup: each call matches scipy on its
    own data; the returned axis vectors belong to the caller; nperseg > n keeps warning."""
    kw = {"nperseg": 128, "fs": 8.0, "axis": 0}
    for _ in range(3):
        x = make_sig(rng, (700, 3))
        out = getattr(msig, fn)(torch.from_numpy(x).cuda(), **kw)
        ref = getattr(sps, fn)(x.astype(np.float64), **kw)
        for a, b in zip(out, ref):
            assert_close(a, b)
        out[0].fill_(-1.0)
        out[1].fill_(-1.0)
    xs = torch.from_numpy(make_sig(rng, (100,))).cuda()
    for _ in range(2):
        with pytest.warns(UserWarning, match="nperseg"):
            getattr(msig, fn)(xs, nperseg=256)


def test_istft_plan_repeats_and_warns(rng, monkeypatch):
    from mlx_signal_b200 import spectral

    built = []

    class Counting(spectral._IstftPlan):
        def __init__(self, *a, **k):
            built.append(1)
            super().__init__(*a, **k)

    monkeypatch.setattr(spectral, "_IstftPlan", Counting)
    spectral._ISTFT_PLANS.clear()
    for _ in range(3):
        x = make_sig(rng, (2, 5000))
        _, _, z = sps.stft(x.astype(np.float64), nperseg=256)
        zt = torch.from_numpy(z.astype(np.complex64)).cuda()
        t, xr = msig.istft(zt, nperseg=256)
        _, x_ref = sps.istft(z, nperseg=256)
        # N-d input: the time vector follows the output time axis (as in the reference)
        assert_close(t, np.arange(x_ref.shape[-1], dtype=np.float64))
        assert_close(xr, x_ref)
        t.fill_(-1.0)
    # one plan, built by the first call and found by the two repeats under the call's full key
    assert len(built) == 1
    assert [k[0] for k in spectral._ISTFT_PLANS] == ["istft"]
    # boxcar with no overlap and no boundary padding gaps -> NOLA fails on every call
    z = torch.from_numpy(sps.stft(make_sig(rng, (4096,)), window=("tukey", 0.0), nperseg=256,
                                  noverlap=0)[2].astype(np.complex64)).cuda()
    for _ in range(2):
        with pytest.warns(UserWarning, match="NOLA"):
            msig.istft(z, window=("tukey", 0.9), nperseg=256, noverlap=0)


# 50%-overlap per-frame kernel (k_frames_half): boundary extension, padding, detrend variants
@pytest.mark.parametrize("nperseg", [64, 256, 1024, 2048, 4096])
@pytest.mark.parametrize("boundary,padded", [("zeros", True), ("even", True), ("odd", False),
                                             ("constant", True), (None, False), (None, True)])
def test_half_overlap_stft_matches_scipy(rng, nperseg, boundary, padded):
    n = 3 * nperseg + 37
    x = make_sig(rng, (3, n))
    x[1] += 3.0  # a DC offset exercises the detrend variants
    for detrend in (False, "constant"):
        kw = dict(nperseg=nperseg, boundary=boundary, padded=padded, detrend=detrend)
        f_ref, t_ref, z_ref = sps.stft(x.astype(np.float64), **kw)
        f, t, z = msig.stft(x, **kw)
        assert tuple(z.shape) == z_ref.shape
        assert_close(t, t_ref)
        assert_close(z, z_ref)


@pytest.mark.parametrize("nperseg", [64, 512, 1024, 4096])
@pytest.mark.parametrize("detrend", [False, "constant"])
@pytest.mark.parametrize("mode", ["psd", "complex", "magnitude"])
def test_half_overlap_spectrogram_matches_scipy(rng, nperseg, detrend, mode):
    x = make_sig(rng, (2, 5 * nperseg + 11))
    x[0] += 2.0
    kw = dict(nperseg=nperseg, noverlap=nperseg // 2, window="hann", detrend=detrend, mode=mode)
    f_ref, t_ref, s_ref = sps.spectrogram(x.astype(np.float64), **kw)
    f, t, s = msig.spectrogram(x, **kw)
    assert tuple(s.shape) == s_ref.shape
    assert_close(s, s_ref)
    # tukey window: its spectrum is not confined to low bins -> time-domain constant detrend
    kw["window"] = ("tukey", 0.25)
    f_ref, t_ref, s_ref = sps.spectrogram(x.astype(np.float64), **kw)
    assert_close(msig.spectrogram(x, **kw)[2], s_ref)


def test_half_overlap_single_and_odd_frame_counts(rng):
    for n, nperseg in [(1024, 1024), (1536, 1024), (2048, 1024), (64, 64), (97, 64)]:
        x = make_sig(rng, (2, n))
        for padded in (False, True):
            _, _, z_ref = sps.stft(x.astype(np.float64), nperseg=nperseg, boundary=None,
                                   padded=padded)
            _, _, z = msig.stft(x, nperseg=nperseg, boundary=None, padded=padded)
            assert tuple(z.shape) == z_ref.shape
            assert_close(z, z_ref)


# non-power-of-two nfft: fused Bluestein frame kernels
@pytest.mark.parametrize("kw", [{"nperseg": 1000}, {"nperseg": 300, "noverlap": 123},
                                {"nperseg": 77, "nfft": 81, "boundary": "even"},
                                {"nperseg": 500, "detrend": "constant", "boundary": None,
                                 "padded": False},
                                {"nperseg": 1500, "detrend": "linear", "boundary": "odd"},
                                {"nperseg": 6, "return_onesided": False}])
def test_bluestein_stft_matches_scipy(rng, kw):
    x = make_sig(rng, (2, 7001))
    x[1] += 2.0
    f_ref, t_ref, z_ref = sps.stft(x.astype(np.float64), **kw)
    f, t, z = msig.stft(x, **kw)
    assert tuple(z.shape) == z_ref.shape
    assert_close(f, f_ref)
    assert_close(z, z_ref)


@pytest.mark.parametrize("mode", ["psd", "complex", "magnitude", "phase"])
def test_bluestein_spectrogram_matches_scipy(rng, mode):
    x = make_sig(rng, (3, 9000))
    kw = dict(nperseg=441, noverlap=220, mode=mode, fs=44100.0)
    f_ref, t_ref, s_ref = sps.spectrogram(x.astype(np.float64), **kw)
    f, t, s = msig.spectrogram(x, **kw)
    assert tuple(s.shape) == s_ref.shape
    assert_close(s, s_ref, rtol=1e-3 if mode == "phase" else 1e-4)


# complex input, power-of-two nfft: fused two-sided complex-input frame kernels
@pytest.mark.parametrize("kw", [{}, {"nperseg": 1024, "boundary": "even"},
                                {"nperseg": 128, "noverlap": 96, "boundary": "odd"},
                                {"nperseg": 256, "boundary": "constant", "detrend": "constant"},
                                {"nperseg": 64, "nfft": 128, "boundary": None, "padded": False,
                                 "detrend": "linear"}])
def test_complex_input_stft_matches_scipy(rng, kw):
    x = (make_sig(rng, (2, 5001)) + 1j * make_sig(rng, (2, 5001))).astype(np.complex64)
    x[0] += 1.0 + 1.0j
    f_ref, t_ref, z_ref = sps.stft(x.astype(np.complex128), **kw)
    f, t, z = msig.stft(torch.from_numpy(x).cuda(), **kw)
    assert tuple(z.shape) == z_ref.shape
    assert_close(f, f_ref)
    assert_close(t, t_ref)
    assert_close(z, z_ref)


@pytest.mark.parametrize("mode", ["psd", "complex", "magnitude"])
def test_complex_input_spectrogram_matches_scipy(rng, mode):
    x = (make_sig(rng, (3, 6000)) + 1j * make_sig(rng, (3, 6000))).astype(np.complex64)
    kw = dict(nperseg=256, noverlap=64, mode=mode)
    f_ref, t_ref, s_ref = sps.spectrogram(x.astype(np.complex128), **kw)
    f, t, s = msig.spectrogram(x, **kw)
    assert tuple(s.shape) == s_ref.shape
    assert_close(s, s_ref)


@pytest.mark.parametrize("nperseg,nfft,noverlap", [(200, 256, 100), (256, 512, 128),
                                                  (256, 512, 200), (100, 128, 25),
                                                  (1000, 1024, 500)])
def test_istft_zero_padded_fused(rng, nperseg, nfft, noverlap):
    """nfft > nperseg (any nperseg): the fused kernel inverts nfft-point spectra and keeps the
    first nperseg samples of each frame; no composed-path warning."""
    import warnings

    x = make_sig(rng, (2, 6000))
    kw = dict(nperseg=nperseg, nfft=nfft, noverlap=noverlap)
    _, _, z = sps.stft(x.astype(np.float64), **kw)
    t_ref, x_ref = sps.istft(z, **kw)
    with warnings.catch_warnings():
        warnings.simplefilter("error", msig.FallbackWarning)
        warnings.simplefilter("ignore", msig.DowncastWarning)
        t2, x2 = msig.istft(z, **kw)
    assert x_ref.shape == tuple(x2.shape)
    assert len(t2) == x_ref.shape[-1]  # (scipy's t of an N-d input has the first axis' length)
    assert_close(x2, x_ref)


@pytest.mark.parametrize("kw", [{}, {"nperseg": 128, "noverlap": 96}, {"nperseg": 200,
                                                                       "nfft": 256}])
def test_istft_two_sided_complex_fused(rng, kw):
    """Two-sided spectra of a complex signal: fused complex inverse + overlap-add, complex64
    output equal to scipy's."""
    import warnings

    x = (make_sig(rng, (3000,)) + 1j * make_sig(rng, (3000,))).astype(np.complex128)
    _, _, z = sps.stft(x, return_onesided=False, **kw)
    _, x_ref = sps.istft(z, input_onesided=False, **kw)
    with warnings.catch_warnings():
        warnings.simplefilter("error", msig.FallbackWarning)
        warnings.simplefilter("ignore", msig.DowncastWarning)
        _, x2 = msig.istft(z, input_onesided=False, **kw)
    assert x2.is_complex() and x_ref.shape == tuple(x2.shape)
    assert_close(x2, x_ref)


@pytest.mark.parametrize("kw", [{"nperseg": 8192}, {"nperseg": 8192, "noverlap": 6000},
                                {"nperseg": 8192, "detrend": "constant"}])
def test_stft_spectrogram_nfft_8192_fused(rng, kw):
    import warnings

    x = make_sig(rng, (2, 1 << 16))
    _, _, z_ref = sps.stft(x.astype(np.float64), **kw)
    _, _, s_ref = sps.spectrogram(x.astype(np.float64), window="hann", **kw)
    with warnings.catch_warnings():
        warnings.simplefilter("error", msig.FallbackWarning)
        _, _, z = msig.stft(x, **kw)
        _, _, s = msig.spectrogram(x, window="hann", **kw)
    assert_close(z, z_ref)
    assert_close(s, s_ref)


@pytest.mark.parametrize("nperseg,nfft,noverlap", [(1000, None, 500), (300, None, 200),
                                                  (100, 150, 60), (999, 1500, None),
                                                  (37, None, 20)])
def test_istft_non_power_of_two_fused(rng, nperseg, nfft, noverlap):
    """A non-power-of-two nfft runs the chirp-z fused inverse (no composed-path warning)."""
    import warnings

    x = make_sig(rng, (2, 5000))
    kw = dict(nperseg=nperseg, nfft=nfft, noverlap=noverlap)
    _, _, z = sps.stft(x.astype(np.float64), **kw)
    _, x_ref = sps.istft(z, **kw)
    with warnings.catch_warnings():
        warnings.simplefilter("error", msig.FallbackWarning)
        warnings.simplefilter("ignore", msig.DowncastWarning)
        _, x2 = msig.istft(z, **kw)
    assert x_ref.shape == tuple(x2.shape)
    assert_close(x2, x_ref)
