"""GPU parity: welch / periodogram / csd / coherence against float64 scipy.signal.

Cases follow the reference's tests/test_spectral.py (WELCH_CASES, multidim axes, csd
mean/median/broadcast/unequal, coherence, grouped-vs-scipy over nperseg 64..2048) and add the
float32 accuracy bar (max relative error <= 1e-5 on bins above 1e-6 of the peak).
"""

import numpy as np
import pytest
import scipy.signal as sps
import torch

import mlx_signal_b200 as msig
from _utils import assert_close, assert_cuda_f32, make_sig, rel_err_bins

pytestmark = pytest.mark.gpu

WELCH_CASES = [
    {},
    {"nperseg": 128},
    {"nperseg": 128, "noverlap": 96},
    {"nperseg": 128, "window": "hamming"},
    {"nperseg": 100, "window": ("tukey", 0.25)},
    {"nperseg": 128, "detrend": "linear"},
    {"nperseg": 128, "detrend": False},
    {"nperseg": 128, "scaling": "spectrum"},
    {"nperseg": 128, "return_onesided": False},
    {"nperseg": 128, "average": "median"},
    {"nperseg": 128, "nfft": 256},
    {"nperseg": 129, "noverlap": 37, "fs": 250.0},
]


@pytest.mark.parametrize("n", [1024, 999, 4093])
@pytest.mark.parametrize("case", WELCH_CASES)
def test_welch_matches_scipy(rng, n, case):
    x = make_sig(rng, (n,))
    f_ref, p_ref = sps.welch(x.astype(np.float64), **case)
    f, p = msig.welch(x, **case)
    assert_cuda_f32(f)
    assert_cuda_f32(p)
    assert_close(f, f_ref)
    assert_close(p, p_ref)


def test_welch_array_window(rng):
    x = make_sig(rng, (2048,))
    w = sps.get_window("hann", 200)
    f_ref, p_ref = sps.welch(x.astype(np.float64), window=w)
    f, p = msig.welch(x, window=w.astype(np.float32))
    assert_close(f, f_ref)
    assert_close(p, p_ref)


@pytest.mark.parametrize(
    "shape,axis", [((3, 2000), -1), ((2000, 3), 0), ((2, 3, 1500), -1), ((2, 1500, 3), 1)]
)
def test_welch_multidim(rng, shape, axis):
    x = make_sig(rng, shape)
    f_ref, p_ref = sps.welch(x.astype(np.float64), nperseg=128, axis=axis)
    f, p = msig.welch(x, nperseg=128, axis=axis)
    assert p_ref.shape == tuple(p.shape)
    assert_close(p, p_ref)
    assert_close(f, f_ref)


def test_welch_complex_input_switches_twosided(rng):
    x = make_sig(rng, (2048,), complex_=True)
    f_ref, p_ref = sps.welch(x.astype(np.complex128), nperseg=256)
    f, p = msig.welch(x, nperseg=256)
    assert_close(f, f_ref)
    assert_close(p, p_ref)


def test_welch_short_signal_warns(rng):
    x = make_sig(rng, (100,))
    with pytest.warns(UserWarning, match="nperseg"):
        f_ref, p_ref = sps.welch(x.astype(np.float64))
    with pytest.warns(UserWarning, match="nperseg"):
        f, p = msig.welch(x)
    assert_close(f, f_ref)
    assert_close(p, p_ref)


@pytest.mark.parametrize(
    "case",
    [{}, {"nfft": 4096}, {"nfft": 1000}, {"scaling": "spectrum"}, {"detrend": False},
     {"window": "hann"}, {"return_onesided": False}],
)
def test_periodogram_matches_scipy(rng, case):
    x = make_sig(rng, (2048,))
    f_ref, p_ref = sps.periodogram(x.astype(np.float64), **case)
    f, p = msig.periodogram(x, **case)
    assert_close(f, f_ref)
    assert_close(p, p_ref)


def test_periodogram_array_window(rng):
    x = make_sig(rng, (1024,))
    w = sps.get_window("blackman", 1024)
    _, p_ref = sps.periodogram(x.astype(np.float64), window=w)
    _, p = msig.periodogram(x, window=w)
    assert_close(p, p_ref)
    _, p_t = msig.periodogram(x, window=torch.from_numpy(w).float().cuda())  # device window
    assert_close(p_t, p_ref)


def test_parseval_periodogram(rng):
    x = make_sig(rng, (4096,))
    fs = 10.0
    f, p = msig.periodogram(x, fs=fs, detrend=False)
    total = float(p.double().sum().item()) * fs / len(x)
    np.testing.assert_allclose(total, np.mean(x.astype(np.float64) ** 2), rtol=1e-3)


@pytest.mark.parametrize("average", ["mean", "median"])
def test_csd_matches_scipy(rng, average):
    x = make_sig(rng, (4096,))
    y = make_sig(rng, (4096,))
    f_ref, p_ref = sps.csd(x.astype(np.float64), y.astype(np.float64), nperseg=256,
                           average=average)
    f, p = msig.csd(x, y, nperseg=256, average=average)
    assert p.dtype == torch.complex64
    assert_close(f, f_ref)
    assert_close(p, p_ref, rtol=2e-4)


def test_csd_broadcast(rng):
    x = make_sig(rng, (4096,))
    y = make_sig(rng, (3, 4096))
    f_ref, p_ref = sps.csd(x.astype(np.float64), y.astype(np.float64), nperseg=256)
    f, p = msig.csd(x, y, nperseg=256)
    assert p_ref.shape == tuple(p.shape)
    assert_close(p, p_ref, rtol=2e-4)


def test_csd_unequal_lengths(rng):
    x = make_sig(rng, (3000,))
    y = make_sig(rng, (4096,))
    f_ref, p_ref = sps.csd(x.astype(np.float64), y.astype(np.float64), nperseg=256)
    f, p = msig.csd(x, y, nperseg=256)
    assert_close(p, p_ref, rtol=2e-4)


def test_coherence_matches_scipy(rng):
    x = make_sig(rng, (8192,))
    y = 0.5 * x + 0.5 * make_sig(rng, (8192,))
    f_ref, c_ref = sps.coherence(x.astype(np.float64), y.astype(np.float64), nperseg=256)
    f, c = msig.coherence(x, y, nperseg=256)
    assert_close(c, c_ref, rtol=1e-3)
    assert float(c.min()) >= 0.0 and float(c.max()) <= 1.0


@pytest.mark.parametrize("nperseg", [64, 128, 256, 512, 1024, 2048])
@pytest.mark.parametrize("detrend", [False, "constant"])
def test_grouped_spectral_means_match_scipy(rng, nperseg, detrend):
    n = nperseg + (nperseg // 2) * 130
    x = make_sig(rng, (16, n))
    y = (0.5 * x + 0.5 * make_sig(rng, (16, n))).astype(np.float32)
    x64, y64 = x.astype(np.float64), y.astype(np.float64)
    _, pw = msig.welch(x, nperseg=nperseg, detrend=detrend)
    _, pw_ref = sps.welch(x64, nperseg=nperseg, detrend=detrend)
    assert_close(pw, pw_ref, rtol=1e-4)
    assert rel_err_bins(pw, pw_ref) < 1e-5
    _, pc = msig.csd(x, y, nperseg=nperseg, detrend=detrend)
    _, pc_ref = sps.csd(x64, y64, nperseg=nperseg, detrend=detrend)
    assert_close(pc, pc_ref, rtol=2e-4)
    _, co = msig.coherence(x, y, nperseg=nperseg, detrend=detrend)
    _, co_ref = sps.coherence(x64, y64, nperseg=nperseg, detrend=detrend)
    assert_close(co, co_ref, rtol=1e-3)


def test_grouped_spectral_reduces_peak_memory(rng):
    """Segment sums accumulate in the kernels: no per-frame spectra are materialised (the
    reference's tests/test_spectral.py:233-263 bounds, 64 x 2^19, nperseg 1024, where per-frame
    coherence spectra would take ~512 MiB)."""
    x = torch.from_numpy(rng.standard_normal((64, 1 << 19)).astype(np.float32)).cuda()
    y = torch.from_numpy(rng.standard_normal((64, 1 << 19)).astype(np.float32)).cuda()
    msig.welch(x, nperseg=1024)
    msig.coherence(x, y, nperseg=1024)
    msig.csd(x, y, nperseg=1024)
    torch.cuda.synchronize()

    def peak_mib(fn):
        base = torch.cuda.memory_allocated()
        torch.cuda.reset_peak_memory_stats()
        out = fn()
        torch.cuda.synchronize()
        peak = (torch.cuda.max_memory_allocated() - base) / (1 << 20)
        del out
        return peak

    welch_mib = peak_mib(lambda: msig.welch(x, nperseg=1024))
    coh_mib = peak_mib(lambda: msig.coherence(x, y, nperseg=1024))
    csd_mib = peak_mib(lambda: msig.csd(x, y, nperseg=1024))
    assert welch_mib < 16.0, f"welch peak memory too high: {welch_mib:.1f} MiB"
    assert coh_mib < 64.0, f"coherence peak memory too high: {coh_mib:.1f} MiB"
    assert csd_mib < 64.0, f"csd peak memory too high: {csd_mib:.1f} MiB"


def test_grouped_single_group_and_nonlast_axis(rng):
    x_many = make_sig(rng, (2048, 320))
    y_many = (0.5 * x_many + 0.5 * make_sig(rng, (2048, 320))).astype(np.float32)
    assert_close(msig.welch(x_many, nperseg=64)[1],
                 sps.welch(x_many.astype(np.float64), nperseg=64)[1], rtol=1e-4)
    assert_close(msig.coherence(x_many, y_many, nperseg=64)[1],
                 sps.coherence(x_many.astype(np.float64), y_many.astype(np.float64),
                               nperseg=64)[1], rtol=1e-3)
    x_ax = make_sig(rng, (2, 4096, 3))
    y_ax = (0.5 * x_ax + 0.5 * make_sig(rng, (2, 4096, 3))).astype(np.float32)
    x64, y64 = x_ax.astype(np.float64), y_ax.astype(np.float64)
    assert_close(msig.welch(x_ax, nperseg=128, axis=1)[1],
                 sps.welch(x64, nperseg=128, axis=1)[1], rtol=1e-4)
    assert_close(msig.csd(x_ax, y_ax, nperseg=128, axis=1)[1],
                 sps.csd(x64, y64, nperseg=128, axis=1)[1], rtol=2e-4)
    assert_close(msig.coherence(x_ax, y_ax, nperseg=128, axis=1)[1],
                 sps.coherence(x64, y64, nperseg=128, axis=1)[1], rtol=1e-3)


@pytest.mark.parametrize("nfft", [1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096])
@pytest.mark.parametrize("detrend", [False, "constant", "linear"])
def test_fused_welch_every_size(rng, nfft, detrend):
    """Every fused team-FFT plan (single-thread up to 32 points, 8..128-thread teams above),
    with nperseg < nfft zero padding and an odd hop."""
    nperseg = max(1, nfft - nfft // 4)
    hop = max(1, nperseg // 2 - 1) if nperseg > 2 else 1
    x = make_sig(rng, (3, 40 * nfft + 7))
    kw = dict(nperseg=nperseg, noverlap=nperseg - hop, nfft=nfft, detrend=detrend)
    # an absolute floor at the signal power: degenerate cases (linear detrend of 1-2 samples)
    # are exactly zero in float64 and fp32 rounding noise here
    floor = 1e-5 * float(np.mean(x.astype(np.float64) ** 2))
    _, p = msig.welch(x, **kw)
    _, p_ref = sps.welch(x.astype(np.float64), **kw)
    np.testing.assert_allclose(p.cpu().numpy(), p_ref, rtol=1e-4,
                               atol=max(1e-5 * np.abs(p_ref).max(), floor))
    _, c = msig.csd(x, x[::-1].copy(), **kw)
    _, c_ref = sps.csd(x.astype(np.float64), x[::-1].astype(np.float64), **kw)
    np.testing.assert_allclose(c.cpu().numpy(), c_ref, rtol=2e-4,
                               atol=max(2e-5 * np.abs(c_ref).max(), floor))


def test_welch_accuracy_bar(rng):
    """48 kHz multi-tone channels, hann, nperseg 1024 / 50%: <= 1e-5 relative on bins above
    1e-6 of the peak (scaled-down channel count of the 64 x 2^20 workload)."""
    fs = 48000.0
    C, n = 8, 1 << 18
    t = np.arange(n) / fs
    x = rng.standard_normal((C, n))
    for c in range(C):
        for _ in range(rng.integers(1, 5)):
            x[c] += rng.uniform(0.1, 2.0) * np.sin(2 * np.pi * rng.uniform(0, fs / 2) * t)
    x = x.astype(np.float32)
    _, p = msig.welch(x, fs=fs, nperseg=1024, noverlap=512)
    _, p_ref = sps.welch(x.astype(np.float64), fs=fs, nperseg=1024, noverlap=512)
    err = max(rel_err_bins(p[c], p_ref[c]) for c in range(C))
    assert err <= 1e-5, err


def test_torch_inputs_and_outputs(rng):
    x = make_sig(rng, (4, 8192))
    xt = torch.from_numpy(x).cuda()
    f1, p1 = msig.welch(x, nperseg=512)
    f2, p2 = msig.welch(xt, nperseg=512)
    torch.testing.assert_close(p1, p2, rtol=0, atol=0)
    f3, p3 = msig.welch(torch.from_numpy(x), nperseg=512)
    torch.testing.assert_close(p1, p3, rtol=0, atol=0)


@pytest.mark.parametrize("window", ["hann", "hamming", "blackman", "boxcar", ("tukey", 0.25)])
@pytest.mark.parametrize("offset", [0.0, 0.5, 4.0])
def test_half_overlap_detrend_paths(rng, window, offset):
    """50%-overlap fused welch: the spectral constant detrend (sparse window spectra) and the
    time-domain one (tukey) against scipy, including signals with a DC offset."""
    from mlx_signal_b200 import _kernels

    nper = 1024
    x = (rng.standard_normal((4, 40 * nper)) + offset).astype(np.float32)
    w = sps.get_window(window, nper)
    sparse = _kernels.window_low_spectrum((w * 0.01).astype(np.float32), nper) is not None
    assert sparse == (window != ("tukey", 0.25))
    _, p = msig.welch(x, window=window, nperseg=nper, fs=48000.0)
    _, p_ref = sps.welch(x.astype(np.float64), window=window, nperseg=nper, fs=48000.0)
    assert_close(p, p_ref, rtol=1e-4, atol_frac=1e-5)
    err = max(rel_err_bins(p[c], p_ref[c]) for c in range(4))
    assert err <= (1e-5 if offset <= 0.5 else 1e-4), err


def test_spectral_and_time_domain_detrend_agree(rng):
    from mlx_signal_b200 import _kernels

    nper = 256
    x = torch.from_numpy(rng.standard_normal((8, 300 * nper)).astype(np.float32)).cuda()
    w = sps.get_window("hann", nper).astype(np.float32)
    low = _kernels.window_low_spectrum(w, nper)
    assert low is not None and low[1] == 2
    wt = torch.from_numpy(w).cuda()
    a = _kernels.welch_mean(x, wt, nper, nper, nper // 2, 1, True)
    b = _kernels.welch_mean(x, wt, nper, nper, nper // 2, 1, True,
                            wdft=torch.from_numpy(low[0]).cuda())
    torch.testing.assert_close(a, b, rtol=2e-5, atol=1e-6 * float(a.max()))


@pytest.mark.parametrize("nperseg", [16, 64, 256, 512, 1024, 2048, 4096])
@pytest.mark.parametrize("detrend", ["constant", False])
def test_half_overlap_cross_spectra_match_scipy(rng, nperseg, detrend):
    """50%-overlap csd / coherence (the fused half-block kernel: window in the first butterfly
    stage, spectral or time-domain constant detrend) against float64 scipy, with a DC offset."""
    from mlx_signal_b200 import _kernels

    n = 40 * nperseg
    x = (rng.standard_normal((3, n)) + 2.0).astype(np.float32)
    y = (0.6 * np.roll(x, 7, axis=-1) + 0.4 * rng.standard_normal((3, n)) - 1.0).astype(np.float32)
    kw = dict(nperseg=nperseg, fs=100.0, detrend=detrend)
    _, c_ref = sps.csd(x.astype(np.float64), y.astype(np.float64), **kw)
    _, c = msig.csd(x, y, **kw)
    assert rel_err_bins(c, c_ref) <= 1e-5
    _, h_ref = sps.coherence(x.astype(np.float64), y.astype(np.float64), **kw)
    _, h = msig.coherence(x, y, **kw)
    assert_close(h, h_ref, rtol=1e-4, atol_frac=1e-5)
    if detrend == "constant":  # the time-domain detrend variant of the same kernel
        w = msig.spectral.device_vector(
            (msig.windows._window_np("hann", nperseg)
             * np.sqrt(1.0 / (100.0 * (msig.windows._window_np("hann", nperseg) ** 2).sum())))
            .astype(np.float32))
        ct = _kernels.cross_mean("csd", torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda(), w,
                                 nperseg, nperseg, nperseg // 2, 1, True)
        assert rel_err_bins(ct, c_ref) <= 1e-5


@pytest.mark.parametrize("shape,axis", [((3, 4096), -1), ((4096, 2), 0)])
def test_welch_plan_cache_repeats(rng, shape, axis):
    """Repeated calls with one argument set reuse a cached plan: every call still matches scipy,
    the frequency vector is a fresh tensor each time, and other arguments get their own plan."""
    for rep in range(3):
        x = make_sig(rng, shape)
        f, p = msig.welch(torch.from_numpy(x).cuda(), fs=4.0, nperseg=256, axis=axis)
        f_ref, p_ref = sps.welch(x.astype(np.float64), fs=4.0, nperseg=256, axis=axis)
        assert_close(f, f_ref)
        assert_close(p, p_ref)
        f.fill_(-1.0)  # the caller owns the returned vector
    x = make_sig(rng, shape)
    f, p = msig.welch(torch.from_numpy(x).cuda(), fs=4.0, nperseg=128, axis=axis,
                      scaling="spectrum")
    f_ref, p_ref = sps.welch(x.astype(np.float64), fs=4.0, nperseg=128, axis=axis,
                             scaling="spectrum")
    assert_close(f, f_ref)
    assert_close(p, p_ref)


def test_welch_plan_cache_keeps_warnings_and_errors(rng):
    xt = torch.from_numpy(make_sig(rng, (100,))).cuda()
    for _ in range(2):
        with pytest.warns(UserWarning, match="nperseg"):
            msig.welch(xt)
    xt = torch.from_numpy(make_sig(rng, (1024,))).cuda()
    msig.welch(xt, detrend=False, nperseg=128)
    with pytest.raises(ValueError):
        msig.welch(xt, detrend=0, nperseg=128)


# non-power-of-two nfft: fused Bluestein (chirp-z) kernels
@pytest.mark.parametrize("kw", [{"nperseg": 1000}, {"nperseg": 768, "noverlap": 100},
                                {"nperseg": 100, "nfft": 150}, {"nperseg": 3},
                                {"nperseg": 2047, "detrend": "linear"},
                                {"nperseg": 999, "detrend": False, "scaling": "spectrum"},
                                {"nperseg": 300, "return_onesided": False},
                                {"nperseg": 129, "window": ("tukey", 0.3), "fs": 44.1}])
def test_bluestein_welch_matches_scipy(rng, kw):
    x = make_sig(rng, (3, 20000))
    x[0] += 1.5
    f_ref, p_ref = sps.welch(x.astype(np.float64), **kw)
    f, p = msig.welch(x, **kw)
    assert tuple(p.shape) == p_ref.shape
    assert_close(f, f_ref)
    assert_close(p, p_ref)
    assert rel_err_bins(p, p_ref) <= 1e-5


def test_bluestein_welch_accuracy_bar(rng):
    """64 x 2^18 channels, nperseg 1000: the 1e-5 bar on bins above 1e-6 of the peak."""
    x = make_sig(rng, (64, 1 << 18))
    f_ref, p_ref = sps.welch(x.astype(np.float64), fs=48000, nperseg=1000)
    f, p = msig.welch(torch.from_numpy(x).cuda(), fs=48000, nperseg=1000)
    assert rel_err_bins(p, p_ref) <= 1e-5


# complex input, power-of-two nfft: fused two-sided complex-input kernel
@pytest.mark.parametrize("kw", [{}, {"nperseg": 1024}, {"nperseg": 128, "noverlap": 100},
                                {"nperseg": 64, "nfft": 256, "detrend": "linear"},
                                {"nperseg": 4096, "detrend": False, "scaling": "spectrum"},
                                {"nperseg": 1}, {"nperseg": 32, "window": ("tukey", 0.5)}])
def test_complex_input_welch_matches_scipy(rng, kw):
    x = (make_sig(rng, (3, 9000)) + 1j * make_sig(rng, (3, 9000))).astype(np.complex64)
    x[1] += 0.5 - 2j
    f_ref, p_ref = sps.welch(x.astype(np.complex128), fs=2.0, **kw)
    f, p = msig.welch(torch.from_numpy(x).cuda(), fs=2.0, **kw)
    assert tuple(p.shape) == p_ref.shape and p.dtype == torch.float32
    assert_close(f, f_ref)
    assert_close(p, p_ref)


def test_complex_input_welch_axis_and_rows(rng):
    x = (make_sig(rng, (4000, 2, 3)) + 1j * make_sig(rng, (4000, 2, 3))).astype(np.complex64)
    f_ref, p_ref = sps.welch(x.astype(np.complex128), nperseg=256, axis=0)
    f, p = msig.welch(x, nperseg=256, axis=0)
    assert tuple(p.shape) == p_ref.shape
    assert_close(p, p_ref)


@pytest.mark.parametrize("kw", [{"nperseg": 1000}, {"nperseg": 300, "noverlap": 250},
                                {"nperseg": 77, "nfft": 99, "detrend": "linear"},
                                {"nperseg": 1500, "detrend": False, "scaling": "spectrum"}])
def test_bluestein_csd_coherence_match_scipy(rng, kw):
    x = make_sig(rng, (2, 30000))
    y = (0.6 * np.roll(x, 5, axis=-1) + 0.4 * make_sig(rng, (2, 30000))).astype(np.float32)
    f_ref, c_ref = sps.csd(x.astype(np.float64), y.astype(np.float64), **kw)
    f, c = msig.csd(x, y, **kw)
    assert tuple(c.shape) == c_ref.shape
    assert_close(c, c_ref, rtol=2e-4)
    kc = {k: v for k, v in kw.items() if k != "scaling"}
    f_ref, h_ref = sps.coherence(x.astype(np.float64), y.astype(np.float64), **kc)
    f, h = msig.coherence(x, y, **kc)
    assert tuple(h.shape) == h_ref.shape
    assert_close(h, h_ref, rtol=1e-3)


# average='median': column-median kernel over the per-frame spectra
@pytest.mark.parametrize("n,kw", [(20000, {"nperseg": 128}), (20000, {"nperseg": 256}),
                                  (4096, {"nperseg": 512, "noverlap": 0}),
                                  (3000, {"nperseg": 1000}), (9000, {"nperseg": 64,
                                                                     "detrend": "linear"})])
def test_median_welch_csd_match_scipy(rng, n, kw):
    x = make_sig(rng, (3, n))
    y = (0.5 * x + 0.5 * make_sig(rng, (3, n))).astype(np.float32)
    f_ref, p_ref = sps.welch(x.astype(np.float64), average="median", **kw)
    f, p = msig.welch(x, average="median", **kw)
    assert tuple(p.shape) == p_ref.shape
    assert_close(p, p_ref)
    f_ref, c_ref = sps.csd(x.astype(np.float64), y.astype(np.float64), average="median", **kw)
    f, c = msig.csd(x, y, average="median", **kw)
    assert_close(c, c_ref, rtol=2e-4)


def test_median_ties_and_even_counts(rng):
    """Repeated values (zero signal, constant rows) and even / odd segment counts."""
    x = np.zeros((2, 1024 * 9), np.float32)
    x[1] = 1.0
    for nperseg in (1024, 2048):  # 17 and 8 segments
        f_ref, p_ref = sps.welch(x.astype(np.float64), nperseg=nperseg, average="median",
                                 detrend=False)
        f, p = msig.welch(x, nperseg=nperseg, average="median", detrend=False)
        assert_close(p, p_ref)


@pytest.mark.parametrize("kw", [{"nperseg": 256}, {"nperseg": 1024, "detrend": "linear"},
                                {"nperseg": 64, "nfft": 128, "noverlap": 16}])
def test_complex_csd_and_coherence_match_scipy(rng, kw):
    x = (make_sig(rng, (2, 12000)) + 1j * make_sig(rng, (2, 12000))).astype(np.complex64)
    y = (0.5 * np.roll(x, 3, axis=-1) + 0.5 * make_sig(rng, (2, 12000))).astype(np.complex64)
    f_ref, c_ref = sps.csd(x.astype(np.complex128), y.astype(np.complex128), **kw)
    f, c = msig.csd(x, y, **kw)
    assert tuple(c.shape) == c_ref.shape and c.dtype == torch.complex64
    assert_close(f, f_ref)
    assert_close(c, c_ref, rtol=2e-4)
    xr = make_sig(rng, (2, 12000))  # real x with complex y (scipy wants the two-sided request)
    f_ref, c_ref = sps.csd(xr.astype(np.float64), y.astype(np.complex128),
                           return_onesided=False, **kw)
    assert_close(msig.csd(xr, y, return_onesided=False, **kw)[1], c_ref, rtol=2e-4)
    f_ref, h_ref = sps.coherence(x.astype(np.complex128), y.astype(np.complex128), **kw)
    f, h = msig.coherence(x, y, **kw)
    assert_close(h, h_ref, rtol=1e-3)


def _welch_f64_chunked(x, nperseg, chunk_segments=1 << 15):
    """float64 scipy welch of a long 1-D signal, computed over blocks of whole segments (the
    mean of periodograms is a weighted mean of the blocks' means): bounded host memory."""
    hop = nperseg // 2
    nseg = (x.shape[0] - nperseg) // hop + 1
    total = None
    for s0 in range(0, nseg, chunk_segments):
        s1 = min(nseg, s0 + chunk_segments)
        part = x[s0 * hop : (s1 - 1) * hop + nperseg].astype(np.float64)
        f, p = sps.welch(part, nperseg=nperseg)
        total = p * (s1 - s0) if total is None else total + p * (s1 - s0)
    return f, total / nseg


@pytest.mark.parametrize("nperseg", [256, 2048])
def test_welch_long_channel_segment_sums(nperseg):
    """One 2^26-sample channel in a single row: at nperseg 256 (524287 segments, ~37 per team
    over four CTA waves, register blocks folded into a shared-memory total) and at nperseg 2048
    (65535 segments over 592 single-team CTAs, ~112 per team: plain FP32 register sums, within
    the 128-segment limit of that form). Both stay within 1e-5 relative of float64 scipy on bins
    above 1e-6 of the peak, for a tone-plus-noise input with a large dynamic range."""
    n = 1 << 26
    g = torch.Generator(device="cuda")
    g.manual_seed(26)
    x = torch.randn(n, generator=g, device="cuda")
    t = torch.arange(n, device="cuda", dtype=torch.float64)
    x += (3.0 * torch.sin(2 * np.pi * 0.123 * t)).float()
    _, p = msig.welch(x, nperseg=nperseg)
    xh = x.cpu().numpy()
    _, pref = _welch_f64_chunked(xh, nperseg)
    assert rel_err_bins(p.cpu().numpy(), pref) <= 1e-5


def test_welch_block_totals_at_large_nperseg():
    """64 x 2^21 at nperseg 4096: 65472 segments over 296 single-team CTAs put ~222 segments in
    each team's range, past the 128-segment limit of plain register sums, so the nfft >= 2048
    kernel that folds register blocks into a shared-memory total runs; rows from both ends of
    the grid match float64 scipy within 1e-5 on bins above 1e-6 of the peak."""
    g = torch.Generator(device="cuda")
    g.manual_seed(21)
    x = torch.randn((64, 1 << 21), generator=g, device="cuda")
    t = torch.arange(1 << 21, device="cuda", dtype=torch.float64)
    x[::7] += (2.0 * torch.sin(2 * np.pi * 0.0371 * t)).float()
    _, p = msig.welch(x, nperseg=4096)
    rows = [0, 7, 40, 63]
    xh = x[rows].cpu().numpy().astype(np.float64)
    _, pref = sps.welch(xh, nperseg=4096)
    assert rel_err_bins(p[rows].cpu().numpy(), pref) <= 1e-5


def _csd_f64_chunked(x, y, nperseg, chunk_segments=1 << 15):
    """float64 scipy csd of two long 1-D signals over blocks of whole segments (as above)."""
    hop = nperseg // 2
    nseg = (x.shape[0] - nperseg) // hop + 1
    total = None
    for s0 in range(0, nseg, chunk_segments):
        s1 = min(nseg, s0 + chunk_segments)
        sl = slice(s0 * hop, (s1 - 1) * hop + nperseg)
        f, p = sps.csd(x[sl].astype(np.float64), y[sl].astype(np.float64), nperseg=nperseg)
        total = p * (s1 - s0) if total is None else total + p * (s1 - s0)
    return f, total / nseg


def test_cross_long_channel_segment_sums():
    """csd and coherence of one 2^26-sample pair at nperseg 256 (524287 segments in one row):
    each team's FP32 sums are flushed into FP64 partial slots every 32 segments, and both stay
    within 1e-5 relative of float64 scipy on bins above 1e-6 of the peak (tone plus noise, y a
    delayed noisy copy of x)."""
    n = 1 << 26
    g = torch.Generator(device="cuda")
    g.manual_seed(27)
    x = torch.randn(n, generator=g, device="cuda")
    t = torch.arange(n, device="cuda", dtype=torch.float64)
    x += (3.0 * torch.sin(2 * np.pi * 0.123 * t)).float()
    y = 0.7 * torch.roll(x, 17) + 0.3 * torch.randn(n, generator=g, device="cuda")
    _, pxy = msig.csd(x, y, nperseg=256)
    _, coh = msig.coherence(x, y, nperseg=256)
    xh, yh = x.cpu().numpy(), y.cpu().numpy()
    _, ref_xy = _csd_f64_chunked(xh, yh, 256)
    assert rel_err_bins(pxy.cpu().numpy(), ref_xy) <= 1e-5
    _, ref_xx = _welch_f64_chunked(xh, 256)
    _, ref_yy = _welch_f64_chunked(yh, 256)
    ref_coh = np.abs(ref_xy) ** 2 / (ref_xx * ref_yy)
    assert rel_err_bins(coh.cpu().numpy(), ref_coh) <= 1e-5


@pytest.mark.parametrize("kw", [
    {"nperseg": 8192},
    {"nperseg": 8192, "detrend": "linear"},
    {"nperseg": 8192, "detrend": False, "window": "hamming"},
    {"nperseg": 8192, "noverlap": 2048},
    {"nperseg": 6000, "nfft": 8192},
    {"nperseg": 8192, "average": "median"},
])
def test_welch_nfft_8192_fused(rng, kw):
    """nfft = 8192 runs the fused kernels (one 512-thread team per CTA), no composed path."""
    import warnings

    x = make_sig(rng, (3, 1 << 17))
    _, p_ref = sps.welch(x.astype(np.float64), **kw)
    with warnings.catch_warnings():
        warnings.simplefilter("error", msig.FallbackWarning)
        _, p = msig.welch(x, **kw)
    assert_close(p, p_ref)
    if kw.get("average") != "median":
        assert rel_err_bins(p, p_ref) <= 1e-5


@pytest.mark.parametrize("noverlap", [None, 1000])
def test_csd_coherence_nfft_8192_fused(rng, noverlap):
    import warnings

    x = make_sig(rng, (2, 1 << 17))
    y = 0.6 * np.roll(x, 9, axis=-1) + 0.4 * make_sig(rng, (2, 1 << 17))
    kw = {"nperseg": 8192, "noverlap": noverlap}
    _, c_ref = sps.csd(x.astype(np.float64), y.astype(np.float64), **kw)
    _, h_ref = sps.coherence(x.astype(np.float64), y.astype(np.float64), **kw)
    with warnings.catch_warnings():
        warnings.simplefilter("error", msig.FallbackWarning)
        _, c = msig.csd(x, y, **kw)
        _, h = msig.coherence(x, y, **kw)
    assert_close(c, c_ref, rtol=2e-4)
    assert_close(h, h_ref, rtol=1e-3)


@pytest.mark.parametrize("kw", [{"nperseg": 3000}, {"nperseg": 4000, "detrend": "linear"},
                                {"nperseg": 2500, "nfft": 3500}])
def test_bluestein_long_nfft_fused(rng, kw):
    """Non-power-of-two nfft in (2048, 4096]: the chirp-z kernels on 8192-point transforms."""
    import warnings

    x = make_sig(rng, (2, 1 << 16))
    _, p_ref = sps.welch(x.astype(np.float64), **kw)
    _, _, z_ref = sps.stft(x[0].astype(np.float64), **kw)
    with warnings.catch_warnings():
        warnings.simplefilter("error", msig.FallbackWarning)
        _, p = msig.welch(x, **kw)
        _, _, z = msig.stft(x[0], **kw)
    assert_close(p, p_ref)
    assert rel_err_bins(p, p_ref) <= 1e-5
    assert_close(z, z_ref)
