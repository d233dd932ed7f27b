"""GPU parity of the long-FFT consumers against float64 scipy: hilbert, resample (Fourier
method), fftconvolve, oaconvolve (ports of the reference's filtering / resampling / convolution
tests). Lengths cover both the three-pass kernels (power-of-two transforms >= 2^12) and the
composed cuFFT path (other lengths)."""

import numpy as np
import pytest
import scipy.signal as sps
import torch

import mlx_signal_b200 as msig

pytestmark = pytest.mark.gpu


def peak_err(got, ref):
    got = got.cpu().numpy() if isinstance(got, torch.Tensor) else np.asarray(got)
    return float(np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-30))


@pytest.mark.parametrize("n,N", [(1000, None), (1 << 14, None), (1 << 21, None), (5000, 1 << 13),
                                 (1 << 20, 1 << 21), (777, None)])
def test_hilbert_matches_scipy(rng, n, N):
    x = rng.standard_normal((2, n)).astype(np.float32)
    ref = sps.hilbert(x.astype(np.float64), N=N, axis=-1)
    got = msig.hilbert(x, N=N)
    assert got.dtype == torch.complex64 and tuple(got.shape) == ref.shape
    assert peak_err(got, ref) < 2e-6


@pytest.mark.parametrize("n,shape_axis", [(1 << 13, ((3, 1 << 13), -1)),
                                         (1 << 14, ((1 << 14, 2), 0)),
                                         (1 << 16, ((1, 1 << 16), -1))])
def test_hilbert_fused_chain(rng, monkeypatch, n, shape_axis):
    """Power-of-two lengths run sp_hilbert_c64 (forward three-pass transform, masked-spectrum
    untangle, inverse three-pass transform); the kernels are routed from 2^12 points here."""
    from mlx_signal_b200 import fft as bfft

    monkeypatch.setattr(bfft, "KERNEL_MIN_LOG2", 12)
    shape, axis = shape_axis
    x = rng.standard_normal(shape).astype(np.float32)
    ref = sps.hilbert(x.astype(np.float64), axis=axis)
    got = msig.hilbert(x, axis=axis)
    assert bfft.device_status() == 0
    assert tuple(got.shape) == ref.shape
    assert peak_err(got, ref) < 2e-6
    # the analytic signal of a cosine is the complex exponential
    t = np.arange(n)
    c = np.cos(2 * np.pi * 37 * t / n).astype(np.float32)
    assert peak_err(msig.hilbert(c), np.exp(2j * np.pi * 37 * t / n)) < 2e-6


def test_hilbert_axis_and_errors(rng):
    x = rng.standard_normal((4096, 3)).astype(np.float32)
    assert peak_err(msig.hilbert(x, axis=0), sps.hilbert(x.astype(np.float64), axis=0)) < 2e-6
    with pytest.raises(ValueError):
        msig.hilbert(x.astype(np.complex64))
    with pytest.raises(ValueError):
        msig.hilbert(x, N=0)


@pytest.mark.parametrize("n,num", [(1 << 14, 3000), (1 << 14, 1 << 15), (1000, 1500),
                                   (1001, 600), (1 << 21, 1 << 20), (1 << 20, 1 << 22)])
@pytest.mark.parametrize("window", [None, "hann"])
def test_resample_real_matches_scipy(rng, n, num, window):
    x = rng.standard_normal((2, n)).astype(np.float32)
    ref = sps.resample(x.astype(np.float64), num, axis=-1, window=window)
    got = msig.resample(x, num, axis=-1, window=window)
    assert tuple(got.shape) == ref.shape
    assert peak_err(got, ref) < 5e-6


@pytest.mark.parametrize("n,num", [(4096, 1000), (4096, 9000), (999, 1000), (1000, 999)])
def test_resample_complex_and_freq_domain(rng, n, num):
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    ref = sps.resample(x.astype(np.complex128), num)
    assert peak_err(msig.resample(x, num), ref) < 5e-6
    X = np.fft.fft(x.astype(np.complex128))
    ref_f = sps.resample(X, num, domain="freq")
    assert peak_err(msig.resample(X.astype(np.complex64), num, domain="freq"), ref_f) < 5e-6
    t = np.linspace(0, 1, n, endpoint=False)
    _, nt_ref = sps.resample(x.astype(np.complex128), num, t=t)
    _, nt = msig.resample(x, num, t=t)
    np.testing.assert_allclose(nt.cpu().numpy(), nt_ref, rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("n1,n2", [(1 << 20, 1 << 20), (1 << 21, 4097), (5000, 300), (300, 5000),
                                   (1 << 15, 1 << 12)])
@pytest.mark.parametrize("mode", ["full", "same", "valid"])
def test_fftconvolve_matches_scipy(rng, n1, n2, mode):
    a = rng.standard_normal(n1).astype(np.float32)
    b = rng.standard_normal(n2).astype(np.float32)
    ref = sps.fftconvolve(a.astype(np.float64), b.astype(np.float64), mode=mode)
    got = msig.fftconvolve(a, b, mode=mode)
    assert tuple(got.shape) == ref.shape
    assert peak_err(got, ref) < 5e-6


def test_fftconvolve_nd_complex_and_errors(rng):
    a = rng.standard_normal((3, 2000)).astype(np.float32)
    b = rng.standard_normal((1, 300)).astype(np.float32)
    ref = sps.fftconvolve(a.astype(np.float64), b.astype(np.float64), mode="same", axes=-1)
    assert peak_err(msig.fftconvolve(a, b, mode="same", axes=-1), ref) < 5e-6
    c = (rng.standard_normal((40, 50)) + 1j * rng.standard_normal((40, 50))).astype(np.complex64)
    d = rng.standard_normal((7, 9)).astype(np.float32)
    ref2 = sps.fftconvolve(c.astype(np.complex128), d.astype(np.float64))
    assert peak_err(msig.fftconvolve(c, d), ref2) < 5e-6
    with pytest.raises(ValueError):
        msig.fftconvolve(a, b[0])
    with pytest.raises(ValueError):
        msig.fftconvolve(a, b, mode="nope")


@pytest.mark.parametrize("n1,n2", [(1 << 20, 513), (100000, 2048), (3000, 3000), (257, 4096)])
@pytest.mark.parametrize("mode", ["full", "same", "valid"])
def test_oaconvolve_matches_scipy(rng, n1, n2, mode):
    a = rng.standard_normal((2, n1)).astype(np.float32)
    b = rng.standard_normal((2, n2)).astype(np.float32)
    ref = sps.oaconvolve(a.astype(np.float64), b.astype(np.float64), mode=mode, axes=-1)
    got = msig.oaconvolve(a, b, mode=mode, axes=-1)
    assert tuple(got.shape) == ref.shape
    assert peak_err(got, ref) < 5e-6


# fused overlap-save convolution: real rows, one shared filter of <= 2049 taps
@pytest.mark.parametrize("n1,n2", [(1 << 20, 1025), (100000, 1), (100000, 2), (70001, 64),
                                   (5000, 255), (5000, 256), (4099, 2049), (3000, 2049),
                                   (1, 1), (17, 5), (300, 1500)])
@pytest.mark.parametrize("mode", ["full", "same", "valid"])
@pytest.mark.parametrize("fn", ["fftconvolve", "oaconvolve"])
def test_fused_conv_matches_scipy(rng, n1, n2, mode, fn):
    a = rng.standard_normal((3, n1)).astype(np.float32)
    b = rng.standard_normal((1, n2)).astype(np.float32)
    if mode == "valid" and n1 < n2:
        a, b = a[:1], np.broadcast_to(b, (1, n2))
    ref = getattr(sps, fn)(a.astype(np.float64), b.astype(np.float64), mode=mode, axes=-1)
    got = getattr(msig, fn)(a, b, mode=mode, axes=-1)
    assert got.dtype == torch.float32 and tuple(got.shape) == ref.shape
    assert peak_err(got, ref) < 2e-6


def test_fused_conv_axis_swap_and_batch_edges(rng):
    # filter first (convolution commutes), non-last axis, torch CUDA input, 1-D
    x = rng.standard_normal((20000, 2)).astype(np.float32)
    h = rng.standard_normal((33, 1)).astype(np.float32)
    for mode in ("full", "same", "valid"):
        ref = sps.oaconvolve(x.astype(np.float64), h.astype(np.float64), mode=mode, axes=0)
        got = msig.oaconvolve(torch.from_numpy(x).cuda(), h, mode=mode, axes=0)
        assert tuple(got.shape) == ref.shape and peak_err(got, ref) < 2e-6
        ref = sps.fftconvolve(h.astype(np.float64), x.astype(np.float64), mode=mode, axes=0)
        got = msig.fftconvolve(h, x, mode=mode, axes=0)
        assert tuple(got.shape) == ref.shape and peak_err(got, ref) < 2e-6
    # 'same' centres on in1's shape on every axis, the batch axis included
    a = rng.standard_normal((1, 900)).astype(np.float32)
    b = rng.standard_normal((4, 50)).astype(np.float32)
    for fn in ("fftconvolve", "oaconvolve"):
        ref = getattr(sps, fn)(b.astype(np.float64), a.astype(np.float64), mode="same", axes=-1)
        got = getattr(msig, fn)(b, a, mode="same", axes=-1)
        assert tuple(got.shape) == ref.shape and peak_err(got, ref) < 2e-6
    a1 = rng.standard_normal(12345).astype(np.float32)
    h1 = rng.standard_normal(700).astype(np.float32)
    assert peak_err(msig.fftconvolve(a1, h1), np.convolve(a1.astype(np.float64), h1)) < 2e-6


def test_conv_ols_capi_windows(rng):
    """The C-ABI entry point writes exactly the requested window of the full convolution into a
    strided output, leaving the row padding untouched."""
    from mlx_signal_b200 import _lib
    from mlx_signal_b200._array import stream_handle

    lib = _lib.load()
    x = rng.standard_normal((2, 9000)).astype(np.float32)
    h = rng.standard_normal(129).astype(np.float32)
    full = np.stack([np.convolve(r.astype(np.float64), h) for r in x])
    xd, hd = torch.from_numpy(x).cuda(), torch.from_numpy(h).cuda()
    for j0, nout in [(0, 9128), (5, 100), (128, 8872), (9127, 1), (3000, 4000)]:
        out = torch.full((2, nout + 7), 7.0, device="cuda")
        _lib.check(lib.sp_conv_ols_f32(xd.data_ptr(), 2, 9000, 9000, hd.data_ptr(), 129, j0, nout,
                                       out.data_ptr(), nout + 7, stream_handle()), "conv")
        o = out.cpu().numpy()
        assert peak_err(torch.from_numpy(o[:, :nout]), full[:, j0 : j0 + nout]) < 2e-6
        assert np.all(o[:, nout:] == 7.0)


@pytest.mark.parametrize("n,num", [(1 << 14, 3 << 13), (3 << 13, 1 << 14), (5 << 13, 3 << 13),
                                   (3 << 13, 5 << 13), (1 << 15, 1 << 14), (1 << 14, 1 << 15),
                                   (3 << 13, 3 << 13), (15 << 13, 1 << 13)])
def test_resample_fused_matches_scipy(rng, monkeypatch, n, num):
    """Real input, no window: one sp_resample_f32 call (forward transform writing only the kept
    bins, unpaired-bin fix-up and num/n scale inside the inverse pretwist), power-of-two and
    odd-factor lengths, against float64 scipy."""
    from mlx_signal_b200 import fft as bfft

    monkeypatch.setattr(bfft, "RESAMPLE_MIN_LOG2", 12)
    assert bfft._resample_in_range(n, num)
    x = rng.standard_normal((2, n)).astype(np.float32)
    ref = sps.resample(x.astype(np.float64), num, axis=-1)
    got = msig.resample(x, num, axis=-1)
    assert tuple(got.shape) == ref.shape
    assert peak_err(got, ref) < 5e-6
    xt = np.ascontiguousarray(x.T)
    got0 = msig.resample(xt, num, axis=0)
    assert peak_err(got0, sps.resample(xt.astype(np.float64), num, axis=0)) < 5e-6
    assert bfft.device_status() == 0


def test_resample_fused_full_size(rng):
    """2^22 -> 3 2^20 samples through the default routing (both lengths on the kernels), with
    sample positions, against float64 scipy."""
    n, num = 1 << 22, 3 << 20
    x = rng.standard_normal(n).astype(np.float32)
    t = np.arange(n) * 1e-3
    got, nt = msig.resample(x, num, t=t)
    ref, nt_ref = sps.resample(x.astype(np.float64), num, t=t)
    assert peak_err(got, ref) < 5e-6
    np.testing.assert_allclose(nt.cpu().numpy(), nt_ref, rtol=1e-6)
