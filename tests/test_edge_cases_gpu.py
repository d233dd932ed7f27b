"""GPU edge cases after the reference's own regression tests: empty inputs and nperseg = 1
(tests/test_edge_cases.py:37-111), length-one FFT axes (:114-138, :331-346), 0-d inputs and the
0-d dtype policy (:311-320, :349-358), singleton convolution axes (:228-243), the dtype policy
through the public functions (tests/test_dispatch_dtypes.py:35-83), odd / prime / padded FFT
lengths (tests/test_fourstep.py:44-83), the long transforms the reference routes around its
Metal FFT (tests/test_metal_fft_workaround.py:16-96) and the Hilbert envelope
(tests/test_resample_hilbert.py:111-116). Every result must be a torch CUDA float32/complex64
tensor with scipy's shape; values against float64 scipy / numpy."""

import warnings

import numpy as np
import pytest
import scipy.signal as sps
import torch

import mlx_signal_b200 as msig
from _utils import as_np, assert_close, assert_cuda_f32

pytestmark = pytest.mark.gpu


def _rel(got, ref):
    """Max error relative to the peak of the reference (the reference's test_fourstep._rel)."""
    got = as_np(got)
    return float(np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-30))


# ---------------------------------------------------------------------------------------------
# empty inputs and nperseg = 1
# ---------------------------------------------------------------------------------------------


@pytest.mark.parametrize("func", ["welch", "csd", "coherence", "periodogram", "stft"])
@pytest.mark.parametrize("shape", [(0,), (3, 0)])
def test_empty_input_matches_scipy(func, shape, rng):
    x = np.zeros(shape, dtype=np.float32)
    y = rng.standard_normal(shape).astype(np.float32)
    args = (x, y) if func in ("csd", "coherence") else (x,)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        ref = getattr(sps, func)(*args)
        got = getattr(msig, func)(*args)
    assert len(got) == len(ref)
    for g, r in zip(got, ref):
        assert tuple(as_np(g).shape) == r.shape


def test_welch_nperseg_1_matches_scipy(rng):
    x = rng.standard_normal(64).astype(np.float32)
    f_ref, p_ref = sps.welch(x.astype(np.float64), nperseg=1)
    f, p = msig.welch(x, nperseg=1)
    assert_cuda_f32(p)
    np.testing.assert_allclose(as_np(f), f_ref)
    np.testing.assert_allclose(as_np(p), p_ref, rtol=1e-5)


def test_welch_nperseg_1_linear_detrend(rng):
    """Linear detrend of a single point is mean removal: an all-zero PSD, as scipy."""
    x = rng.standard_normal(64).astype(np.float32)
    _, p_ref = sps.welch(x.astype(np.float64), nperseg=1, detrend="linear")
    _, p = msig.welch(x, nperseg=1, detrend="linear")
    np.testing.assert_allclose(as_np(p), p_ref, rtol=1e-5, atol=1e-12)


def test_stft_nperseg_1_matches_scipy(rng):
    x = rng.standard_normal(32).astype(np.float32)
    f_ref, t_ref, z_ref = sps.stft(x.astype(np.float64), nperseg=1)
    f, t, z = msig.stft(x, nperseg=1)
    assert_cuda_f32(z, complex_ok=True)
    assert tuple(z.shape) == z_ref.shape
    np.testing.assert_allclose(as_np(t), t_ref)
    np.testing.assert_allclose(as_np(z), z_ref, rtol=1e-5, atol=1e-6)


def test_spectrogram_nperseg_1_matches_scipy(rng):
    x = rng.standard_normal(32).astype(np.float32)
    _, _, s_ref = sps.spectrogram(x.astype(np.float64), nperseg=1)
    _, _, s = msig.spectrogram(x, nperseg=1)
    assert tuple(s.shape) == s_ref.shape
    np.testing.assert_allclose(as_np(s), s_ref, rtol=1e-5, atol=1e-12)


def test_csd_nperseg_1_matches_scipy(rng):
    x = rng.standard_normal(48).astype(np.float32)
    y = rng.standard_normal(48).astype(np.float32)
    _, p_ref = sps.csd(x.astype(np.float64), y.astype(np.float64), nperseg=1)
    _, p = msig.csd(x, y, nperseg=1)
    np.testing.assert_allclose(as_np(p), p_ref, rtol=1e-5, atol=1e-7)


def test_periodogram_single_sample(rng):
    x = rng.standard_normal(1).astype(np.float32)
    f_ref, p_ref = sps.periodogram(x.astype(np.float64))
    f, p = msig.periodogram(x)
    assert tuple(p.shape) == p_ref.shape
    np.testing.assert_allclose(as_np(f), f_ref)
    np.testing.assert_allclose(as_np(p), p_ref, atol=1e-12)


# ---------------------------------------------------------------------------------------------
# FFT lengths: one, odd, prime, padded
# ---------------------------------------------------------------------------------------------


def test_fft_length_one_axis(rng):
    x = rng.standard_normal((4, 1)).astype(np.float32)
    np.testing.assert_allclose(as_np(msig.fft.rfft(x, axis=-1)), np.fft.rfft(x, axis=-1),
                               rtol=1e-6)
    xc = x.astype(np.complex64)
    np.testing.assert_allclose(as_np(msig.fft.fft(xc, axis=-1)), np.fft.fft(xc, axis=-1),
                               rtol=1e-6)
    back = msig.fft.irfft(msig.fft.rfft(x, axis=-1), n=1, axis=-1)
    np.testing.assert_allclose(as_np(back), np.fft.irfft(np.fft.rfft(x, axis=-1), n=1, axis=-1),
                               rtol=1e-6, atol=1e-7)
    # along axis 0 of a (1, 4) array as well
    np.testing.assert_allclose(as_np(msig.fft.rfft(x.T, axis=0)), np.fft.rfft(x.T, axis=0),
                               rtol=1e-6)


@pytest.mark.parametrize("n", [999_999, 999_983])  # odd composite; prime
def test_rfft_odd_and_prime_lengths(rng, n):
    x = rng.standard_normal(n).astype(np.float32)
    ref = np.fft.rfft(x.astype(np.float64))
    got = msig.fft.rfft(x)
    assert got.dtype == torch.complex64 and tuple(got.shape) == ref.shape
    assert _rel(got, ref) < 5e-6
    back = msig.fft.irfft(got, n=n)
    assert _rel(back, x.astype(np.float64)) < 5e-6


def test_rfft_padding_and_truncation(rng):
    x = rng.standard_normal(1_500_000).astype(np.float32)
    for n in (1 << 21, 1 << 20):  # pad up onto the kernels; truncate
        ref = np.fft.rfft(x.astype(np.float64), n=n)
        assert _rel(msig.fft.rfft(x, n=n), ref) < 5e-6


def test_large_fft_values_via_wrappers(rng):
    x = rng.standard_normal(1 << 21).astype(np.float32)
    assert _rel(msig.fft.rfft(x), np.fft.rfft(x.astype(np.float64))) < 5e-6
    x2 = rng.standard_normal(3_000_000).astype(np.float32)
    assert _rel(msig.fft.rfft(x2), np.fft.rfft(x2.astype(np.float64))) < 5e-6


# ---------------------------------------------------------------------------------------------
# long transforms through the consumers (the reference's Metal-FFT "hole" sizes)
# ---------------------------------------------------------------------------------------------


def test_fftconvolve_long_signal_long_filter(rng):
    """2^20 samples x 4097 taps: longer than the fused overlap-save filter limit."""
    a = rng.standard_normal(1 << 20).astype(np.float32)
    b = rng.standard_normal(4097).astype(np.float32)
    ref = sps.fftconvolve(a.astype(np.float64), b.astype(np.float64))
    out = msig.fftconvolve(a, b)
    assert_cuda_f32(out)
    assert_close(out, ref, rtol=2e-4, atol_frac=3e-5)


def test_fftconvolve_two_long_inputs(rng):
    a = rng.standard_normal(600_000).astype(np.float32)
    b = rng.standard_normal(600_000).astype(np.float32)
    ref = sps.fftconvolve(a.astype(np.float64), b.astype(np.float64))
    assert_close(msig.fftconvolve(a, b), ref, rtol=2e-4, atol_frac=3e-5)


def test_resample_and_hilbert_600k(rng):
    x = rng.standard_normal(600_000).astype(np.float32)
    assert_close(msig.resample(x, 300_000), sps.resample(x.astype(np.float64), 300_000),
                 rtol=2e-4, atol_frac=3e-5)
    assert_close(msig.hilbert(x), sps.hilbert(x.astype(np.float64)), rtol=2e-4, atol_frac=3e-5)


def test_welch_large_nfft(rng):
    """nperseg 2^20 zero-padded to nfft 2^21 (beyond the framed kernels: composed path)."""
    x = rng.standard_normal(1 << 21).astype(np.float32)
    _, p_ref = sps.welch(x.astype(np.float64), nperseg=1 << 20, nfft=1 << 21)
    _, p = msig.welch(x, nperseg=1 << 20, nfft=1 << 21)
    assert_cuda_f32(p)
    assert_close(p, p_ref, rtol=2e-4, atol_frac=3e-5)


def test_hilbert_envelope():
    t = np.arange(4096, dtype=np.float32) / 4096
    x = (1.0 + 0.5 * np.sin(2 * np.pi * 3 * t)) * np.sin(2 * np.pi * 400 * t)
    env = np.abs(as_np(msig.hilbert(x.astype(np.float32))))
    expected = 1.0 + 0.5 * np.sin(2 * np.pi * 3 * t)
    np.testing.assert_allclose(env[64:-64], expected[64:-64], atol=2e-2)


# ---------------------------------------------------------------------------------------------
# dtype policy through the public functions, 0-d inputs, singleton convolution axes
# ---------------------------------------------------------------------------------------------


def test_float64_downcast_warns_and_matches(rng):
    x = rng.standard_normal(65536)  # float64
    with msig.config_context(warn_on_downcast=True):
        with pytest.warns(msig.DowncastWarning):
            _, p = msig.welch(x, nperseg=256)
    assert_cuda_f32(p)
    assert_close(p, sps.welch(x, nperseg=256)[1])


def test_float64_strict_raises(rng):
    x = rng.standard_normal(65536)
    with msig.config_context(float64="strict"):
        with pytest.raises(TypeError, match="float64"):
            msig.welch(x, nperseg=256)
        with pytest.raises(TypeError, match="strict"):
            msig.stft(torch.from_numpy(x), nperseg=256)


def test_complex128_and_float64_consumers(rng):
    x = rng.standard_normal(65536) + 1j * rng.standard_normal(65536)
    with msig.config_context(warn_on_downcast=True):
        with pytest.warns(msig.DowncastWarning):
            out = msig.hilbert(np.abs(x))  # float64 input
        with pytest.warns(msig.DowncastWarning):
            z = msig.fft.fft(x)
    assert out.dtype == torch.complex64 and z.dtype == torch.complex64


def test_int_input_accepted(rng):
    x = rng.integers(-100, 100, size=70000).astype(np.int32)
    out = msig.fftconvolve(x, x[:100])
    assert_cuda_f32(out)
    ref = sps.fftconvolve(x.astype(np.float64), x[:100].astype(np.float64))
    assert_close(out, ref, rtol=1e-4)


def test_list_input_silent(rng):
    x = [float(v) for v in rng.standard_normal(100)]
    with warnings.catch_warnings():
        warnings.simplefilter("error", msig.DowncastWarning)
        f, p = msig.periodogram(x)
    assert_cuda_f32(p)
    assert_close(p, sps.periodogram(np.asarray(x))[1])


def test_torch_cuda_passthrough(rng):
    x = torch.from_numpy(rng.standard_normal(65536).astype(np.float32)).cuda()
    f, p = msig.welch(x, nperseg=1024)
    assert_cuda_f32(p)
    assert_close(p, sps.welch(x.double().cpu().numpy(), nperseg=1024)[1])


def test_zero_dim_inputs():
    out = msig.fftconvolve(np.float32(2.0), np.float32(3.0))
    ref = sps.fftconvolve(np.float32(2.0), np.float32(3.0))
    assert tuple(out.shape) == np.shape(ref) == ()
    np.testing.assert_allclose(as_np(out), ref)
    with msig.config_context(float64="strict"):
        with pytest.raises(TypeError, match="strict"):
            msig.fftconvolve(np.array(2.0), np.array(3.0))
    with msig.config_context(float64="downcast", warn_on_downcast=True):
        with pytest.warns(msig.DowncastWarning):
            assert tuple(msig.oaconvolve(np.array(2.0), np.float32(3.0)).shape) == ()


@pytest.mark.parametrize("conv", [msig.fftconvolve, msig.oaconvolve])
def test_convolve_singleton_axes(conv, rng):
    """(1, n) with axes=[0]: every convolution axis has length 1, so the result is a product."""
    a = rng.standard_normal((1, 3)).astype(np.float32)
    b = rng.standard_normal((1, 3)).astype(np.float32)
    ref = sps.fftconvolve(a, b, axes=[0])
    out = conv(a, b, axes=[0])
    assert tuple(out.shape) == ref.shape
    np.testing.assert_allclose(as_np(out), ref, rtol=1e-5)
    with pytest.raises(ValueError, match="integers"):
        conv(a, b, axes=0.5)
