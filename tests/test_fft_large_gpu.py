"""GPU parity: the three-pass long FFTs against float64 numpy (ports of the reference's
tests/test_fourstep.py: sizes 2^21..2^23, both directions, batched/axis, padding, structured
signals, round trip), plus the largest sizes and the error word."""

import ctypes

import numpy as np
import pytest
import torch

from mlx_signal_b200 import fft as bfft

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def kernels_from_2p12(monkeypatch):
    """These tests exercise the kernels at every length the C-ABI takes (the public routing
    sends complex lengths below 2^22, and odd-factor forward transforms, to cuFFT)."""
    monkeypatch.setattr(bfft, "KERNEL_MIN_LOG2", 12)
    monkeypatch.setattr(bfft, "ODD_FORWARD", True)


def _rel(got, ref):
    got = got.cpu().numpy() if isinstance(got, torch.Tensor) else got
    return float(np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-30))


@pytest.mark.parametrize("e", [12, 16, 21, 22, 23])
@pytest.mark.parametrize("inverse", [False, True])
def test_fft3_matches_numpy(rng, e, inverse):
    n = 1 << e
    x = (rng.standard_normal((2, n)) + 1j * rng.standard_normal((2, n))).astype(np.complex64)
    got = (bfft.ifft if inverse else bfft.fft)(x)
    ref = (np.fft.ifft if inverse else np.fft.fft)(x.astype(np.complex128), axis=-1)
    for i in range(2):
        assert _rel(got[i], ref[i]) < 2e-6


@pytest.mark.parametrize("e", [13, 22, 23, 24])
def test_rfft_irfft_large(rng, e):
    n = 1 << e
    x = rng.standard_normal(n).astype(np.float32)
    ref = np.fft.rfft(x.astype(np.float64))
    got = bfft.rfft(x)
    assert tuple(got.shape) == ref.shape
    assert _rel(got, ref) < 5e-6
    back = bfft.irfft(got, n=n)
    assert _rel(back, x) < 5e-6


@pytest.mark.parametrize("e", [25, 26])
def test_fft3_largest_sizes(rng, e):
    n = 1 << e
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    assert _rel(bfft.fft(x), np.fft.fft(x.astype(np.complex128))) < 2e-6


def test_batched_and_axis(rng):
    n = 1 << 21
    x = rng.standard_normal((3, n)).astype(np.float32)
    ref = np.fft.rfft(x.astype(np.float64), axis=-1)
    assert _rel(bfft.rfft(x, axis=-1), ref) < 5e-6
    xt = np.ascontiguousarray(x.T)
    ref0 = np.fft.rfft(xt.astype(np.float64), axis=0)
    got0 = bfft.rfft(xt, axis=0)
    assert tuple(got0.shape) == ref0.shape
    assert _rel(got0, ref0) < 5e-6


def test_padding_semantics(rng):
    x = rng.standard_normal(1_500_000).astype(np.float32)
    n = 1 << 21
    assert _rel(bfft.rfft(x, n=n), np.fft.rfft(x.astype(np.float64), n=n)) < 5e-6


def test_structured_signals():
    n = 1 << 21
    t = np.arange(n)
    tone = np.exp(2j * np.pi * (98765 / n) * t).astype(np.complex64)
    imp = np.zeros(n, np.complex64)
    imp[4097] = 1.0
    for x in (tone, imp):
        assert _rel(bfft.fft(x), np.fft.fft(x.astype(np.complex128))) < 2e-6


def test_roundtrip(rng):
    n = 1 << 21
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    assert _rel(bfft.ifft(bfft.fft(x)), x) < 2e-6


def test_non_pow2_lengths_use_composed_path(rng):
    x = rng.standard_normal(600_000).astype(np.float32)
    assert _rel(bfft.rfft(x), np.fft.rfft(x.astype(np.float64))) < 5e-6


def test_error_word_clear_after_transform(rng):
    from mlx_signal_b200 import _lib

    n = 1 << 21
    x = torch.from_numpy((rng.standard_normal(n) + 0j).astype(np.complex64)).cuda()
    out = torch.empty_like(x)
    lib = _lib.load()
    ws = torch.empty(int(lib.sp_fft_workspace_size(n, 1)), dtype=torch.uint8, device="cuda")
    assert lib.sp_fft_c64(x.data_ptr(), out.data_ptr(), 1, n, 0, ws.data_ptr(), ws.numel(),
                          torch.cuda.current_stream().cuda_stream) == 0
    off = ctypes.c_int64(0)
    assert lib.sp_fft_error_word(ws.data_ptr(), n, 1, ctypes.byref(off)) == 0
    torch.cuda.synchronize()
    assert int(ws[off.value : off.value + 4].view(torch.int32).item()) == 0


def test_bounded_wait_runs_out_and_reports_timeout(rng, monkeypatch):
    """Failure detection without a fault: with a poll limit of 0 every tile-copy wait runs out,
    each CTA records SP_ERR_TIMEOUT in the error word, drains its own copies (bounded) and
    returns; the host reads the word through the C-ABI and through the Python watchdog, and the
    next transform with the default limit is clean and correct."""
    from mlx_signal_b200 import _lib

    lib = _lib.load()
    n = 1 << 16
    x = torch.from_numpy((rng.standard_normal(n) + 1j * rng.standard_normal(n))
                         .astype(np.complex64)).cuda()
    out = torch.empty_like(x)
    ws = torch.zeros(int(lib.sp_fft_workspace_size(n, 1)), dtype=torch.uint8, device="cuda")
    off = ctypes.c_int64(0)
    assert lib.sp_fft_error_word(ws.data_ptr(), n, 1, ctypes.byref(off)) == 0
    stream = torch.cuda.current_stream().cuda_stream
    assert bfft.device_status() == 0 and lib.sp_fft_sticky_error(0) == 0
    prev = lib.sp_fft_set_wait_limit(0)
    try:
        assert lib.sp_fft_c64(x.data_ptr(), out.data_ptr(), 1, n, 0, ws.data_ptr(), ws.numel(),
                              stream) == 0
        torch.cuda.synchronize()
        assert int(ws[off.value : off.value + 4].view(torch.int32).item()) == _lib.SP_ERR_TIMEOUT
        # the process-wide sticky word (mapped pinned host memory) holds it too until cleared
        assert lib.sp_fft_sticky_error(0) == _lib.SP_ERR_TIMEOUT
        with pytest.raises(bfft.DeviceWaitTimeout):
            bfft.device_status()
        assert lib.sp_fft_sticky_error(0) == 0
        # the Python path: the watchdog raises on the host once the transform has run
        monkeypatch.setattr(bfft, "KERNEL_MIN_LOG2", 12)
        xr = torch.from_numpy(rng.standard_normal(2 * n).astype(np.float32)).cuda()
        bfft.rfft(xr)
        with pytest.raises(bfft.DeviceWaitTimeout) as info:
            bfft.device_status()
        assert info.value.status == _lib.SP_ERR_TIMEOUT
    finally:
        lib.sp_fft_set_wait_limit(prev)
    assert bfft.device_status() == 0  # nothing outstanding
    # the context stays usable: default limit, clean word, correct result
    assert lib.sp_fft_c64(x.data_ptr(), out.data_ptr(), 1, n, 0, ws.data_ptr(), ws.numel(),
                          stream) == 0
    torch.cuda.synchronize()
    assert int(ws[off.value : off.value + 4].view(torch.int32).item()) == 0
    ref = np.fft.fft(x.cpu().numpy().astype(np.complex128))
    assert _rel(out, ref) < 5e-6
    xr = torch.from_numpy(rng.standard_normal(2 * n).astype(np.float32)).cuda()
    got = bfft.rfft(xr)
    assert bfft.device_status() == 0
    assert _rel(got, np.fft.rfft(xr.cpu().numpy().astype(np.float64))) < 5e-6


def test_routing_below_the_threshold_uses_cufft(rng, monkeypatch):
    monkeypatch.setattr(bfft, "KERNEL_MIN_LOG2", 20)
    assert not bfft._pow2_in_range(1 << 19) and bfft._pow2_in_range(1 << 20)
    x = rng.standard_normal(1 << 14).astype(np.float32)
    assert _rel(bfft.rfft(x), np.fft.rfft(x.astype(np.float64))) < 5e-6


@pytest.mark.parametrize("c", [3, 5, 7, 9, 11, 13, 15])
def test_rfft_irfft_odd_factor_lengths(rng, c):
    """n = 2 C 2^12: C decimated branches through one batch of packed 2^12-point transforms and
    the radix-C untangle/combine and fold/pretwist kernels, against float64 numpy."""
    n = 2 * c * (1 << 12)
    assert bfft._real_split(n) == (c, 12) and bfft._real_in_range(n)
    x = rng.standard_normal((2, n)).astype(np.float32)
    ref = np.fft.rfft(x.astype(np.float64), axis=-1)
    got = bfft.rfft(x)
    assert tuple(got.shape) == ref.shape
    for i in range(2):
        assert _rel(got[i], ref[i]) < 5e-6
    X = (rng.standard_normal((2, n // 2 + 1)) + 1j * rng.standard_normal((2, n // 2 + 1)))
    X = X.astype(np.complex64)
    back = bfft.irfft(X, n=n)
    ref_back = np.fft.irfft(X.astype(np.complex128), n=n, axis=-1)
    for i in range(2):
        assert _rel(back[i], ref_back[i]) < 5e-6
    assert bfft.device_status() == 0


@pytest.mark.parametrize("n,nbins", [(3 << 13, 1000), (3 << 13, (3 << 12) + 1),
                                     (5 << 13, (5 << 12) + 700), (15 << 13, 7)])
def test_irfft_odd_factor_truncation_and_padding(rng, n, nbins):
    """numpy irfft semantics on the mixed path: fewer bins than n/2+1 are zero-padded, more are
    cut; the imaginary parts of DC and Nyquist are ignored."""
    X = (rng.standard_normal(nbins) + 1j * rng.standard_normal(nbins)).astype(np.complex64)
    assert _rel(bfft.irfft(X, n=n), np.fft.irfft(X.astype(np.complex128), n=n)) < 5e-6


def test_odd_factor_structured_and_roundtrip(rng):
    """A tone on a non-bin frequency and an impulse (exercise every residue class of the
    combine), the largest packed size class here, and the irfft(rfft(x)) round trip."""
    n = 3 << 20
    t = np.arange(n)
    tone = np.cos(2 * np.pi * (123456.25 / n) * t).astype(np.float32)
    imp = np.zeros(n, np.float32)
    imp[98765] = 1.0
    for x in (tone, imp):
        assert _rel(bfft.rfft(x), np.fft.rfft(x.astype(np.float64))) < 5e-6
    x = rng.standard_normal((3, 7 << 13)).astype(np.float32)
    assert _rel(bfft.irfft(bfft.rfft(x), n=7 << 13), x) < 5e-6
    xt = np.ascontiguousarray(x.T)
    assert _rel(bfft.rfft(xt, axis=0), np.fft.rfft(xt.astype(np.float64), axis=0)) < 5e-6


def test_odd_factor_default_routing(monkeypatch):
    """With the public threshold (2^22 complex points) an odd-factor irfft runs the kernels once
    n/2 reaches 2^22, the forward stays on cuFFT; odd factors above 15 or packed lengths outside
    [2^12, 2^26] never run them."""
    monkeypatch.setattr(bfft, "KERNEL_MIN_LOG2", 22)
    monkeypatch.setattr(bfft, "ODD_FORWARD", False)
    assert bfft._real_in_range(3 << 22, inverse=True) and not bfft._real_in_range(3 << 22)
    assert not bfft._real_in_range(3 << 20, inverse=True)
    assert bfft._real_split(17 << 14) is None and bfft._real_split(3 << 12) is None
    x = np.random.default_rng(3).standard_normal(3 << 22).astype(np.float32)
    X = bfft.rfft(x)  # cuFFT
    assert _rel(bfft.irfft(X, n=3 << 22), x) < 5e-6  # kernels


def test_long_transforms_capture_in_a_cuda_graph(rng):
    """The public long transforms can be captured and replayed (the watchdog stands aside while
    the stream captures): rfft of a power-of-two and of an odd-factor length, and irfft."""
    from mlx_signal_b200 import graphs

    for n in (1 << 14, 3 << 13):
        x0 = torch.from_numpy(rng.standard_normal((2, n)).astype(np.float32)).cuda()
        call = graphs.GraphedCall(lambda t: bfft.irfft(bfft.rfft(t) * 2.0, n=n), x0)
        for _ in range(2):
            x = rng.standard_normal((2, n)).astype(np.float32)
            got = call(torch.from_numpy(x).cuda())
            torch.cuda.synchronize()
            assert _rel(got, 2.0 * x.astype(np.float64)) < 5e-6
        del call
    assert bfft.device_status() == 0


@pytest.mark.parametrize("e", [22, 23])
def test_rfft_batched_rows(rng, e):
    """A batch of 2^22- and 2^23-sample rows through the packed three-pass transform against
    float64 numpy, and the inverse."""
    n = 1 << e
    x = rng.standard_normal((3, n)).astype(np.float32)
    ref = np.fft.rfft(x.astype(np.float64), axis=-1)
    got = bfft.rfft(x)
    for i in range(3):
        assert _rel(got[i], ref[i]) < 5e-6
    assert _rel(bfft.irfft(got, n=n), x) < 5e-6
    assert bfft.device_status() == 0
