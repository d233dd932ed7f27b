"""CPU: host-side argument logic that runs before any device call (no GPU needed)."""

import numpy as np
import pytest

import mlx_signal_b200 as msig
from mlx_signal_b200 import _kernels, spectral
from mlx_signal_b200.windows import ByteBudgetCache, _window_np


def test_triage_string_window_and_short_signal_warning():
    with pytest.warns(UserWarning, match="nperseg"):
        w, n = spectral._triage_segments("hann", 512, input_length=100)
    assert n == 100 and w.shape == (100,)
    w, n = spectral._triage_segments(("tukey", 0.25), None, input_length=1000)
    assert n == 256


def test_triage_array_window_errors():
    with pytest.raises(ValueError, match="1-D"):
        spectral._triage_segments(np.ones((2, 2)), None, 100)
    with pytest.raises(ValueError, match="longer than input"):
        spectral._triage_segments(np.ones(200), None, 100)
    with pytest.raises(ValueError, match="different from length of window"):
        spectral._triage_segments(np.ones(64), 32, 100)


def test_detrend_codes():
    assert spectral._detrend_code(False) == 0
    assert spectral._detrend_code("constant") == 1
    assert spectral._detrend_code("l") == 2
    with pytest.raises(ValueError, match="Trend type"):
        spectral._detrend_code("quadratic")
    with pytest.raises(NotImplementedError):
        spectral._detrend_code(lambda d: d)


def test_istft_axes_validation():
    assert spectral._istft_axes((2, 3, 129, 40), -2, -1) == (2, 3, [0, 1, 3, 2])
    with pytest.raises(ValueError, match="at least 2d"):
        spectral._istft_axes((16,), -2, -1)
    with pytest.raises(ValueError, match="differing"):
        spectral._istft_axes((4, 5), 1, -1)
    with pytest.raises(IndexError):
        spectral._istft_axes((4, 5), 5, -1)


def test_onesided_factor_and_median_bias():
    f = spectral._onesided_factor_np(8)
    assert f.tolist() == [1, 2, 2, 2, 1]
    assert spectral._onesided_factor_np(7).tolist() == [1, 2, 2, 2]
    assert spectral._median_bias(1) == 1.0
    assert abs(spectral._median_bias(5) - (1 + 1 / 3 - 1 / 2 + 1 / 5 - 1 / 4)) < 1e-15


def test_fused_routing_rule():
    assert _kernels.fused_mean_ok(1024) and _kernels.fused_mean_ok(1)
    assert _kernels.fused_mean_ok(8192) and not _kernels.fused_mean_ok(16384)
    assert not _kernels.fused_mean_ok(100) and not _kernels.fused_complex_ok(8192)
    assert _kernels.blue_ok(1000) and _kernels.blue_ok(3) and _kernels.blue_ok(2047)
    assert _kernels.blue_ok(2049) and _kernels.blue_ok(4095)
    assert not _kernels.blue_ok(1024) and not _kernels.blue_ok(4097)


def test_config_validation_and_context():
    with pytest.raises(ValueError, match="no CPU"):
        msig.set_config(dispatch="scipy")
    with pytest.raises(TypeError):
        msig.set_config(nonsense=1)
    base = msig.get_config().float64
    with msig.config_context(float64="strict"):
        assert msig.get_config().float64 == "strict"
    assert msig.get_config().float64 == base


def test_dtype_policy_without_device():
    from mlx_signal_b200 import _array

    with msig.config_context(float64="strict"):
        with pytest.raises(TypeError, match="strict"):
            _array.check_dtype_policy(np.zeros(4))
    with msig.config_context(float64="downcast", warn_on_downcast=True):
        with pytest.warns(msig.DowncastWarning):
            _array.check_dtype_policy(np.zeros(4, dtype=np.complex128))


def test_window_cache_and_byte_budget():
    w = _window_np("hann", 64)
    assert w.dtype == np.float64 and not w.flags.writeable
    c = ByteBudgetCache(100)
    c.put(("a",), 1, 60)
    c.put(("b",), 2, 60)
    assert c.get(("a",)) is None and c.get(("b",)) == 2
    c.put(("huge",), 3, 1000)
    assert c.get(("huge",)) is None


def test_conv_ols_block_choice_and_argument_errors():
    """Host side of the fused convolution entry point: block length per filter length (fewest FFT
    operations per output with a step of at least half a block) and argument checks, which run
    before any device work."""
    from mlx_signal_b200 import _lib

    lib = _lib.load()
    assert lib.sp_conv_block_len(1) == 256
    assert lib.sp_conv_block_len(129) == 1024  # 10*1024/896 < 9*512/384 < 8*256/128
    assert lib.sp_conv_block_len(1025) == 4096
    assert lib.sp_conv_block_len(2049) == 4096
    assert lib.sp_conv_block_len(2050) == _lib.SP_ERR_UNSUPPORTED
    assert lib.sp_conv_block_len(0) == _lib.SP_ERR_UNSUPPORTED
    dummy = 16  # never dereferenced: the checks below fail before any launch
    assert lib.sp_conv_ols_f32(dummy, 1, 100, 100, dummy, 10, 0, 110, dummy, 110, None) == \
        _lib.SP_ERR_ARG  # window past the full length 109
    assert lib.sp_conv_ols_f32(dummy, 1, 100, 99, dummy, 10, 0, 10, dummy, 10, None) == \
        _lib.SP_ERR_ARG  # row stride below n1
    assert lib.sp_conv_ols_f32(dummy, 1, 4000, 4000, dummy, 2050, 0, 10, dummy, 10, None) == \
        _lib.SP_ERR_UNSUPPORTED
    assert lib.sp_conv_ols_f32(dummy, 0, 100, 100, dummy, 10, 0, 109, dummy, 109, None) == _lib.SP_OK


def test_convolve_axes_validation():
    """scipy's axis rules for fftconvolve / oaconvolve (the reference's
    tests/test_edge_cases.py:246-256): integer axes only, in range, unique; singleton axes
    dropped. Shapes only, so CPU tensors stand in for the device inputs."""
    import torch

    from mlx_signal_b200.convolution import _init_axes

    a = torch.zeros((4, 5))
    for bad, msg in ((2, "exceeds dimensionality"), ([-3], "exceeds dimensionality"),
                     (1.5, "integers"), ([0.5, 1], "integers"), ([1, -1], "unique")):
        with pytest.raises(ValueError, match=msg):
            _init_axes(a, a, "full", bad)
    assert _init_axes(a, a, "full", np.int64(1))[2] == [1]
    assert _init_axes(a, a, "full", [np.int32(0), -1])[2] == [0, 1]
    one = torch.zeros((1, 3))
    assert _init_axes(one, one, "full", [0])[2] == []  # every conv axis is length 1: a product
    with pytest.raises(ValueError, match="mode flags"):
        _init_axes(a, a, "circular", None)


def test_profiling_workloads_listed():
    import workloads  # the top-level profiling entry the ncu summaries name

    assert workloads.main(["--list"]) == 0
    assert {"welch_64x2p20_n1024", "conv_8x2p22_t1025", "rfft_2p23"} <= set(workloads.WORKLOADS)


def test_real_length_split_and_routing(monkeypatch):
    """Real transform lengths n = 2 C 2^e (C odd <= 15, e in [12, 26]) and their routing
    threshold; everything else goes to the composed path."""
    from mlx_signal_b200 import fft as bfft

    assert bfft._real_split(1 << 23) == (1, 22)
    assert bfft._real_split(3 << 20) == (3, 19)
    assert bfft._real_split(15 << 13) == (15, 12)
    for n in (0, 1, 3 << 11, 17 << 14, 600_000, (1 << 27) + 2, 1 << 28, 9999):
        assert bfft._real_split(n) is None
    assert bfft.KERNEL_MIN_LOG2 == 22 and not bfft.ODD_FORWARD
    assert bfft._real_in_range(1 << 23) and not bfft._real_in_range(1 << 22)
    assert bfft._real_in_range(3 << 22, inverse=True) and not bfft._real_in_range(3 << 22)
    assert not bfft._real_in_range(3 << 21, inverse=True)
    assert bfft._resample_in_range(1 << 22, 3 << 20) and bfft._resample_in_range(1 << 21, 3 << 19)
    assert not bfft._resample_in_range(1 << 20, 3 << 18)
    assert not bfft._resample_in_range(1 << 22, 1001)
    monkeypatch.setattr(bfft, "KERNEL_MIN_LOG2", 12)
    monkeypatch.setattr(bfft, "ODD_FORWARD", True)
    assert bfft._real_in_range(3 << 13) and bfft._real_in_range(1 << 13)
