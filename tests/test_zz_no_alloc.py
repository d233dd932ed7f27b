"""GPU: the no-allocation welch entry point (sp_welch_f32_noalloc) against sp_welch_f32.

sp_welch_f32_noalloc serves callers that cannot allocate device memory (plugin hosts that only
receive input/output pointers, loops that must not call cudaMalloc after start-up): its scratch
is a fixed static device array. This file is collected last so that a run stopping at the
first failure has already run every other test; it also passes alone in a fresh process.
"""

import numpy as np
import pytest
import torch

from _utils import assert_close

pytestmark = pytest.mark.gpu


def _window(nperseg, fs):
    import scipy.signal as sps

    w = sps.get_window("hann", nperseg)
    scale = 1.0 / (fs * float((w * w).sum()))
    return torch.from_numpy((w * np.sqrt(scale)).astype(np.float32)).cuda()


def _noalloc(lib, x, win, nperseg, hop, detrend, onesided):
    rows, n = x.shape
    nout = nperseg // 2 + 1 if onesided else nperseg
    out = torch.empty((rows, nout), dtype=torch.float32, device=x.device)
    st = lib.sp_welch_f32_noalloc(x.data_ptr(), rows, n, x.stride(0), win.data_ptr(), nperseg,
                                  nperseg, hop, detrend, int(onesided), out.data_ptr(),
                                  torch.cuda.current_stream().cuda_stream)
    return st, out


def test_noalloc_matches_workspace_entry_point_on_two_calls():
    from mlx_signal_b200 import _kernels, _lib

    lib = _lib.load()
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    fs = 48000.0
    cases = [
        (torch.randn((8, 1 << 17), generator=g, device="cuda"), 1024, 512, 1, True),
        (torch.randn((3, 50_000), generator=g, device="cuda"), 256, 100, 2, False),
    ]
    for x, nperseg, hop, detrend, onesided in cases:  # two calls in a row, different shapes
        win = _window(nperseg, fs)
        ref = _kernels.welch_mean(x, win, nperseg, nperseg, hop, detrend, onesided)
        st, out = _noalloc(lib, x, win, nperseg, hop, detrend, onesided)
        assert st == 0, _lib.last_error()
        torch.cuda.synchronize()
        assert_close(out, ref.cpu().numpy(), rtol=1e-4, atol_frac=1e-5)
    # and the first shape again after the second one overwrote the shared scratch
    x, nperseg, hop, detrend, onesided = cases[0]
    win = _window(nperseg, fs)
    ref = _kernels.welch_mean(x, win, nperseg, nperseg, hop, detrend, onesided)
    st, out = _noalloc(lib, x, win, nperseg, hop, detrend, onesided)
    assert st == 0, _lib.last_error()
    torch.cuda.synchronize()
    assert_close(out, ref.cpu().numpy(), rtol=1e-4, atol_frac=1e-5)
    # and directly against float64 scipy on two rows: max relative error <= 1e-5 on bins above
    # 1e-6 of the row peak (2^17 samples at nperseg 1024: 255 segments per row)
    import scipy.signal as sps

    _, pref = sps.welch(x[:2].double().cpu().numpy(), fs=fs, nperseg=nperseg,
                        noverlap=nperseg - hop, detrend="constant")
    got = out[:2].double().cpu().numpy()
    keep = pref > 1e-6 * pref.max(axis=-1, keepdims=True)
    assert np.max(np.abs(got - pref)[keep] / pref[keep]) <= 1e-5


def test_noalloc_rejects_shapes_beyond_the_fixed_scratch():
    from mlx_signal_b200 import _lib

    lib = _lib.load()
    rows, n, nperseg = 4096, 1 << 16, 1024
    need = lib.sp_mean_workspace_size(0, rows, n, nperseg, nperseg, nperseg // 2, 1)
    assert need > (16 << 20)
    # the size check runs on the plan before any pointer is used: a small placeholder buffer
    # stands in for the (rows, n) input, which is never read
    x = torch.empty(16, dtype=torch.float32, device="cuda")
    win = _window(nperseg, 1.0)
    out = torch.empty(16, dtype=torch.float32, device="cuda")
    st = lib.sp_welch_f32_noalloc(x.data_ptr(), rows, n, n, win.data_ptr(), nperseg, nperseg,
                                  nperseg // 2, 1, 1, out.data_ptr(),
                                  torch.cuda.current_stream().cuda_stream)
    assert st == _lib.SP_ERR_WORKSPACE
    assert "built-in scratch" in _lib.last_error()
