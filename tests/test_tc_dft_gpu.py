"""GPU: batched 32-point complex DFTs on the tensor cores (sp_dft32_tc_c64) against float64
numpy. The stage uses FP16 head/tail operand splits with three products and FP32 accumulation;
the bar is an FP32-FFT-class error: max |error| <= 2e-6 of each vector's peak."""

import numpy as np
import pytest
import torch

from mlx_signal_b200 import _kernels

pytestmark = pytest.mark.gpu


def _rel_rows(got, ref):
    got = got.cpu().numpy().astype(np.complex128)
    peak = np.abs(ref).max(axis=-1)
    keep = peak > 0
    return float(np.max(np.abs(got - ref).max(axis=-1)[keep] / peak[keep]))


@pytest.mark.parametrize("scale", [1.0, 1e-6, 3e5])
def test_dft32_tc_matches_numpy(rng, scale):
    nvec = 1000  # not a multiple of the 128-vector tile
    z = (rng.standard_normal((nvec, 32)) + 1j * rng.standard_normal((nvec, 32))) * scale
    z = z.astype(np.complex64)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    y = _kernels.dft32_tc(torch.from_numpy(z).cuda(), err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = np.fft.fft(z.astype(np.complex128), axis=-1)
    assert _rel_rows(y, ref) <= 2e-6


def test_dft32_tc_structured_and_repeats(rng):
    # tones, impulses, a constant and an all-zero vector in one batch; repeating the MMA chain
    # gives the same bits
    n = np.arange(32)
    rows = [np.exp(2j * np.pi * k * n / 32) for k in (0, 1, 5, 16, 31)]
    rows += [np.eye(32)[i] for i in (0, 7)]
    rows += [np.full(32, 2.5 - 1j), np.zeros(32)]
    rows += list(rng.standard_normal((300, 32)) + 1j * rng.standard_normal((300, 32)))
    z = np.asarray(rows).astype(np.complex64)
    zt = torch.from_numpy(z).cuda()
    y1 = _kernels.dft32_tc(zt)
    y4 = _kernels.dft32_tc(zt, reps=4)
    assert torch.equal(y1, y4)
    ref = np.fft.fft(z.astype(np.complex128), axis=-1)
    assert _rel_rows(y1, ref) <= 2e-6
    assert float(y1[8].abs().max()) == 0.0
