"""GPU: a long channel split by segment ranges (the multi-GPU layout) computed on one device --
each virtual rank's weighted partial from the CUDA welch kernels, summed, equals the one-shot
welch of the whole channel."""

import numpy as np
import pytest
import torch

import mlx_signal_b200 as msig
from mlx_signal_b200 import sharding
from _utils import rel_err_bins

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3, 8])
def test_segment_split_sums_to_full_welch(rng, world):
    n, N = 1 << 20, 1024
    x = torch.from_numpy(rng.standard_normal(n).astype(np.float32)).cuda()
    hop = N // 2
    nseg = (n - N) // hop + 1
    total = None
    for r in range(world):
        s0, s1 = sharding.segment_range(nseg, world, r)
        a, b = sharding.segment_slice(n, N, hop, s0, s1)
        _, p = sharding.welch_long(x[a:b], nseg, s0, s1, nperseg=N, fs=48000.0)
        total = p.double() if total is None else total + p.double()
    _, ref = msig.welch(x, nperseg=N, fs=48000.0)
    assert rel_err_bins(total.float(), ref.double().cpu().numpy()) <= 2e-6
