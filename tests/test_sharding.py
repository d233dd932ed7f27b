"""CPU: multi-rank partitioning of the spectral path (world size 2 over gloo, spawned ranks).
Rows / requests / streams shard with no collective; one long channel split by segment ranges
combines its partial sums with one all-reduce and equals the single-device result. The oracle
(scipy, float64) stands in for the per-rank kernel here."""

import socket

import numpy as np
import pytest
import scipy.signal as sps
import torch.multiprocessing as mp

import _dist_workers as W
from mlx_signal_b200 import sharding


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_row_range_partitions_every_row_once():
    for rows in (0, 1, 5, 64, 1001):
        for world in (1, 2, 3, 8):
            got = [sharding.row_range(rows, world, r) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == rows
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            sizes = [b - a for a, b in got]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        sharding.row_range(4, 2, 2)


def test_assign_requests_is_deterministic_and_balanced(rng):
    costs = rng.integers(1, 1000, 300).tolist()
    a = sharding.assign_requests(costs, 4)
    assert a == sharding.assign_requests(costs, 4)
    loads = np.zeros(4)
    for c, r in zip(costs, a):
        loads[r] += c
    assert loads.max() - loads.min() <= max(costs)
    assert sharding.assign_requests([5.0], 3) == [0]


@pytest.mark.parametrize("n,N,hop", [(10000, 256, 128), (4096, 1024, 256), (1024, 1024, 512),
                                     (77777, 512, 100)])
def test_segment_slices_cover_every_segment(n, N, hop):
    nseg = (n - N) // hop + 1
    for world in (1, 2, 3, 7):
        seen = np.zeros(nseg, int)
        for r in range(world):
            s0, s1 = sharding.segment_range(nseg, world, r)
            a, b = sharding.segment_slice(n, N, hop, s0, s1)
            assert 0 <= a <= b <= n
            for s in range(s0, s1):
                assert a <= s * hop and s * hop + N <= b
                seen[s] += 1
        assert np.all(seen == 1)


@pytest.mark.parametrize("n,kw", [
    (50000, {"nperseg": 256}),
    (40000, {"nperseg": 512, "noverlap": 384, "detrend": "linear", "scaling": "spectrum"}),
    (1500, {"nperseg": 1024}),  # one segment: rank 1 has none and contributes zeros
])
def test_welch_long_channel_over_two_ranks(tmp_path, n, kw):
    mp.spawn(W.welch_long_rank, args=(2, _port(), n, kw, 9, str(tmp_path)), nprocs=2)
    x = np.random.default_rng(9).standard_normal(n)
    f_ref, p_ref = sps.welch(x, **kw)
    for r in range(2):
        p = np.load(tmp_path / f"p{r}.npy")
        f = np.load(tmp_path / f"f{r}.npy")
        np.testing.assert_allclose(p, p_ref, rtol=1e-6, atol=0)
        np.testing.assert_allclose(f, f_ref, rtol=1e-6)


def test_rows_shard_without_collective_on_the_data_path(tmp_path):
    mp.spawn(W.rows_rank, args=(2, _port(), 5, 4096, 4, str(tmp_path)), nprocs=2)
    x = np.random.default_rng(4).standard_normal((5, 4096))
    _, p_ref = sps.welch(x, nperseg=128)
    for r in range(2):
        np.testing.assert_allclose(np.load(tmp_path / f"rows{r}.npy"), p_ref, rtol=1e-12)
