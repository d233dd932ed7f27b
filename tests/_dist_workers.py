"""Rank bodies for the gloo multi-process tests (importable by spawned children)."""

import os

import numpy as np
import torch
import torch.distributed as dist


def _init(rank, world, port):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)


def _oracle_welch(x, **kw):
    from oracle import cpu_reference

    f, p = cpu_reference.welch(np.asarray(x, dtype=np.float64), **kw)
    return torch.from_numpy(f), torch.from_numpy(p)


def welch_long_rank(rank, world, port, n, kw, seed, out_dir):
    from mlx_signal_b200 import sharding

    _init(rank, world, port)
    try:
        x = np.random.default_rng(seed).standard_normal(n)
        N = kw["nperseg"]
        hop = N - kw.get("noverlap", N // 2)
        nseg = (n - N) // hop + 1
        s0, s1 = sharding.segment_range(nseg, world, rank)
        a, b = sharding.segment_slice(n, N, hop, s0, s1)
        f, p = sharding.welch_long(x[a:b], nseg, s0, s1, psd_mean=_oracle_welch, **kw)
        np.save(os.path.join(out_dir, f"p{rank}.npy"), p.numpy())
        np.save(os.path.join(out_dir, f"f{rank}.npy"), f.numpy())
    finally:
        dist.destroy_process_group()


def rows_rank(rank, world, port, rows, n, seed, out_dir):
    from mlx_signal_b200 import sharding

    _init(rank, world, port)
    try:
        x = np.random.default_rng(seed).standard_normal((rows, n))
        r0, r1 = sharding.row_range(rows, world, rank)
        _, p = _oracle_welch(x[r0:r1], nperseg=128)
        parts = [None] * world
        dist.all_gather_object(parts, (r0, r1, p.numpy()))
        full = np.concatenate([q for _, _, q in sorted(parts, key=lambda t: t[0])], axis=0)
        np.save(os.path.join(out_dir, f"rows{rank}.npy"), full)
    finally:
        dist.destroy_process_group()
