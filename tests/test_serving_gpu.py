"""GPU: the continuous-batching server. Every result is the same alone and in the mix
(bit-identical: a request's schedule depends only on its own shape), welch results meet the
accuracy bar against float64 scipy, stream chunks reproduce scipy.signal.stft of the
concatenated stream, admission respects the HBM budget, and the open-loop Poisson driver and the
per-request baseline complete their schedules."""

import pytest
import scipy.signal as sps
import torch

from mlx_signal_b200 import serving as sv
from _utils import assert_close, rel_err_bins

pytestmark = pytest.mark.gpu


def _pool(n=1 << 24, seed=3):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return torch.randn(n, generator=g, device="cuda")


def _submit(server, sched):
    rids = []
    for _, kind, x, p in sched:
        if kind == sv.KIND_WELCH:
            rids.append(server.submit_welch(x, nperseg=p["nperseg"]))
        else:
            rids.append(server.submit_chunk(p["stream"], x))
    return rids


def _small_sched(pool, n=160, seed=1, streams=6):
    return sv.poisson_schedule(1e6, n / 1e6, pool, seed=seed, n_streams=streams,
                               chunk=(700, 9000), welch_rows=(1, 4), welch_log2n=(10, 15))


def test_results_alone_equal_results_in_mix():
    pool = _pool()
    sched = _small_sched(pool)
    assert len(sched) > 50
    mix = sv.SpectralServer(hbm_budget=256 << 20, max_batch=48, slots=3, keep_results=True,
                            max_streams=8)
    rids = _submit(mix, sched)
    mix.drain()
    assert mix.stats.completed == len(sched)
    assert mix.stats.batches > 1
    # welch requests: each alone in a fresh server
    for rid, (_, kind, x, p) in zip(rids, sched):
        if kind != sv.KIND_WELCH:
            continue
        alone = sv.SpectralServer(hbm_budget=64 << 20, max_batch=4, slots=1, keep_results=True)
        r1 = alone.submit_welch(x, nperseg=p["nperseg"])
        alone.drain()
        assert torch.equal(alone.result(r1), mix.result(rid))
    # stream chunks: each stream replayed alone, chunk by chunk
    by_stream = {}
    for rid, (_, kind, x, p) in zip(rids, sched):
        if kind == sv.KIND_STREAM:
            by_stream.setdefault(p["stream"], []).append((rid, x))
    for s, items in by_stream.items():
        alone = sv.SpectralServer(hbm_budget=64 << 20, max_batch=4, slots=2, keep_results=True,
                                  max_streams=8)
        for rid, x in items:
            r1 = alone.submit_chunk(s, x)
            alone.drain()
            f0a, za = alone.result(r1)
            f0m, zm = mix.result(rid)
            assert f0a == f0m
            assert torch.equal(za, zm)


def test_server_matches_scipy():
    pool = _pool(seed=4)
    sched = _small_sched(pool, n=120, seed=2)
    srv = sv.SpectralServer(hbm_budget=256 << 20, max_batch=32, slots=2, keep_results=True,
                            max_streams=6)
    rids = _submit(srv, sched)
    srv.drain()
    streams = {}
    for rid, (_, kind, x, p) in zip(rids, sched):
        if kind == sv.KIND_WELCH:
            N = p["nperseg"]
            _, pref = sps.welch(x.double().cpu().numpy(), nperseg=N)
            got = srv.result(rid)
            nseg = (x.shape[-1] - N) // (N // 2) + 1
            if nseg >= 8:
                assert rel_err_bins(got, pref) <= 1e-5
            else:
                assert_close(got, pref, rtol=1e-4, atol_frac=1e-5)
        else:
            streams.setdefault(p["stream"], []).append((rid, x))
    for s, items in streams.items():
        xs = torch.cat([x for _, x in items]).double().cpu().numpy()
        frames = [srv.result(rid)[1] for rid, _ in items]
        got = torch.cat(frames, dim=-1).cpu().numpy()
        _, _, zref = sps.stft(xs, nperseg=1024, noverlap=768, boundary=None, padded=False)
        assert got.shape == zref.shape
        assert_close(got, zref, rtol=1e-4, atol_frac=1e-5)


def test_admission_respects_budget():
    pool = _pool(seed=5)
    sched = _small_sched(pool, n=80, seed=3)
    budget = 8 << 20
    srv = sv.SpectralServer(hbm_budget=budget, max_batch=64, slots=3, max_streams=6)
    big = pool[: 5 << 20].view(1, -1)
    with pytest.raises(ValueError):
        srv.submit_welch(big, nperseg=1024)
    _submit(srv, sched)
    srv.drain()
    assert srv.stats.completed == len(sched)
    assert 0 < srv.stats.peak_bytes <= budget
    assert srv.used == 0


def test_open_loop_poisson_and_baseline():
    pool = _pool(seed=6)
    sched = sv.poisson_schedule(4000.0, 0.1, pool, seed=7, n_streams=32)
    srv = sv.SpectralServer(hbm_budget=1 << 30, max_batch=256, slots=3, max_streams=32)
    st = sv.run_schedule(srv, sched)
    s = st.summary()
    assert s["completed"] == len(sched) and s["p99_ms"] >= s["p50_ms"] > 0
    base = sv.run_per_request(sched[:60])
    assert base.summary()["completed"] == 60
