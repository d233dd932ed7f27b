"""CPU: host logic of the batched persistent launch -- validation, the descriptor table the
encoder writes, the work decomposition the kernel walks (every segment / frame exactly once,
disjoint partial slots), the stream tail arithmetic against scipy, and the schedule cache.
No device calls: sp_batch_plan / sp_batch_encode only write host memory, and device pointers
here are placeholders that are never dereferenced."""

import ctypes

import numpy as np
import pytest
import scipy.signal as sps

from mlx_signal_b200 import _lib
from mlx_signal_b200.autotune import ScheduleCache, channels_bucket
from mlx_signal_b200.batch import BatchRequest, _desc_bytes

FAKE = 1 << 40  # placeholder device addresses

REQ_DT = np.dtype([
    ("x", "<u8"), ("win", "<u8"), ("wdft", "<u8"), ("out", "<u8"), ("part", "<u8"),
    ("cnt", "<u8"), ("tail_in", "<u8"), ("tail_out", "<u8"), ("ld", "<i8"), ("tail_ld", "<i8"),
    ("kind", "<i4"), ("log_l", "<i4"), ("rows", "<i4"), ("nseg", "<i4"), ("G", "<i4"),
    ("chunks", "<i4"), ("tasks", "<i4"), ("nbins", "<i4"), ("n_low", "<i4"),
    ("onesided", "<i4"), ("tail_len", "<i4"), ("new_tail_len", "<i4"), ("hop", "<i4"),
    ("pad0", "<i4"), ("scale", "<f4"), ("pad1", "<f4"),
])
assert REQ_DT.itemsize == 144
TEAMS = {8: 8, 9: 4, 10: 4, 11: 1, 12: 1}


def welch_req(nperseg, rows, n, detrend=1, G=0, onesided=1, k=0):
    r = BatchRequest()
    r.kind = 0
    r.nperseg = nperseg
    r.hop = nperseg // 2
    r.detrend = detrend
    r.onesided = onesided
    r.n_low = 2 if detrend == 1 else 0
    r.seg_per_task = G
    r.rows = rows
    r.n = n
    r.ld = n
    r.x = FAKE + 0x1000000 * k
    r.win = FAKE + 0x10
    r.win_dft_low = FAKE + 0x20 if detrend == 1 else None
    r.out = FAKE + 0x100000 * k + 0x40
    r.scale = 0.5
    return r


def stream_req(nperseg, hop, rows, n, tail_len, G=0, k=0):
    r = BatchRequest()
    r.kind = 1
    r.nperseg = nperseg
    r.hop = hop
    r.onesided = 1
    r.seg_per_task = G
    r.tail_len = tail_len
    r.rows = rows
    r.n = n
    r.ld = n
    r.tail_ld = nperseg
    r.x = FAKE + 0x2000000 * k
    r.win = FAKE + 0x30
    r.tail_in = FAKE + 0x4000000 + 0x10000 * k
    r.tail_out = FAKE + 0x5000000 + 0x10000 * k
    r.out = FAKE + 0x6000000 + 0x100000 * k
    r.scale = 1.0
    return r


def arr(reqs):
    a = (BatchRequest * max(1, len(reqs)))()
    for i, r in enumerate(reqs):
        a[i] = r
    return a


def plan(reqs):
    d, w = ctypes.c_int64(0), ctypes.c_int64(0)
    a = arr(reqs)
    st = _lib.load().sp_batch_plan(ctypes.addressof(a), len(reqs), ctypes.byref(d),
                                   ctypes.byref(w))
    return st, d.value, w.value


def encode(reqs, ws_base=FAKE + (1 << 36)):
    st, d, w = plan(reqs)
    assert st == 0, _lib.last_error()
    assert d == _desc_bytes(len(reqs))
    blob = np.zeros(d, np.uint8)
    a = arr(reqs)
    st = _lib.load().sp_batch_encode(ctypes.addressof(a), len(reqs), ws_base, w,
                                     blob.ctypes.data, d)
    assert st == 0, _lib.last_error()
    hdr = blob[:16].view("<i4")
    nreq = int(hdr[1])
    ib = blob[16 : 16 + 4 * (nreq + 1)].view("<i4")
    off = 16 + ((4 * (nreq + 1) + 15) & ~15)
    recs = blob[off : off + 144 * nreq].view(REQ_DT)
    return hdr, ib, recs, w, ws_base


def test_stream_frames_formula():
    lib = _lib.load()
    nt = ctypes.c_int64(0)
    for tail, n, N, hop in [(0, 4096, 1024, 256), (768, 5000, 1024, 256), (0, 100, 256, 128),
                            (255, 1, 256, 128), (1000, 0, 1024, 1024)]:
        f = lib.sp_batch_stream_frames(tail, n, N, hop, ctypes.byref(nt))
        m = tail + n
        ef = (m - N) // hop + 1 if m >= N else 0
        assert f == ef and nt.value == m - ef * hop
        assert 0 <= nt.value < N or ef == 0
    assert lib.sp_batch_stream_frames(0, 10, 256, 0, ctypes.byref(nt)) == _lib.SP_ERR_ARG


@pytest.mark.parametrize("bad,code", [
    (lambda: welch_req(128, 1, 10000), _lib.SP_ERR_UNSUPPORTED),
    (lambda: welch_req(300, 1, 10000), _lib.SP_ERR_UNSUPPORTED),
    (lambda: welch_req(1024, 1, 1000), _lib.SP_ERR_ARG),           # n < nperseg
    (lambda: welch_req(1024, 1, 10000, detrend=2), _lib.SP_ERR_ARG),  # linear not batched
    (lambda: (lambda r: (setattr(r, "hop", 256), r)[1])(welch_req(1024, 1, 10000)),
     _lib.SP_ERR_ARG),
    (lambda: (lambda r: (setattr(r, "n_low", 0), r)[1])(welch_req(1024, 1, 10000)),
     _lib.SP_ERR_ARG),
    (lambda: (lambda r: (setattr(r, "n_low", 33), r)[1])(welch_req(1024, 1, 10000)),
     _lib.SP_ERR_ARG),
    (lambda: stream_req(1024, 256, 1, 5000, 1024), _lib.SP_ERR_ARG),  # tail_len >= nperseg
    (lambda: (lambda r: (setattr(r, "tail_out", r.tail_in), r)[1])(
        stream_req(1024, 256, 1, 5000, 0)), _lib.SP_ERR_ARG),
    (lambda: (lambda r: (setattr(r, "kind", 7), r)[1])(welch_req(1024, 1, 10000)),
     _lib.SP_ERR_ARG),
])
def test_plan_rejects(bad, code):
    st, _, _ = plan([welch_req(256, 1, 4096), bad()])
    assert st == code
    assert "request 1" in _lib.last_error()


def test_encode_rejects_small_buffers():
    reqs = [welch_req(1024, 4, 1 << 16)]
    st, d, w = plan(reqs)
    assert st == 0
    blob = np.zeros(d, np.uint8)
    a = arr(reqs)
    lib = _lib.load()
    assert lib.sp_batch_encode(ctypes.addressof(a), 1, FAKE, w - 1, blob.ctypes.data,
                               d) == _lib.SP_ERR_WORKSPACE
    assert lib.sp_batch_encode(ctypes.addressof(a), 1, FAKE, w, blob.ctypes.data,
                               d - 1) == _lib.SP_ERR_WORKSPACE


def _mixed(rng, k=40):
    reqs = []
    for i in range(k):
        if rng.random() < 0.3:
            N = int(rng.choice([256, 512, 1024, 4096]))
            hop = int(rng.choice([N // 4, N // 2, N]))
            reqs.append(stream_req(N, hop, int(rng.integers(1, 4)), int(rng.integers(0, 20000)),
                                   int(rng.integers(0, N)), G=int(rng.choice([0, 2, 6])), k=i))
        else:
            N = int(rng.choice([256, 512, 1024, 4096]))
            n = int(2 ** rng.uniform(np.log2(N), 17))
            reqs.append(welch_req(N, int(rng.integers(1, 9)), n, detrend=int(rng.integers(0, 2)),
                                  G=int(rng.choice([0, 3, 8, 64])),
                                  onesided=int(rng.integers(0, 2)), k=i))
    return reqs


def test_descriptor_layout_and_order(rng):
    reqs = _mixed(rng)
    hdr, ib, recs, w, ws = encode(reqs)
    assert hdr[0] == 0x42415443 and hdr[1] == len(reqs)
    # larger classes first, stable within a class
    assert np.all(np.diff(recs["log_l"]) <= 0)
    items = np.diff(ib)
    assert ib[0] == 0 and hdr[2] == ib[-1]
    # the 4096 class (the 256-thread kernel's work) holds items [0, first_small)
    assert hdr[3] == ib[int(np.sum(recs["log_l"] == 12))]
    for rec, it in zip(recs, items):
        assert it == -(-int(rec["tasks"]) // TEAMS[int(rec["log_l"])])
        assert rec["tasks"] == rec["rows"] * rec["chunks"]
        assert rec["G"] % 2 == 0 and rec["G"] >= 2
    # every input request appears exactly once (matched by its x pointer)
    assert sorted(recs["x"].tolist()) == sorted(r.x for r in reqs)


def test_work_decomposition_covers_every_segment_once(rng):
    """Walk items -> tasks -> segment ranges as the kernel does; each (request, row, segment)
    is produced by exactly one task and welch partial slots are disjoint and inside ws."""
    reqs = _mixed(rng, 60)
    hdr, ib, recs, w, ws = encode(reqs)
    slots = []
    counters = set()
    for rec, i0, i1 in zip(recs, ib[:-1], ib[1:]):
        L = 1 << int(rec["log_l"])
        T = TEAMS[int(rec["log_l"])]
        seen = np.zeros((int(rec["rows"]), max(int(rec["nseg"]), 1)), np.int32)
        tail_writes = 0
        for local in range(i1 - i0):
            for team in range(T):
                task = local * T + team
                if task >= rec["tasks"]:
                    continue
                row, ch = divmod(task, int(rec["chunks"]))
                s0 = ch * int(rec["G"])
                s1 = min(s0 + int(rec["G"]), int(rec["nseg"]))
                seen[row, s0:s1] += 1
                if rec["kind"] == 0:
                    slots.append((int(rec["part"]) + 4 * task * (L // 2 + 1), 4 * (L // 2 + 1)))
                elif ch == rec["chunks"] - 1:
                    tail_writes += 1
        if rec["nseg"] > 0:
            assert np.all(seen[:, : int(rec["nseg"])] == 1)
        if rec["kind"] == 0:
            for r in range(int(rec["rows"])):
                c = int(rec["cnt"]) + 4 * r
                assert c not in counters
                counters.add(c)
        else:
            assert tail_writes == rec["rows"]
    slots.sort()
    for (a, n), (b, _) in zip(slots, slots[1:]):
        assert a + n <= b
    assert all(ws + 256 <= a and a + n <= ws + w for a, n in slots)
    assert all(ws + 256 <= c < slots[0][0] for c in counters)


def test_stream_tail_arithmetic_matches_scipy(rng):
    """The chunk/tail state machine (frames per chunk, new tail length, frame offsets) emulated
    on the host reproduces scipy.signal.stft of the concatenated stream frame by frame."""
    lib = _lib.load()
    N, hop = 256, 64
    x = rng.standard_normal(20000)
    chunks = np.split(x, np.sort(rng.choice(np.arange(1, 20000), 9, replace=False)))
    tail = np.zeros(0)
    frames = []
    nt = ctypes.c_int64(0)
    win = sps.get_window("hann", N)
    for c in chunks:
        f = lib.sp_batch_stream_frames(len(tail), len(c), N, hop, ctypes.byref(nt))
        u = np.concatenate([tail, c])
        for j in range(f):
            frames.append(np.fft.rfft(u[j * hop : j * hop + N] * win) / win.sum())
        tail = u[f * hop :]
        assert len(tail) == nt.value
    _, _, Z = sps.stft(x, nperseg=N, noverlap=N - hop, boundary=None, padded=False)
    got = np.stack(frames, axis=-1)
    assert got.shape == Z.shape
    np.testing.assert_allclose(got, Z, rtol=1e-10, atol=1e-12)


def test_empty_batch_encodes():
    hdr, ib, recs, w, ws = encode([])
    assert hdr[1] == 0 and hdr[2] == 0 and len(recs) == 0 and w == 256


def test_schedule_cache_roundtrip(tmp_path):
    p = tmp_path / "sched.json"
    c = ScheduleCache(p)
    assert c.get("welch", 1024, 7) == 64  # default
    c.put("welch", 1024, 7, 64, timings_us={32: 10.0, 64: 9.0})
    assert c.get("welch", 1024, 5) == 64  # same channels bucket (8)
    assert c.get("welch", 1024, 9) == 64  # next bucket (default)
    c2 = ScheduleCache(p)
    assert c2.get("welch", 1024, 8) == 64
    assert "welch/1024/float32/c8" in c2.entries()
    assert [channels_bucket(v) for v in (1, 2, 3, 5, 17, 64, 500)] == [1, 2, 4, 8, 32, 64, 64]


def test_two_chunks_of_one_stream_are_rejected():
    a = stream_req(1024, 256, 1, 5000, 0, k=1)
    b = stream_req(1024, 256, 1, 5000, 0, k=2)
    b.tail_in = a.tail_out  # b continues a's stream inside the same batch
    st, _, _ = plan([a, b])
    assert st == _lib.SP_ERR_ARG
    assert "share a stream tail buffer" in _lib.last_error()
