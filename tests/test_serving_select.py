"""Host logic of the serving loop's admission (no device needed): SpectralServer._select on a
stand-in server state."""

import collections
import types

import numpy as np

from mlx_signal_b200 import serving as sv


def _state(max_batch=4, budget=100, nstreams=4):
    return types.SimpleNamespace(pending=collections.deque(), held={}, busy=np.zeros(nstreams, bool),
                                 budget=budget, used=0, max_batch=max_batch)


def _chunk(rid, stream, nbytes=1):
    return sv._Pending(rid, sv.KIND_STREAM, None, float(rid), 1024, stream, 0, 1.0, 1, nbytes, 0)


def _welch(rid, nbytes=1):
    return sv._Pending(rid, sv.KIND_WELCH, None, float(rid), 256, -1, 1, 1.0, 1, nbytes, 0)


def _select(st):
    return [r.rid for r in sv.SpectralServer._select(st)]


def test_stream_chunks_keep_their_order_and_one_per_batch():
    st = _state(max_batch=8)
    st.pending.extend([_chunk(0, 0), _chunk(1, 0), _welch(2), _chunk(3, 1), _chunk(4, 0)])
    assert _select(st) == [0, 2, 3]            # one chunk of stream 0 per batch
    assert [r.rid for r in st.held[0]] == [1, 4] and not st.pending
    st.busy[0] = True                           # chunk 0 in flight
    st.pending.append(_chunk(5, 0))
    st.pending.append(_welch(6))
    assert _select(st) == [6]                   # stream 0 waits; 5 queues behind 1 and 4
    assert [r.rid for r in st.held[0]] == [1, 4, 5]
    st.busy[0] = False
    assert _select(st) == [1]                   # held chunks first, still one per batch
    assert _select(st) == [4] and _select(st) == [5] and 0 not in st.held


def test_batch_cap_and_budget_stop_admission():
    st = _state(max_batch=2, budget=10)
    st.pending.extend([_welch(0, 4), _welch(1, 4), _welch(2, 4)])
    assert _select(st) == [0, 1]                # batch cap
    st.used = 8
    assert _select(st) == []                    # 4 bytes do not fit in the 2 left
    st.used = 0
    assert _select(st) == [2]
    st.held[3] = collections.deque([_chunk(7, 3, nbytes=20)])
    st.pending.append(_welch(8, 1))
    assert _select(st) == []                    # the oldest waiting chunk does not fit: stop
    assert [r.rid for r in st.pending] == [8]


def test_backlog_selection_does_not_rescan():
    """A backlog of chunks of busy streams moves to the held queues once: later selections pop
    only what they admit."""
    st = _state(max_batch=16, nstreams=8)
    st.busy[:] = True
    st.pending.extend(_chunk(i, i % 8) for i in range(4000))
    st.pending.append(_welch(4000))
    assert _select(st) == [4000]
    assert sum(len(q) for q in st.held.values()) == 4000 and not st.pending
    st.busy[3] = False
    assert _select(st) == [3]
    assert sum(len(q) for q in st.held.values()) == 3999
