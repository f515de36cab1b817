"""Host-side scheduling of a batch (xfmm_batch_schedule, no device work): how xfmm_batch_evaluate deals
the systems' per-system stages to its concurrent streams."""
import ctypes

import numpy as np


def _deal(sizes, nstreams):
    from exafmm import _lib
    n = len(sizes)
    s = np.asarray(sizes, dtype=np.int64)
    out = np.full(n, -1, dtype=np.int32)
    _lib.check(_lib.lib().xfmm_batch_schedule(s.ctypes.data_as(ctypes.c_void_p), n, nstreams,
                                              out.ctypes.data_as(ctypes.c_void_p)))
    lists = [[] for _ in range(max(out.max() + 1, 0) if n else 0)]
    order = sorted(range(n), key=lambda k: -sizes[k])  # stable: ties in index order
    for k in order:
        lists[out[k]].append(k)
    return out, lists


def test_every_system_on_exactly_one_stream():
    sizes = [5, 100, 40, 60, 7, 1, 33, 33]
    for ns in (1, 2, 3, 8, 20):
        out, lists = _deal(sizes, ns)
        assert sorted(i for l in lists for i in l) == list(range(8))
        assert out.min() >= 0 and out.max() < min(ns, 8)
        assert len(lists) == min(ns, 8)


def test_largest_first_to_the_least_loaded_stream():
    # 100 -> s0, 60 -> s1, 40 -> s2, then 7, 5 and 1 each to the lightest stream (s2 every time)
    assert _deal([5, 100, 40, 60, 7, 1], 3)[1] == [[1], [3], [2, 4, 0, 5]]
    assert _deal([5, 100, 40, 60, 7, 1], 1)[1] == [[1, 3, 2, 4, 0, 5]]


def test_loads_stay_within_the_largest_system():
    rng = np.random.default_rng(3)
    sizes = [int(v) for v in np.exp(rng.uniform(np.log(2000), np.log(200000), 256))]
    for ns in (4, 8, 16):
        out, lists = _deal(sizes, ns)
        load = [sum(sizes[k] for k in l) for l in lists]
        assert max(load) - min(load) <= max(sizes)


def test_bad_arguments_are_errors():
    from exafmm import _lib
    out = np.zeros(2, dtype=np.int32)
    s = np.ones(2, dtype=np.int64)
    rc = _lib.lib().xfmm_batch_schedule(s.ctypes.data_as(ctypes.c_void_p), 2, 0, out.ctypes.data_as(ctypes.c_void_p))
    assert rc != 0
    assert _lib.lib().xfmm_batch_schedule(None, 2, 2, None) != 0
