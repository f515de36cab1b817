"""Host-side scheduling of exafmm.batch.BatchedFmm (no device work): how systems are dealt to the
concurrent streams of the captured graph."""
import pytest

pytest.importorskip("torch")


def _dealer(sizes):
    from exafmm.batch import BatchedFmm
    b = BatchedFmm.__new__(BatchedFmm)  # only the sizes are needed to deal
    b.n = list(sizes)
    return b


def test_every_system_on_exactly_one_stream():
    b = _dealer([5, 100, 40, 60, 7, 1, 33, 33])
    for ns in (1, 2, 3, 8, 20):
        lists = b._deal(ns)
        assert sorted(i for l in lists for i in l) == list(range(8))
        assert len(lists) == min(ns, 8)


def test_largest_first_to_the_least_loaded_stream():
    b = _dealer([5, 100, 40, 60, 7, 1])
    # 100 -> s0, 60 -> s1, 40 -> s2, then 7, 5 and 1 each to the lightest stream (s2 every time)
    assert b._deal(3) == [[1], [3], [2, 4, 0, 5]]
    assert b._deal(1) == [[1, 3, 2, 4, 0, 5]]
