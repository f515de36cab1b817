"""Batched systems in one captured CUDA graph (exafmm.batch): the graph replay gives the results of
the same evaluates launched one by one, follows charges written in place, and each system agrees
with FP64 direct summation to the FMM's accuracy at p = 6."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _batch(precision):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import exafmm.laplace as lap
    from exafmm.batch import BatchedFmm, batched_workload
    systems = batched_workload(nsys=8, nmin=2000, nmax=20000, seed=7)
    return systems, BatchedFmm(systems, lambda: lap.LaplaceFmm(6, 64, precision=precision))


def test_graph_replay_equals_one_by_one_fp64():
    systems, b = _batch("fp64")
    seq = [o.clone() for o in b.evaluate_each()]
    b.capture()
    rep = b.replay()
    torch.cuda.synchronize()
    for a, c in zip(seq, rep):
        assert torch.equal(a, c)


def test_graph_on_concurrent_streams_equals_one_by_one_fp64():
    systems, b = _batch("fp64")
    seq = [o.clone() for o in b.evaluate_each()]
    b.capture(nstreams=3)
    for o in b.outs:
        o.zero_()
    rep = b.replay()
    torch.cuda.synchronize()
    for a, c in zip(seq, rep):
        assert torch.equal(a, c)


def test_autotune_keeps_a_timed_stream_count():
    systems, b = _batch("fp64")
    seq = [o.clone() for o in b.evaluate_each()]
    ns = b.autotune(candidates=(1, 2, 4), reps=2, tile_candidates=(1, 4))
    assert ns in (1, 2, 4) and set(b.tuning) == {1, 2, 4}
    assert b.tuning[ns] == min(b.tuning.values())
    assert set(b.tile_tuning) == {1, 4} and b.tile_tuning[b.tiles_per_cta] == min(b.tile_tuning.values())
    rep = b.replay()
    torch.cuda.synchronize()
    for a, c in zip(seq, rep):
        assert torch.equal(a, c)


def test_graph_follows_charges_written_in_place():
    systems, b = _batch("mixed")
    b.capture()
    first = [o.clone() for o in b.replay()]
    for q in b.charges:
        q.mul_(2.0)
    second = b.replay()
    torch.cuda.synchronize()
    for a, c in zip(first, second):
        assert float(torch.linalg.norm(c - 2 * a) / torch.linalg.norm(2 * a)) < 1e-6


def test_batched_systems_match_direct_sums():
    from oracle import orc
    systems, b = _batch("mixed")
    b.capture()
    outs = b.replay()
    torch.cuda.synchronize()
    rng = np.random.default_rng(0)
    for (x, q), o in zip(systems[:4], outs[:4]):
        s = rng.choice(len(x), 200, replace=False)
        pe, ge = orc.rel_l2(o.cpu().numpy()[s], orc.direct("laplace", x, q, x[s]))
        assert pe < 1e-4 and ge < 1e-3, (pe, ge)

