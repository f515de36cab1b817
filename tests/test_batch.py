"""Batched systems in one captured CUDA graph (exafmm.batch over xfmm_batch_*): the graph replay of
the batched evaluate (concurrent per-system streams, one persistent near-field kernel over every
system's target leaves) gives the results of the same evaluates launched one by one bit for bit in
FP64, follows charges written in place, and each system agrees with FP64 direct summation to the
FMM's accuracy at p = 6."""
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
    shapes = ((0, 2), (2, 1))
    ns = b.autotune(candidates=(1, 2, 4), near_shapes=shapes, reps=2, tile_candidates=(1, 4))
    assert set(b.tuning) == {(s, c, t) for s in (1, 2, 4) for c, t in shapes}
    assert b.tuning[(ns, b.near_ctas_per_sm, b.near_tpl)] == min(b.tuning.values())
    assert set(b.tile_tuning) == {1, 4} and b.tile_tuning[b.tiles_per_cta] == min(b.tile_tuning.values())
    rep = b.replay()
    torch.cuda.synchronize()
    for a, c in zip(seq, rep):
        assert torch.equal(a, c)


def test_batched_evaluate_without_graph_equals_one_by_one_fp64():
    systems, b = _batch("fp64")
    seq = [o.clone() for o in b.evaluate_each()]
    for shape in ((0, 2), (1, 1)):
        b.set_near_shape(*shape)
        for o in b.outs:
            o.zero_()
        rep = b.evaluate_batch(nstreams=4)
        torch.cuda.synchronize()
        for a, c in zip(seq, rep):
            assert torch.equal(a, c)


def test_mixed_batch_matches_one_by_one():
    """Mixed path: the sparse M2L Hadamard adds its FP32 products with atomics, so two evaluates of the
    same system differ in rounding (order 1e-7 relative); the batch stays within 5e-7 of one by one."""
    systems, b = _batch("mixed")
    seq = [o.clone() for o in b.evaluate_each()]
    b.capture(nstreams=4)
    rep = b.replay()
    torch.cuda.synchronize()
    for a, c in zip(seq, rep):
        assert float(torch.linalg.norm(c - a) / torch.linalg.norm(a)) < 5e-7


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



def test_laplace_systems_share_one_operator_set():
    systems, b = _batch("fp64")
    assert b.n_operator_sets == 1 and len({round(t.dump()["r0"], 12) for t in b.trees}) > 1
    # each system against its own freshly precomputed operators (the reference's per-radius precompute)
    import exafmm.laplace as lap
    seq = [o.clone() for o in b.evaluate_each()]
    torch.cuda.synchronize()
    for (x, q), o in list(zip(systems, seq))[:3]:
        fmm = lap.LaplaceFmm(6, 64, precision="fp64")
        tree = lap.setup(lap.init_sources(x, q), lap.init_targets(x), fmm)
        own = lap.evaluate(tree, fmm)
        ref = o.cpu().numpy()
        rel = np.linalg.norm(own - ref) / np.linalg.norm(own)
        assert rel < 1e-9, rel


def test_yukawa_batch_keeps_one_operator_set_per_system():
    """Modified Helmholtz operators depend on the root radius: each system keeps its own, the batch runs
    the per-system M2L and far field and the generic persistent near-field kernel, and agrees with the
    systems evaluated one by one (the mixed path's sparse Hadamard adds with atomics: 5e-7)."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import exafmm.modified_helmholtz as Y
    from exafmm.batch import BatchedFmm, batched_workload
    systems = batched_workload(nsys=4, nmin=3000, nmax=12000, seed=5)
    b = BatchedFmm(systems, lambda: Y.ModifiedHelmholtzFmm(5, 64, 3.0, precision="mixed"))
    assert b.n_operator_sets == 4
    seq = [o.clone() for o in b.evaluate_each()]
    b.capture(nstreams=2)
    for o in b.outs:
        o.zero_()
    rep = b.replay()
    torch.cuda.synchronize()
    for a, c in zip(seq, rep):
        assert float(torch.linalg.norm(c - a) / torch.linalg.norm(a)) < 5e-7
