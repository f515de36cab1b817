"""Parity of the CUDA path (through the C ABI) with the reference, on a B200.

Integer/tree work is compared bit for bit with fixtures produced by the reference
itself (tests/golden); FP64 potentials and gradients within 1e-9 relative L2 of the
reference's own FMM; the mixed path within 5e-6 of the reference at p=4..6 (its own
FMM truncation error dominates there) and against the FP64 direct-sum oracle."""
import numpy as np
import pytest

from oracle import fmm_np, orc
from tests.golden_cases import TREE_KEYS, case_names, load, load_p2p

pytestmark = pytest.mark.gpu

CASES = case_names()
FP64_TOL = 1e-9     # FP64 GPU vs reference FMM (same algorithm, different SVD/FFT libraries and sum order)
MIXED_TOL = 5e-6    # mixed GPU vs reference FMM at these small p


def _mod(kernel):
    import exafmm.helmholtz
    import exafmm.laplace
    import exafmm.modified_helmholtz
    return {"laplace": exafmm.laplace, "helmholtz": exafmm.helmholtz,
            "modified_helmholtz": exafmm.modified_helmholtz}[kernel]


def _fmm(g, precision):
    m = _mod(g["kernel"])
    if g["kernel"] == "laplace":
        return m.LaplaceFmm(g["p"], g["ncrit"], precision=precision)
    if g["kernel"] == "helmholtz":
        return m.HelmholtzFmm(g["p"], g["ncrit"], g["wavek"], precision=precision)
    return m.ModifiedHelmholtzFmm(g["p"], g["ncrit"], g["wavek"].real, precision=precision)


def _setup(g, precision):
    m = _mod(g["kernel"])
    fmm = _fmm(g, precision)
    tree = m.setup(m.init_sources(g["src"], g["q"]), m.init_targets(g["trg"]), fmm,
                   nonadaptive_depth=g["nonadaptive_depth"])
    return m, fmm, tree


@pytest.mark.parametrize("name", CASES)
def test_tree_and_lists_bit_exact(name):
    g = load(name)
    _, fmm, tree = _setup(g, "fp64")
    d = tree.dump()
    for k in TREE_KEYS:
        assert np.array_equal(d[k], g["tree"][k]), k
    assert d["depth"] == g["tree"]["depth"]
    assert d["r0"] == g["tree"]["r0"]
    assert fmm.depth == g["tree"]["depth"] and fmm.r0 == g["tree"]["r0"]


@pytest.mark.parametrize("kernel,wk,qkey", [("laplace", 0.0, "q"), ("modified_helmholtz", 10.0, "q"),
                                            ("helmholtz", 5.0 + 10.0j, "qc")])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 2e-6)])
def test_p2p_kernels_match_reference(kernel, wk, qkey, precision, tol):
    g = load_p2p()
    from exafmm import _core
    out = _core.gradient_p2p(kernel, g["src"], g[qkey], g["trg"], wk, precision)
    pe, ge = orc.rel_l2(out, g[kernel])
    assert pe < tol and ge < tol, (pe, ge)


@pytest.mark.parametrize("name", CASES)
def test_fmm_fp64_matches_reference(name):
    g = load(name)
    m, fmm, tree = _setup(g, "fp64")
    out = m.evaluate(tree, fmm)
    pe, ge = orc.rel_l2(out, g["out"])
    assert pe < FP64_TOL and ge < FP64_TOL, (pe, ge)


@pytest.mark.parametrize("name", CASES)
def test_fmm_mixed_matches_reference(name):
    g = load(name)
    m, fmm, tree = _setup(g, "mixed")
    out = m.evaluate(tree, fmm)
    pe, ge = orc.rel_l2(out, g["out"])
    assert pe < MIXED_TOL and ge < MIXED_TOL, (pe, ge)


def test_fmm_p8_against_oracle_and_direct():
    rng = np.random.default_rng(11)
    x = rng.random((20000, 3))
    q = rng.uniform(-1, 1, 20000)
    import exafmm.laplace as L
    ref = fmm_np.NpFmm("laplace", 8, 128).setup(x, q, x).evaluate()
    ex = orc.direct("laplace", x, q, x[:500])
    for prec, tol in (("fp64", 1e-10), ("mixed", 1e-6)):
        fmm = L.LaplaceFmm(8, 128, precision=prec)
        tree = L.setup(L.init_sources(x, q), L.init_targets(x), fmm)
        out = L.evaluate(tree, fmm)
        if prec == "fp64":
            pe, ge = orc.rel_l2(out, ref)
            assert pe < tol and ge < tol, (prec, pe, ge)
        pe, ge = orc.rel_l2(out[:500], ex)
        assert pe < 1e-6 and ge < 3e-6, (prec, pe, ge)


def test_update_charges_and_reevaluate():
    g = load("laplace_cube_p4")
    m, fmm, tree = _setup(g, "fp64")
    out1 = m.evaluate(tree, fmm)
    m.update_charges(tree, 2.0 * g["q"])
    m.clear_values(tree)
    out2 = m.evaluate(tree, fmm)
    assert np.allclose(out2, 2.0 * out1, rtol=1e-12, atol=1e-12 * np.abs(out1).max())


@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_update_charges_rejects_non_finite_and_keeps_the_old_charges(bad):
    g = load("laplace_cube_p4")
    m, fmm, tree = _setup(g, "fp64")
    out1 = m.evaluate(tree, fmm)
    q = g["q"].copy()
    q[len(q) // 2] = bad
    with pytest.raises(RuntimeError, match="non-finite value in charges"):
        m.update_charges(tree, q)
    out2 = m.evaluate(tree, fmm)
    assert np.array_equal(out1, out2)


def test_verify_matches_oracle():
    g = load("laplace_cube_p4")
    m, fmm, tree = _setup(g, "fp64")
    out = m.evaluate(tree, fmm)
    e = fmm.verify(tree.leafs, sample=False)
    pe, ge = orc.rel_l2(out, orc.direct("laplace", g["src"], g["q"], g["trg"]))
    assert abs(e[0] - pe) < 1e-3 * pe and abs(e[1] - ge) < 1e-3 * ge


F32_CASES = ["f32ref_laplace_cube_p8", "f32ref_yukawa_sphere_p6"]


@pytest.mark.parametrize("name", F32_CASES)
def test_mixed_matches_the_reference_single_precision_build(name):
    """The mixed path against the reference's own FP32 FMM (-DFLOAT build, same inputs): at least as
    accurate against FP64 direct sums at every target, and its output within the two errors of the
    reference build's output."""
    from golden_cases import load_f32ref
    g = load_f32ref(name)
    mod = {"laplace": "exafmm.laplace", "modified_helmholtz": "exafmm.modified_helmholtz"}[g["kernel"]]
    import importlib
    m = importlib.import_module(mod)
    fmm = m.LaplaceFmm(g["p"], g["ncrit"], precision="mixed") if g["kernel"] == "laplace" else \
        m.ModifiedHelmholtzFmm(g["p"], g["ncrit"], g["wavek"].real, precision="mixed")
    tree = m.setup(m.init_sources(g["src"], g["q"]), m.init_targets(g["src"]), fmm)
    out = m.evaluate(tree, fmm)
    ex = g["direct"]  # FP64 direct sums at every target
    ours = orc.rel_l2(out, ex)
    theirs = orc.rel_l2(g["out32"], ex)
    assert ours[0] <= theirs[0] and ours[1] <= theirs[1], (ours, theirs)
    diff = orc.rel_l2(out, g["out32"])  # triangle bound: within the two errors
    assert diff[0] <= 1.01 * (ours[0] + theirs[0]) and diff[1] <= 1.01 * (ours[1] + theirs[1]), (diff, ours, theirs)


def test_hadamard_tcgen05_form(monkeypatch):
    """The dense M2L Hadamard on tcgen05 (TMEM operands, single-thread MMA issue; chosen per workspace by
    XFMM_HADAMARD_TCGEN05=1) against the default mma.sync form and the FP64 direct sum."""
    import exafmm.laplace as L
    rng = np.random.default_rng(5)
    x = rng.random((60000, 3))
    q = rng.uniform(-1, 1, 60000)
    ex = orc.direct("laplace", x, q, x[:400])
    outs = []
    for flag in ("0", "1"):
        monkeypatch.setenv("XFMM_HADAMARD_TCGEN05", flag)
        fmm = L.LaplaceFmm(8, 64, precision="mixed")
        tree = L.setup(L.init_sources(x, q), L.init_targets(x), fmm)
        out = L.evaluate(tree, fmm)
        fmm.stage_times(tree)  # raises if a bounded device wait ran out
        pe, ge = orc.rel_l2(out[:400], ex)
        assert pe < 1e-6 and ge < 3e-6, (flag, pe, ge)
        outs.append(out)
    pe, ge = orc.rel_l2(outs[1], outs[0])
    assert pe < 5e-7 and ge < 5e-7, (pe, ge)


# Orders beyond the fixtures: the slabbed real transforms at p = 3 (one partial slab), p = 9 (odd order:
# a partial last slab) and p = 10 (the other occupancy setting), and the complex transforms at p = 3, 9
# and 12, against FP64 direct sums (bounded by the FMM's truncation error at that order); the mixed path
# also against the FP64 path on the same tree.
@pytest.mark.parametrize("kernel,p,wk", [("laplace", 3, 0.0), ("laplace", 9, 0.0), ("laplace", 10, 0.0),
                                         ("helmholtz", 3, 5.0), ("helmholtz", 9, 20.0), ("helmholtz", 12, 20.0)])
def test_high_orders_against_direct_sums(kernel, p, wk):
    rng = np.random.default_rng(11)
    n = 20000
    x = rng.random((n, 3))
    q = rng.uniform(-1, 1, n)
    if kernel == "helmholtz":
        q = q + 1j * rng.uniform(-1, 1, n)
    m = _mod(kernel)
    outs = {}
    for prec in ("fp64", "mixed"):
        fmm = (m.LaplaceFmm(p, 64, precision=prec) if kernel == "laplace"
               else m.HelmholtzFmm(p, 64, wk, precision=prec))
        tree = m.setup(m.init_sources(x, q), m.init_targets(x), fmm)
        outs[prec] = m.evaluate(tree, fmm)
    s = rng.choice(n, 300, replace=False)
    ex = orc.direct(kernel, x, q, x[s], wk)
    pe, ge = orc.rel_l2(outs["fp64"][s], ex)
    bound = 5e-2 if p == 3 else 1e-4                 # the FMM's own truncation error at this order
    assert pe < bound and ge < 10 * bound, (pe, ge)
    pm, gm = orc.rel_l2(outs["mixed"], outs["fp64"])
    assert pm < 5e-6 and gm < 5e-6, (pm, gm)        # mixed precision against FP64 on the same tree


# Orders past the own transform kernels (real p > 10, complex p > 12): the M2L runs on cuFFT over the
# materialised convolution grids (k_m2l_grid_up, cuFFT R2C/C2C and the inverse, transposes to and from the
# Hadamard's frequency-major layout), the per-level kernels with one plan pair per level.
@pytest.mark.parametrize("kernel,p,wk", [("laplace", 12, 0.0), ("modified_helmholtz", 11, 5.0),
                                         ("helmholtz", 13, 10.0 + 0.0j)])
def test_cufft_fallback_orders_against_direct_sums(kernel, p, wk):
    rng = np.random.default_rng(12)
    n = 12000
    x = rng.random((n, 3))
    q = rng.uniform(-1, 1, n)
    if kernel == "helmholtz":
        q = q + 1j * rng.uniform(-1, 1, n)
    m = _mod(kernel)
    outs = {}
    for prec in ("fp64", "mixed"):
        if kernel == "laplace":
            fmm = m.LaplaceFmm(p, 64, precision=prec)
        elif kernel == "modified_helmholtz":
            fmm = m.ModifiedHelmholtzFmm(p, 64, float(np.real(wk)), precision=prec)
        else:
            fmm = m.HelmholtzFmm(p, 64, complex(wk), precision=prec)
        tree = m.setup(m.init_sources(x, q), m.init_targets(x), fmm)
        outs[prec] = m.evaluate(tree, fmm)
        fmm.stage_times(tree)  # raises if a bounded device-side wait ran out
    s = rng.choice(n, 300, replace=False)
    ex = orc.direct(kernel, x, q, x[s], wk) if kernel != "laplace" else orc.direct(kernel, x, q, x[s])
    pe, ge = orc.rel_l2(outs["fp64"][s], ex)
    assert pe < 1e-5 and ge < 1e-4, (pe, ge)         # the FMM's own truncation error at this order
    pm, gm = orc.rel_l2(outs["mixed"], outs["fp64"])
    assert pm < 5e-6 and gm < 5e-6, (pm, gm)        # mixed precision against FP64 on the same tree


def test_sparse_hadamard_tile_option():
    """xfmm_set_tuning: the sparse Hadamard's tiles per CTA change the launch, not the result (beyond
    the mixed path's run-to-run rounding); out-of-range values are rejected."""
    import exafmm.laplace as L
    from exafmm._lib import FmmError
    rng = np.random.default_rng(3)
    x = rng.random((60000, 3))
    q = rng.uniform(-1, 1, 60000)
    fmm = L.LaplaceFmm(8, 64, precision="mixed")
    tree = L.setup(L.init_sources(x, q), L.init_targets(x), fmm)
    base = L.evaluate(tree, fmm)
    for tiles in (1, 3, 64, 0):
        tree.set_tuning("sparse_hadamard_tiles_per_cta", tiles)
        pe, ge = orc.rel_l2(L.evaluate(tree, fmm), base)
        assert pe < 1e-6 and ge < 1e-6, (tiles, pe, ge)
    with pytest.raises(FmmError):
        tree.set_tuning("sparse_hadamard_tiles_per_cta", 65)
