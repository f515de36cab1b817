"""Failure detection on the device without a fault: the library's waiting kernels (the tcgen05
Hadamard pipeline) bound every wait and report a wait that runs out through a device status flag.
The self-test entry point makes such a wait run out on purpose (an mbarrier phase that nothing
completes, about a millisecond) and the host reads the status; the device must stay usable."""
import numpy as np
import pytest

from oracle import orc

pytestmark = pytest.mark.gpu

XFMM_ERR_TIMEOUT = 4


def test_bounded_wait_reports_timeout_and_device_stays_usable():
    from exafmm import _lib
    import exafmm.laplace as L
    lib = _lib.lib()
    assert lib.xfmm_selftest_bounded_wait(2_000_000) == XFMM_ERR_TIMEOUT
    assert b"ran out" in lib.xfmm_last_error()
    # the context survives: an ordinary evaluate afterwards is correct
    rng = np.random.default_rng(4)
    x = rng.random((5000, 3))
    q = rng.uniform(-1, 1, 5000)
    fmm = L.LaplaceFmm(6, 64, precision="fp64")
    tree = L.setup(L.init_sources(x, q), L.init_targets(x), fmm)
    out = L.evaluate(tree, fmm)
    pe, ge = orc.rel_l2(out[:200], orc.direct("laplace", x, q, x[:200]))
    assert pe < 1e-5 and ge < 1e-4, (pe, ge)


def test_bounded_wait_rejects_bad_limit():
    from exafmm import _lib
    assert _lib.lib().xfmm_selftest_bounded_wait(0) == 1  # XFMM_ERR_ARG
