"""The C-ABI library loads and exports every entry point declared in include/xfmm.h (no GPU needed)."""
import os
import re

from tests.conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "xfmm.h")).read()
    return sorted(set(re.findall(r"\b(xfmm_[a-z0-9_]+)\s*\(", src)))


def test_header_lists_entry_points():
    names = _declared()
    assert "xfmm_evaluate" in names and "xfmm_build_tree" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    from exafmm import _lib
    L = _lib.lib()
    for name in _declared():
        assert hasattr(L, name), name
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert bound == set(_declared())


def test_status_without_gpu_is_an_error_not_a_crash():
    import numpy as np
    import exafmm.laplace as L
    from exafmm._lib import FmmError
    f = L.LaplaceFmm(4, 32)
    assert f.nsurf == 56 and f.nfreq == 8 * 8 * 5
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    x = np.random.default_rng(0).random((50, 3))
    try:
        L.setup(L.init_sources(x, np.ones(50)), L.init_targets(x), f)
    except FmmError as e:
        assert e.code in (3, 2)
    else:
        raise AssertionError("setup without a GPU must fail loudly")


def test_argument_errors():
    import numpy as np
    import exafmm.laplace as L
    from exafmm._lib import FmmError
    try:
        L.LaplaceFmm(1, 32)
    except FmmError as e:
        assert e.code == 6
    else:
        raise AssertionError("p=1 must be rejected")
    try:
        L.init_sources(np.zeros((5, 2)), np.zeros(5))
    except RuntimeError as e:
        assert "(n, 3)" in str(e)
    else:
        raise AssertionError
    try:
        L.init_sources(np.zeros((5, 3)), np.zeros(4))
    except RuntimeError as e:
        assert "must match" in str(e)
    else:
        raise AssertionError


def test_tuning_option_arguments_checked_without_a_gpu():
    from exafmm import _lib
    L = _lib.lib()
    assert L.xfmm_set_tuning(None, 1, 4) == 1  # XFMM_ERR_ARG: no tree
    assert b"null" in L.xfmm_last_error()
