"""exafmm.modified_helmholtz -- Yukawa kernel G = exp(-k r)/(4 pi r), real k (include/modified_helmholtz.h).

As in the reference (python/exafmm.cpp:390, 423, 438, 488, 499, 532, 537) the body, node and
tree types and the charge functions are shared with the Laplace submodule."""
from functools import partial

from . import _core
from ._core import Bodies, ModifiedHelmholtzFmm, Node, Tree, clear_values, evaluate, init_targets, setup  # noqa
from ._core import update_charges  # noqa: F401

Body = Bodies
init_sources = partial(_core.init_sources, kernel="modified_helmholtz")


def gradient_p2p(src, q, trg, wavek, precision="fp64"):
    return _core.gradient_p2p("modified_helmholtz", src, q, trg, wavek, precision)
