"""exafmm.helmholtz -- Helmholtz kernel G = exp(i k r)/(4 pi r), complex k and charges (include/helmholtz.h)."""
from functools import partial

from . import _core
from ._core import Bodies, HelmholtzFmm, Node, Tree, clear_values, evaluate, init_targets, setup  # noqa: F401
from ._core import update_charges  # noqa: F401

Body = Bodies
init_sources = partial(_core.init_sources, kernel="helmholtz")


def gradient_p2p(src, q, trg, wavek, precision="fp64"):
    return _core.gradient_p2p("helmholtz", src, q, trg, wavek, precision)
