"""exafmm.laplace -- Laplace kernel G = 1/(4 pi r) (include/laplace.h)."""
from functools import partial

from . import _core
from ._core import Bodies, LaplaceFmm, Node, Tree, clear_values, evaluate, init_targets, setup  # noqa: F401
from ._core import update_charges  # noqa: F401

Body = Bodies
init_sources = partial(_core.init_sources, kernel="laplace")
gradient_p2p = partial(_core.gradient_p2p, "laplace")
