"""exafmm -- B200 (sm_100a) implementation of exafmm-t's KIFMM evaluate path.

Drop-in for the reference's pybind11 module ``exafmm`` (python/exafmm.cpp:325-563):
the submodules ``laplace``, ``helmholtz`` and ``modified_helmholtz`` expose the same
classes and functions.  All compute runs in libexafmm_b200.so on the GPU.
"""
from . import _lib
from . import laplace, helmholtz, modified_helmholtz  # noqa: F401

# Load the library now: its CUDA libraries (cuBLAS, cuFFT, cuSOLVER of the toolkit it was built with)
# are then the ones the process uses, also for modules imported later that bundle older copies under
# the same names.  Import exafmm before torch to get them.
_lib.lib()

__all__ = ["laplace", "helmholtz", "modified_helmholtz"]


def version():
    return _lib.lib().xfmm_version().decode()
