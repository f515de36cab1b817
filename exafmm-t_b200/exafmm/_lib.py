"""ctypes binding of libexafmm_b200.so (include/xfmm.h).

The library is built in-tree by ``make -C exafmm-t_b200`` (or ``__graft_entry__.build``).
There is no fallback: if the library is missing, importing ``exafmm`` fails loudly.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# XFMM_LIBRARY overrides the library file (e.g. a build with other compile-time tile sizes)
LIB_PATH = os.environ.get("XFMM_LIBRARY") or os.path.join(os.path.dirname(HERE), "libexafmm_b200.so")

STATUS = {
    0: "OK", 1: "invalid argument", 2: "out of memory", 3: "CUDA error", 4: "device wait timed out",
    5: "call order violated", 6: "unsupported configuration", 7: "numerical failure",
}
KERNEL_IDS = {"laplace": 0, "modified_helmholtz": 1, "helmholtz": 2}
PRECISIONS = {"fp64": 0, "mixed": 1}

# (name, restype, argtypes) for every entry point declared in include/xfmm.h
vp, i32, i64, f64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double
SIGNATURES = [
    ("xfmm_last_error", ctypes.c_char_p, []),
    ("xfmm_version", ctypes.c_char_p, []),
    ("xfmm_fmm_create", i32, [i32, i32, i32, f64, f64, i32, ctypes.POINTER(vp)]),
    ("xfmm_fmm_free", i32, [vp]),
    ("xfmm_fmm_set_operator_file", i32, [vp, ctypes.c_char_p]),
    ("xfmm_fmm_info", i32, [vp, vp, vp]),
    ("xfmm_build_tree", i32, [vp, vp, i64, vp, i64, i32, i32, vp, ctypes.POINTER(vp)]),
    ("xfmm_tree_free", i32, [vp]),
    ("xfmm_build_list", i32, [vp, vp, vp]),
    ("xfmm_m2l_setup", i32, [vp, vp, vp]),
    ("xfmm_precompute", i32, [vp, vp, vp]),
    ("xfmm_set_charges", i32, [vp, vp, vp, i32, vp]),
    ("xfmm_clear_values", i32, [vp, vp, vp]),
    ("xfmm_upward_pass", i32, [vp, vp, vp]),
    ("xfmm_downward_pass", i32, [vp, vp, vp]),
    ("xfmm_get_values", i32, [vp, vp, vp, i32, vp]),
    ("xfmm_evaluate", i32, [vp, vp, vp, i32, vp]),
    ("xfmm_tree_info", i32, [vp, vp]),
    ("xfmm_tree_dump", i32, [vp] * 17),
    ("xfmm_stage_times", i32, [vp, vp, vp]),
    ("xfmm_set_tuning", i32, [vp, i32, i32]),
    ("xfmm_batch_create", i32, [vp, vp, i32, vp, ctypes.POINTER(vp)]),
    ("xfmm_batch_evaluate", i32, [vp, vp, vp, i32, vp]),
    ("xfmm_batch_set_tuning", i32, [vp, i32, i32]),
    ("xfmm_batch_free", i32, [vp]),
    ("xfmm_batch_schedule", i32, [vp, i32, i32, vp]),
    ("xfmm_gradient_p2p", i32, [i32, f64, f64, i32, vp, i64, vp, vp, i64, vp, i32, vp]),
    ("xfmm_verify", i32, [vp, vp, i32, vp, vp]),
    ("xfmm_gradient_p2p_noalloc", i32, [i32, f64, f64, i32, vp, i64, vp, vp, i64, vp, vp]),
    ("xfmm_selftest_bounded_wait", i32, [i64]),
]


class FmmError(RuntimeError):
    """A non-OK xfmm_status; ``code`` is the status, the message is xfmm_last_error()."""

    def __init__(self, code, msg):
        super().__init__("%s (%s)" % (msg, STATUS.get(code, code)))
        self.code = code


_LIB = None


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError("libexafmm_b200.so not built: run `make -C %s`" % os.path.dirname(LIB_PATH))
    L = ctypes.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = L
    return L


def check(code):
    if code != 0:
        raise FmmError(code, lib().xfmm_last_error().decode(errors="replace"))


def ptr(a):
    """Pointer and on-device flag of a numpy array or a torch tensor."""
    if hasattr(a, "data_ptr") and hasattr(a, "is_cuda"):
        return ctypes.c_void_p(a.data_ptr()), int(bool(a.is_cuda))
    return a.ctypes.data_as(ctypes.c_void_p), 0
